"""Benchmark of the exhaustive pairwise epistasis scan on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload cfg3] [--form auto|popc|tensor]
    python bench.py --impl reference ...      the reference's own kernels on the host cores

A step is one full scan of the workload's SNP pairs (test 8 df + 4 df unless the workload
says otherwise) over synthetic data of the workload's shape. `value` is pairs/s with the
genotypes and traits already resident in HBM; `e2e` is the same metric through the C ABI
from host buffers (genotype + trait upload, scan, hit readback inside the timed region).
Multi-GPU (torchrun): every rank scans its own replica of the workload (weak scaling, no
collective on the data path); times are device times, max over ranks.
Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SNP pairs/sec (8df & 4df) on 1 B200: tensor-core vs popcount form, F err<=1e-5"

WORKLOADS = {
    # name: (nid, chromosome sizes, test, traits, description)
    "cfg1": (500, [2000], "f", 1, "plain 8 df scan, N=500 individuals, M=2,000 SNPs, 1 chromosome"),
    "cfg2": (4000, [10000, 10000], "i", 1, "8 df + 4 df scan, N=4,000, M=20,000 SNPs on 2 chromosomes"),
    "cfg3": (10000, [100000], "i", 1, "8 df + 4 df scan, N=10,000 individuals, M=100,000 SNPs, 1 chromosome"),
    "cfg4": (5000, [50000], "f", 64, "8 df scan, N=5,000, M=50,000, 64 phenotype columns (permutations)"),
    "cfg5": (8000, None, "f", 8, "8 df scan, N=8,000, 22 uneven blocks (M=250,000), 8 traits with own masks"),
    # the cfg3 kernel on a block small enough for an ncu capture of one launch
    "cfg3s": (10000, [4000], "i", 1, "8 df + 4 df scan, N=10,000 individuals, M=4,000 SNPs (profiling size)"),
    # the cfg3 kernel with operands larger than L2 (DRAM traffic per pair as in cfg3)
    "cfg3m": (10000, [20000], "i", 1, "8 df + 4 df scan, N=10,000 individuals, M=20,000 SNPs (traffic capture)"),
}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# planted interacting pairs (snp1, snp2) and the share of the phenotypic variance each
# explains: configuration 2 (5 pairs at 0.5%, two of them between the chromosomes) and
# configuration 4 (3 pairs in column 0; the permuted columns carry none)
PLANTED = {
    "cfg2": ([(1500, 300), (12000, 4000), (18500, 11000), (10005, 9995), (9000, 8990)], 0.005),
    "cfg4": ([(31000, 2000), (45000, 44000), (20000, 19000)], 0.02),
}


def workload_data(name, seed=1):
    from epigpu_b200 import synth
    nid, sizes, test, ntraits, desc = WORKLOADS[name]
    if sizes is None:
        sizes = synth.uneven_block_sizes()
    nsnp = sum(sizes)
    gp = synth.packed_on_gpu(nid, nsnp, seed=seed)
    rng = np.random.default_rng(seed + 7)
    planted = PLANTED.get(name)
    if ntraits == 1 and planted:
        pairs, frac = planted
        y = synth.planted_phenotype(synth.planted_rows(gp, nid, pairs), pairs, seed=seed + 1, var_frac=frac,
                                    miss=0.01)
        valid = None
    elif ntraits == 1:
        y = synth.phenotype(nid, seed=seed + 1, miss=0.02 if name == "cfg1" else 0.01)
        valid = None
    elif name == "cfg4":
        from epigpu_b200 import capi
        pairs, frac = planted
        base = synth.planted_phenotype(synth.planted_rows(gp, nid, pairs), pairs, seed=seed + 1, var_frac=frac,
                                       miss=0.0)
        cols = [base] + [capi.permute_phenotype(base, p) for p in range(1, ntraits)]
        y = np.stack(cols, 1)
        valid = np.repeat((rng.random(nid) >= 0.01)[:, None], ntraits, 1)
    else:
        cols, vcols = [], []
        for t in range(ntraits):
            if t % 2 == 0:
                v = rng.standard_normal(nid)
            else:
                v = (rng.gamma(2.0, 1.0, nid) - 2.0) / np.sqrt(2.0)
            cols.append(v.astype(np.float32))
            vcols.append(rng.random(nid) >= rng.uniform(0.0, 0.10))
        y = np.stack(cols, 1)
        valid = np.stack(vcols, 1)
    starts = np.cumsum([0] + sizes[:-1])
    blocks = [(int(starts[i]), sizes[i], int(starts[j]), sizes[j]) for i in range(len(sizes)) for j in range(i + 1)]
    return dict(nid=nid, nsnp=nsnp, sizes=sizes, test=test, ntraits=ntraits, desc=desc, gpack=gp, y=y,
                valid=valid, blocks=blocks, planted=planted[0] if planted else [])


def f_error_sample(ctx, data, form, t1, t2, side=1000, seed=11):
    """F and F2 of every pair of a seeded side x side block (side^2 pairs, both SNP ranges
    inside the first chromosome block, the first above the second) from the GPU form against
    the FP64 oracle, trait 0. Error per pair |F - F_oracle| / max(|F_oracle|, 1): relative
    for F >= 1, absolute below; pairs with df1 = 0 (F undefined) are left out."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    from epigpu_b200 import capi, synth
    nid, m0 = data["nid"], data["sizes"][0]
    side = min(side, m0 // 2)
    rng = np.random.default_rng(seed)
    s2 = int(rng.integers(0, m0 // 2 - side + 1))
    s1 = int(rng.integers(max(m0 // 2, s2 + side), m0 - side + 1))
    blk = (s1, side, s2, side)
    y = data["y"][:, 0] if data["y"].ndim == 2 else data["y"]
    phen = y if data["valid"] is None else np.where(data["valid"][:, 0], y, np.float32(-9.0)).astype(np.float32)
    d = ctx.scan_dump(blk, capi.default_opts(test="i", t1=t1, t2=t2, form=form), trait=0)
    codes = synth.unpack(np.concatenate([data["gpack"][s2:s2 + side], data["gpack"][s1:s1 + side]]), nid)
    _, _, pb = oracles.oracle_scan_block(codes, phen, (side, side, 0, side), test="i", t1=t1, t2=t2, per_pair=True)
    out = {"pairs": side * side, "block": list(blk), "trait": 0,
           "counts_exact": bool(np.array_equal(d["counts"], pb["counts"])),
           "df_exact": bool(np.array_equal(d["df1"], pb["df1"]) and np.array_equal(d["df2"], pb["df2"]))}
    ok = pb["df1"] > 0
    for f in ("F", "F2"):
        ref = pb[f][ok]
        e = np.abs(d[f][ok].astype(np.float64) - ref) / np.maximum(np.abs(ref), 1.0)
        out[f] = {"max": float(e.max()), "median": float(np.median(e))}
    return out


def thresholds(nid):
    from epigpu_b200 import synth
    return synth.f_threshold(8, nid - 9, 1e-6), synth.f_threshold(4, nid - 9, 1e-6)


def max_over_ranks(x, pg, device="cuda"):
    """The largest x over all ranks, on every rank (x itself without a process group): a
    multi-GPU time is the slowest rank's."""
    if not pg:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def block_pairs(b):
    s1, m1, s2, m2 = b
    gx = np.arange(m1, dtype=np.int64)
    return int(np.clip(gx + s1 - s2, 0, m2).sum())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        # nvidia-smi's start-up (driver queries) must not overlap a short timed region: wait
        # for its first sample
        t0 = time.time()
        while self.proc and not self.lines and self.proc.poll() is None and time.time() - t0 < 5.0:
            time.sleep(0.01)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def int8_peak_tops():
    """cuBLAS int8 GEMM throughput on this GPU (torch._int_mm, 8192^3, best of 10), TOP/s."""
    import torch
    n = 8192
    a = torch.randint(-8, 8, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-8, 8, (n, n), dtype=torch.int8, device="cuda")
    for _ in range(3):
        torch._int_mm(a, b)
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def cpu_baseline(data, test, t1, t2, budget_s=12.0, min_m=200):
    """The reference's own kernels (oracle A, built from its sources) on the host cores,
    over a bounded sample: a triangle of the workload's first m SNPs at the workload's N,
    sized to about `budget_s` seconds."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    if not oracles.have_ref():
        return None
    from epigpu_b200 import capi
    nid = data["nid"]
    y = data["y"][:, 0] if data["y"].ndim == 2 else data["y"]
    threads = os.cpu_count() or 1
    gp = data["gpack"]

    def run(m):
        blk = (0, m, 0, m)
        t = time.perf_counter()
        _, total = oracles.ref_scan_block(gp[:m], nid, y, blk, test=test, t1=t1, t2=t2, cap=1 << 16,
                                          nthreads=threads)
        return time.perf_counter() - t, m * (m - 1) // 2

    # small samples run below the threads' full rate (start-up), so the size is refined from
    # each run until one takes at least half the budget
    m = min_m
    for _ in range(4):
        dt, pairs = run(m)
        if dt >= 0.5 * budget_s or m >= data["nsnp"]:
            break
        m = int(min(data["nsnp"], max(m + 1, (2 * pairs / dt * budget_s) ** 0.5)))
    return {"value": pairs / dt, "unit": "pairs/s", "cores": threads, "kind": "reference",
            "sample": "triangle of the first %d SNPs at N=%d (%d pairs, %s test), %.1f s" % (m, nid, pairs,
                                                                                         "8df+4df" if test == "i"
                                                                                         else "8df", dt)}


DATAMODE_METRIC = "PLINK .ped/.map -> .epigpu conversion (epiGPU -Dr), MB of .ped text per second"


def run_datamode(args):
    """The data mode beside the scan (host C, one thread): `epiGPU -Dr` converting a seeded
    PLINK fileset of 2,000 individuals x 5,000 SNPs (40 MB of .ped text) to .epigpu, K timed runs
    after W warm-up runs; with --impl reference the reference's own readplink.c functions
    (oracle/_ref/plinkref, built from its sources) on the same files. The two outputs are
    compared byte for byte."""
    import tempfile
    from epigpu_b200 import synth
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cli = ROOT / "epigpu_b200" / "bin" / "epiGPU"
    ref = ROOT / "oracle" / "_ref" / "plinkref"
    reference = args.impl == "reference"
    exe = ref if reference else cli
    if not exe.exists():
        print(json.dumps({"impl": args.impl, "unavailable": "%s is not built" % exe.relative_to(ROOT)}))
        return 0
    nid, nsnp = 2000, 5000
    with tempfile.TemporaryDirectory() as tmp:
        d = pathlib.Path(tmp)
        ped, mp = synth.write_plink_fileset(d, nid, nsnp, seed=1)
        mb = ped.stat().st_size / 1e6
        out = d / "out.epigpu"
        cmd = [str(ref), "write", str(ped), str(mp), str(out)] if reference else [str(cli), "-Dr", str(ped), str(mp),
                                                                                  str(out)]
        times = []
        for step in range(args.warmup + args.steps):
            t = time.perf_counter()
            subprocess.run(cmd, check=True, capture_output=True)
            if step >= args.warmup:
                times.append(time.perf_counter() - t)
        same = None
        other = cli if reference else ref
        if other.exists():
            cmp = d / "other.epigpu"
            ocmd = [str(cli), "-Dr", str(ped), str(mp), str(cmp)] if reference else [str(ref), "write", str(ped),
                                                                                      str(mp), str(cmp)]
            subprocess.run(ocmd, check=True, capture_output=True)
            same = out.read_bytes() == cmp.read_bytes()
    value = mb * len(times) / sum(times)
    line = {
        "metric": DATAMODE_METRIC, "value": value, "unit": "MB/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "none", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "datamode: PLINK text %d individuals x %d SNPs (%.1f MB .ped)" % (nid, nsnp, mb),
                   "identical_to_other_arm": same},
        "e2e": {"value": value, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "roofline": None, "cpu_baseline": None,
    }
    if reference:
        line["impl"] = "reference"
        line["cpu_baseline"] = {"value": value, "unit": "MB/s", "cores": 1, "kind": "reference",
                                "sample": "the reference's dims/readped/readmap/pack/createpackedbinary on the fileset"}
    print(json.dumps(line))
    return 0


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    name = args.workload
    nid, sizes, test, ntraits, desc = WORKLOADS[name]
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    if not oracles.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libepiref.so (the reference's kernels "
                                                              "built from its sources) is missing"}))
        return 0
    from epigpu_b200 import synth
    nsnp = 4000
    codes = synth.genotype_codes(nid, nsnp, seed=1)
    gp = synth.pack(codes)
    y = synth.phenotype(nid, seed=2, miss=0.01)
    t1, t2 = thresholds(nid)
    threads = os.cpu_count() or 1
    # size the per-step sample to ~8 s on this host; small probes run below the threads' full
    # rate, so the size is refined from each probe until one takes at least half of that
    m = 150
    for _ in range(4):
        t = time.perf_counter()
        oracles.ref_scan_block(gp[:m], nid, y, (0, m, 0, m), test=test, t1=t1, t2=t2, cap=1 << 16,
                               nthreads=threads)
        dt = time.perf_counter() - t
        if dt >= 4.0 or m >= nsnp:
            break
        m = int(min(nsnp, max(m + 1, (2 * (m * (m - 1) / 2) / dt * 8.0) ** 0.5)))
    pairs = m * (m - 1) // 2
    times = []
    for step in range(args.warmup + args.steps):
        t = time.perf_counter()
        oracles.ref_scan_block(gp[:m], nid, y, (0, m, 0, m), test=test, t1=t1, t2=t2, cap=1 << 16,
                               nthreads=threads)
        if step >= args.warmup:
            times.append(time.perf_counter() - t)
    total = sum(times)
    value = pairs * len(times) / total
    sample = ("each step: the reference's OpenCL pair kernels (built as C from its sources) emulating "
              "perform_scan's launches on %d host threads over a triangle of %d SNPs at N=%d (%d pairs)"
              % (threads, m, nid, pairs))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "%s: %s" % (name, desc), "nid": nid, "pairs_per_step": pairs},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=sorted(WORKLOADS) + ["datamode"],
                    help="a scan configuration, or `datamode`: the host's PLINK -> .epigpu conversion")
    ap.add_argument("--form", default="auto", choices=["auto", "popc", "tensor"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", type=int, default=0,
                    help="kernel variant of the form (the scan option tile_config; 0 = the autotuner's choice)")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch each scan's device work directly instead of replaying its captured CUDA graph")
    ap.add_argument("--popc-sample", type=int, default=20000,
                    help="SNPs in the square sample used to time the popcount form next to the tensor form")
    ap.add_argument("--f-err-side", type=int, default=1000,
                    help="side of the square block whose pairs' F error against the FP64 oracle is reported "
                         "(0 = none)")
    args = ap.parse_args()
    if args.workload == "datamode":
        return run_datamode(args)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from epigpu_b200 import capi
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    data = workload_data(args.workload, seed=1 + rank)
    nid, test = data["nid"], data["test"]
    t1, t2 = thresholds(nid)
    form = {"auto": capi.FORM_AUTO, "popc": capi.FORM_POPC, "tensor": capi.FORM_TENSOR}[args.form]
    ctx = capi.Context(local)
    gname, sms = ctx.device_info()
    gp, y, valid = data["gpack"], data["y"], data["valid"]
    ntraits = data["ntraits"]
    opts = capi.default_opts(test=test, t1=t1, t2=t2, form=form, report_trait=0, no_graph=int(args.no_graph),
                             tile_config=args.tile)
    blocks = data["blocks"]
    pairs_step = sum(block_pairs(b) for b in blocks) * ntraits

    def load():
        ctx.load_packed(gp, nid)
        if valid is None:
            ctx.set_phenotype(y)
        else:
            ctx.set_traits(y, valid)

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    load()
    # device-resident throughput
    for _ in range(args.warmup):
        ctx.scan(blocks, opts, ntraits=ntraits)
    kernel_ms, launches = [], 0
    barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nhits = 0
        for _ in range(args.steps):
            hits, n, ex = ctx.scan(blocks, opts, ntraits=ntraits)
            ms, _, nl, used = ctx.last_timing()
            kernel_ms.append(ms)
            launches += nl
            nhits = n
        e1.record(stream)
        barrier()
        dev_s = e0.elapsed_time(e1) / 1e3
    dev_s = max_over_ranks(dev_s, pg)
    value = pairs_step * args.steps * world / dev_s
    kernel_config = ctx.scan_config()
    used_form = "tensor" if used == capi.FORM_TENSOR else "popc"

    # end to end through the C ABI from host buffers
    for _ in range(max(1, args.warmup // 2)):
        load()
        ctx.scan(blocks, opts, ntraits=ntraits)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        load()
        hits, n, ex = ctx.scan(blocks, opts, ntraits=ntraits)
    e1.record(stream)
    barrier()
    e2e_s = e0.elapsed_time(e1) / 1e3
    e2e_s = max_over_ranks(e2e_s, pg)
    h2d = gp.nbytes + y.nbytes + (valid.nbytes if valid is not None else 0)
    d2h = n * 32 + 64

    # popcount form on a square sample, when the headline form is the tensor form
    popc = None
    if used_form == "tensor" and args.popc_sample > 0:
        m = min(args.popc_sample, data["sizes"][0])
        popc_blocks = [(0, m, 0, m)]
        po = capi.default_opts(test=test, t1=t1, t2=t2, form=capi.FORM_POPC)
        ctx.scan(popc_blocks, po, ntraits=ntraits)
        ctx.scan(popc_blocks, po, ntraits=ntraits)
        ms, pp, _, _ = ctx.last_timing()
        popc = {"value": pp / (ms / 1e3), "unit": "pairs/s", "sample": "%d-SNP triangle" % m,
                "kernel": ctx.scan_config()}

    # planted pairs among the last step's hits (trait 0)
    found = set(zip(hits["snp1"].tolist(), hits["snp2"].tolist()))
    planted = {"pairs": len(data["planted"]), "recovered": sum(1 for p in data["planted"] if tuple(p) in found)}

    out = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        clocks = clk.summary()
        kern_s = statistics.mean(kernel_ms) / 1e3
        pairs_launch = pairs_step
        if used_form == "tensor":
            int8 = int8_peak_tops()
            # algorithmic int8 ops per pair: 3 genotype rows x 12 column types (3 genotypes x
            # {count, 3 y digits}) per individual; the 256 x 256 pair tile of 80 x 21 pairs
            # carries 39.0 (8 padding rows per CTA, 4 zero columns)
            ops_pair = 2.0 * 36.0 * nid
            achieved = pairs_launch * ops_pair / kern_s / 1e12
            # DRAM bytes per launch: the ncu capture of the same kernel on the cfg3m workload
            # (N=10,000, M=20,000, operands larger than L2) read and wrote 16.89 GB for
            # 199,990,000 pairs over Np = 10,112 padded individuals; the j rows are streamed
            # once per i tile, so the bytes scale with pairs x Np
            np_pad = (nid + 127) // 128 * 128
            traffic = 16.89e9 / (199990000.0 * 10112.0) * pairs_launch * np_pad
            # peak: twice the dense bf16 rate of MEASURED_PEAKS.json (dense int8 runs at twice
            # bf16; the file holds no int8 figure); beside it, a cuBLAS int8 GEMM timed in this run
            bf16x2 = 2.0 * peaks["bf16_tflops"]
            roof = {"bound": "tensor", "achieved": achieved, "peak": bf16x2, "unit": "TOP/s",
                    "frac": achieved / bf16x2,
                    "peak_source": "2 x dense bf16 of MEASURED_PEAKS.json (%s, %.1f TFLOP/s burst)"
                                   % (peak_kind, peaks["bf16_tflops"]),
                    "cublas_int8_same_run": int8, "frac_of_cublas_int8_same_run": achieved / int8,
                    # the same against the sustained (power-capped) bf16 figure of the file
                    "frac_of_2x_sustained_bf16": (achieved / (2.0 * peaks["bf16_tflops_sustained"])
                                                  if peaks.get("bf16_tflops_sustained") else None),
                    "traffic": traffic, "traffic_unit": "bytes per launch",
                    "traffic_source": "ncu dram__bytes_read+write on cfg3m, scaled by pairs x individuals"}
        else:
            # plain form: 4 FP32 adds per pair and individual (the dense 2 x 2 genotype cells;
            # the rest of the 3 x 3 table and the sum of squares come from per-SNP marginals)
            # against the FP32 pipe's peak at the sampled SM clock; beside it, the same rate in
            # the reference method's 10 FP32 operations per pair and individual (9 cell sums and
            # the sum of squares, src/EpiOpenCL.c:110-228)
            mhz = clocks["sm_mhz"] or 1965.0
            peak = sms * 128 * mhz * 1e6 / 1e12
            achieved = pairs_launch * 4.0 * nid / kern_s / 1e12
            roof = {"bound": "alu", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "reference_method_frac": pairs_launch * 10.0 * nid / kern_s / 1e12 / peak,
                    "peak_source": "%d SMs x 128 FP32 lanes x %.0f MHz sampled SM clock" % (sms, mhz)}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(data, test, t1, t2)
        ferr = None
        if args.f_err_side > 0:
            ferr = f_error_sample(ctx, data, form if form != capi.FORM_AUTO else used, t1, t2, side=args.f_err_side)
        out = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8" if used_form == "tensor" else "fp32",
            "data": "synthetic",
            "config": {"workload": "%s: %s" % (args.workload, data["desc"]), "nid": nid, "nsnp": data["nsnp"],
                       "blocks": len(blocks), "traits": ntraits, "test": test, "t1": t1, "t2": t2,
                       "pairs_per_step": pairs_step, "form": used_form, "hits_per_step": int(nhits),
                       "l2": "inputs larger than L2 (packed genotypes %.0f MB)" % (gp.nbytes / 1e6),
                       "gpu": gname, "planted": planted, "cuda_graph": not args.no_graph,
                       "kernel": kernel_config},
            "e2e": {"value": pairs_step * args.steps * world / e2e_s, "unit": "pairs/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "kernel_ms_per_step": statistics.mean(kernel_ms),
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "f_err": ferr,
        }
        if popc:
            out["popc_form"] = popc
            # kernel time against kernel time (the popcount sample is timed by kernel events)
            out["tensor_over_popc"] = pairs_step / (statistics.mean(kernel_ms) / 1e3) / popc["value"]
        print(json.dumps(out))
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
