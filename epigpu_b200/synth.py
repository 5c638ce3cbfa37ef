"""Seeded synthetic inputs of the scan's shape (no public dataset is involved).

Genotypes: per SNP a minor-allele frequency f ~ U(0.05, 0.5) and Hardy-Weinberg codes
0/1/2 with probabilities (1-f)^2, 2f(1-f), f^2; each call independently missing (code 3)
with probability `miss`. Packing follows the reference layout (src/readplink.c:1066-1102).
Phenotypes: N(0,1) (or standardised gamma(2,1)) with a fraction set to -9 (missing), and
optionally planted interacting pairs whose 3x3 genotype-class effect tables are random,
mean 0, each explaining `var_frac` of the variance.
"""
import numpy as np


def genotype_codes(nid, nsnp, seed, maf=(0.05, 0.5), miss=0.01, chunk=4096):
    """uint8 array (nsnp, nid) of codes 0/1/2/3."""
    rng = np.random.default_rng(seed)
    out = np.empty((nsnp, nid), dtype=np.uint8)
    for s0 in range(0, nsnp, chunk):
        s1 = min(nsnp, s0 + chunk)
        f = rng.uniform(maf[0], maf[1], size=(s1 - s0, 1))
        p0 = (1.0 - f) ** 2
        p1 = p0 + 2.0 * f * (1.0 - f)
        u = rng.random((s1 - s0, nid), dtype=np.float32)
        g = (u >= p0).astype(np.uint8) + (u >= p1).astype(np.uint8)
        if miss > 0:
            g[rng.random((s1 - s0, nid), dtype=np.float32) < miss] = 3
        out[s0:s1] = g
    return out


def pack(codes, chunk=4096):
    """Reference packing (readplink.c:1066-1102): int32 (nsnp, npack1); 16 codes per word,
    first individual in bits 31:30; the tail word holds `remain` codes right-aligned."""
    codes = np.asarray(codes, dtype=np.uint8)
    nsnp, nid = codes.shape
    npack, remain = nid // 16, nid % 16
    npack1 = npack + (1 if remain else 0)
    out = np.empty((nsnp, npack1), dtype=np.uint32)
    shifts = (30 - 2 * np.arange(16)).astype(np.uint32)
    tshifts = (2 * (remain - 1 - np.arange(remain))).astype(np.uint32)
    for s0 in range(0, nsnp, chunk):
        s1 = min(nsnp, s0 + chunk)
        c = codes[s0:s1].astype(np.uint32)
        if npack:
            full = c[:, :16 * npack].reshape(s1 - s0, npack, 16) << shifts
            out[s0:s1, :npack] = np.bitwise_or.reduce(full, axis=2)
        if remain:
            out[s0:s1, npack] = np.bitwise_or.reduce(c[:, 16 * npack:] << tshifts, axis=1)
    return out.view(np.int32)


def unpack(gpack, nid):
    """Inverse of pack (readplink.c:1104-1143)."""
    w = np.asarray(gpack).view(np.uint32)
    nsnp = w.shape[0]
    npack, remain = nid // 16, nid % 16
    out = np.empty((nsnp, nid), dtype=np.uint8)
    if npack:
        shifts = (30 - 2 * np.arange(16)).astype(np.uint32)
        out[:, :16 * npack] = ((w[:, :npack, None] >> shifts) & 3).reshape(nsnp, 16 * npack)
    if remain:
        tshifts = (2 * (remain - 1 - np.arange(remain))).astype(np.uint32)
        out[:, 16 * npack:] = (w[:, npack, None] >> tshifts) & 3
    return out


def phenotype(nid, seed, miss=0.02, dist="normal"):
    rng = np.random.default_rng(seed)
    if dist == "normal":
        y = rng.standard_normal(nid)
    elif dist == "gamma":
        y = rng.gamma(2.0, 1.0, nid)
        y = (y - 2.0) / np.sqrt(2.0)
    else:
        raise ValueError(dist)
    y = y.astype(np.float32)
    if miss > 0:
        y[rng.random(nid) < miss] = -9.0
    return y


def planted_phenotype(codes, pairs, seed, var_frac=0.005, miss=0.01):
    """N(0,1) noise plus one random mean-0 3x3 genotype-class effect per planted pair
    (snp_a, snp_b), each scaled to explain `var_frac` of the phenotypic variance.
    `codes[s]` is SNP s's row of codes: the (nsnp, nid) array or a dict of the planted rows."""
    rng = np.random.default_rng(seed)
    nid = len(codes[pairs[0][0]])
    y = rng.standard_normal(nid)
    for a, b in pairs:
        ga, gb = codes[a].astype(np.int64), codes[b].astype(np.int64)
        ok = (ga != 3) & (gb != 3)
        table = rng.standard_normal((3, 3))
        eff = np.zeros(nid)
        eff[ok] = table[ga[ok], gb[ok]]
        eff[ok] -= eff[ok].mean()
        sd = eff[ok].std()
        if sd > 0:
            eff *= np.sqrt(var_frac) / sd
        y += eff
    y = y.astype(np.float32)
    if miss > 0:
        y[rng.random(nid) < miss] = -9.0
    return y


def f_threshold(df1, df2, p):
    """Upper-tail F quantile (scipy): the threshold for a fixed p-value."""
    from scipy.stats import f
    return float(f.isf(p, df1, df2))


def uneven_block_sizes():
    """22 chromosome-like blocks, M_c = round(2000 + 22000*((21-c)/21)^1.3705), total 250,000."""
    sizes = [int(round(2000 + 22000 * ((21 - c) / 21.0) ** 1.3705)) for c in range(22)]
    sizes[0] += 250000 - sum(sizes)
    return sizes


def planted_rows(gpack, nid, pairs):
    """The code rows of the planted SNPs, unpacked from packed genotypes (a dict for
    planted_phenotype when the whole code matrix is not kept)."""
    snps = sorted({s for p in pairs for s in p})
    rows = unpack(np.asarray(gpack)[snps], nid)
    return {s: rows[i] for i, s in enumerate(snps)}


def packed_on_gpu(nid, nsnp, seed, miss=0.01, chunk=4096):
    """The genotype generator above (HWE, MAF ~ U(0.05, 0.5), `miss` missing calls) drawn on
    the GPU with torch's generator, packed in the reference layout into pinned host memory:
    the inputs of full-size runs, which numpy would take minutes to draw."""
    import torch
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    npack, remain = divmod(nid, 16)
    npack1 = npack + (1 if remain else 0)
    out = torch.empty((nsnp, npack1), dtype=torch.int32, pin_memory=True)
    shifts = torch.tensor([30 - 2 * t for t in range(16)], device=dev, dtype=torch.int64)
    tsh = torch.tensor([2 * (remain - 1 - t) for t in range(remain)], device=dev, dtype=torch.int64)
    for s0 in range(0, nsnp, chunk):
        m = min(chunk, nsnp - s0)
        f = torch.rand((m, 1), generator=g, device=dev) * 0.45 + 0.05
        p0 = (1 - f) ** 2
        p1 = p0 + 2 * f * (1 - f)
        u = torch.rand((m, nid), generator=g, device=dev)
        c = (u >= p0).to(torch.int64) + (u >= p1).to(torch.int64)
        c[torch.rand((m, nid), generator=g, device=dev) < miss] = 3
        parts = []
        if npack:
            parts.append((c[:, :16 * npack].reshape(m, npack, 16) << shifts).sum(-1))
        if remain:
            parts.append((c[:, 16 * npack:] << tsh).sum(-1, keepdim=True))
        w = torch.cat(parts, 1)
        w = torch.where(w >= 2 ** 31, w - 2 ** 32, w).to(torch.int32)
        out[s0:s0 + m].copy_(w.cpu())
    return out.numpy()


def write_plink_fileset(directory, nid, nsnp, seed, nchr=4):
    """A seeded PLINK text fileset (`x.ped`, `x.map`) for timing the data mode: per SNP two of
    A/C/G/T; genotypes among both homozygotes, both heterozygote orders and missing (0 0);
    individual 0 homozygous and individual 1 heterozygous at every SNP (the reference's reader
    needs a homozygote to code the alleles); a normal trait with every seventh value -9;
    SNPs on `nchr` chromosomes in order. Built with array operations (a 2,000 x 5,000 fileset,
    40 MB of .ped text, in about a second)."""
    import pathlib
    d = pathlib.Path(directory)
    rng = np.random.default_rng(seed)
    letters = np.frombuffer(b"ACGT", np.uint8)
    al = np.argsort(rng.random((nsnp, 4)), axis=1)[:, :2]
    a, b = letters[al[:, 0]], letters[al[:, 1]]
    g = rng.choice(5, (nid, nsnp), p=[0.35, 0.15, 0.15, 0.3, 0.05])
    g[0, :] = 0
    g[min(1, nid - 1), :] = 1
    zero = np.uint8(ord("0"))
    first = np.select([g == 0, g == 1, g == 2, g == 3], [a, a, b, b], zero).astype(np.uint8)
    second = np.select([g == 0, g == 1, g == 2, g == 3], [a, b, a, b], zero).astype(np.uint8)
    row = np.empty((nid, nsnp, 4), np.uint8)
    row[..., 0], row[..., 1], row[..., 2], row[..., 3] = first, 32, second, 32
    row[:, -1, 3] = 10
    y = rng.standard_normal(nid)
    with open(d / "x.ped", "wb") as f:
        for i in range(nid):
            phen = "-9" if i % 7 == 3 else "%.6f" % y[i]
            f.write(("F%d ind%d 0 pat%d %d %s " % (i // 3, i, i, 1 + i % 2, phen)).encode())
            f.write(row[i].tobytes())
    chrs = np.sort(rng.integers(1, nchr + 1, nsnp))
    with open(d / "x.map", "w") as f:
        f.write("".join("chr%d rs%d %.4f %d\n" % (c, 1000 + j, 0.01 * j, 5000 + 37 * j) for j, c in enumerate(chrs)))
    return d / "x.ped", d / "x.map"
