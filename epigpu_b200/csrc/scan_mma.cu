// scan_mma.cu -- tensor-core form of the pair scan (tcgen05, kind::i8, sm_100a).
//
// Per pair (i, j) the reference accumulates, over individuals k, the 3x3 genotype-cell
// counts and phenotype sums (src/EpiOpenCL.c:110-228). Both are contractions over k:
//     n_ab = sum_k [g_i(k)=a] [g_j(k)=b] w_k        S_ab = sum_k [g_i(k)=a] [g_j(k)=b] y_k
// so for a tile of 40 i-SNPs x 21 j-SNPs they are one integer GEMM
//     D[128 x 252] = A[128 x K] * B[K x 252]
//   A rows (row 32w + l, l < 30): i-SNP 10w + l/3, genotype a = l%3: [g_i(k) == a]
//   B cols: type t = 4b + s (b = 0..2 the j genotype, s = 0..3), [g_j(k) == b] * D_s(k), with
//     D_0 = w_k (phenotype valid) and D_1..3 the balanced base-256 digits of the fixed-point
//     phenotype Y_k = round(y_k * 2^sy) (y centred, 0 when invalid); CTA 0 of the pair holds
//     the types of D_0 and D_1, CTA 1 those of D_2 and D_3, so each builds its half from two
//     digit rows: column of (t, j') in the pair MMA 128 (s / 2) + 6 j' + (2b + s % 2), the six
//     columns of a j-SNP side by side in each half.
// int8 operands, int32 accumulation: counts and digit sums are exact, so
//     S_ab = (D1 + 256 D2 + 65536 D3) * 2^-sy exactly for the quantised phenotype.
// The sum of ytilde^2 (ytilde = Y 2^-sy) over the pair's valid individuals (both genotypes
// known, phenotype valid) follows from per-SNP sums over each SNP's missing individuals:
//     Q_ij = Qtot - QM_i - QM_j + QMM_ij,   QMM_ij = sum of ytilde^2 over the individuals
// missing at both SNPs, 0 <= QMM_ij. Their number and Y sum are exact from the cells:
//     n_mm = N_ij - Nvalid + NM_i + NM_j,   Y_mm = St_ij - Ytot + SM_i + SM_j,
// so QMM_ij = 0 when n_mm = 0 and (Y_mm 2^-sy)^2 when n_mm = 1 (exact); only a pair with two
// or more such individuals that needs exact statistics intersects the two SNPs' missing bits.
// The epilogue screens F and F2 in FP32 with Q_ij >= Qtot - QM_i - QM_j (F and F2 fall as Q
// grows, so the screen bounds them from above) and forms SSB / SSI / F / F2 in FP64 for every
// pair that could be a hit or a new maximum.
//
// The GEMM runs on a CTA pair (a cluster of two CTAs on two SMs, tcgen05 cta_group::2): one
// MMA of M = 256 rows (each CTA's 40 i-SNPs, 3 genotype rows each, in its own shared memory)
// by N = 256 columns (the 252 columns of 21 j-SNPs plus 4 zero columns; each CTA holds and
// builds half of them), so each SM expands half of B per stage. Each CTA's TMEM receives the
// accumulator rows of its own i-SNPs, which its epilogue reads.
//
// A comes straight from HBM: the genotype-indicator rows h3 (row 3s + a = [g_s == a] bytes)
// are TMA-loaded into a 128-byte-swizzled shared-memory stage and read by the MMA from there.
//
// Per CTA, 15 warps (20 in the variants with three epilogue warps per lane quarter or two
// producer groups; Rings below):
//   warp 13       A loader (one thread): per 128-individual stage, the CTA's A stage (four
//                 2-D tiled loads of 30 h3 rows into rows 32w..32w+29); no multicast
//   warp 14       raw loader (one thread): per stage, the j-tile's 21 one-hot rows and the
//                 trait's 4 digit rows, up to RSTAGES stages ahead of the B producers
//   warps 4-7     B producers: raw rows -> this CTA's half of the B stage (K-major, 128-byte
//                 swizzle): CTA 0 the column types of digit rows 0-1, CTA 1 of rows 2-3;
//                 a second producer group (warps 16-19) takes alternate stages in one variant
//   warp 12       CTA 0: MMA issuer (one thread): 4 pair MMAs per stage; CTA 1: forwards the
//                 completion of its own A stages to CTA 0. Both: TMEM allocation (pair form)
//   warps 0-3, 8-11  epilogue, two warps per TMEM lane quarter, seven j rounds between them
// Handshakes: one operand ring (an A stage and a B stage per slot). CTA 0's `full` barrier of a
// slot counts its own A load, CTA 1's forward of its A load and the 8 producer warps of both
// CTAs, so the MMA issuer waits once per stage; its commit arrives on both CTAs' `empty`
// barrier of the slot (multicast), which the A loaders and producers wait on. CTA 0's acc_empty
// also counts CTA 1's epilogue warps; commits arrive on both CTAs' acc_full. TMEM (512
// columns per CTA): accumulators at [0, 256) and [256, 512). All waits are bounded
// (tc_ptx.cuh); a timeout sets counters[2] and every role leaves its loop; the CTAs meet in
// a cluster barrier before the TMEM is released.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "epi_internal.cuh"
#include "tc_ptx.cuh"

namespace epi {
namespace mma {

constexpr int TI = 40;         // i-SNPs per CTA (4 lane quarters x 10 triplets)
constexpr int TIP = 2 * TI;    // i-SNPs per pair tile
constexpr int TJ = 21;         // j-SNPs per tile
constexpr int NTYPE = 12;      // B column types per j-SNP: b (3) x {w, d0, d1, d2}
constexpr int NCOL = TJ * NTYPE;  // 252 columns in use
constexpr int N = 256;         // MMA width (pair MMAs take multiples of 32)
constexpr int NH = N / 2;      // B columns held by each CTA
constexpr int TYH = NTYPE / 2; // column types held by each CTA (6 x 21 = 126 of its 128 rows)
constexpr int M = 256;         // MMA height over the pair
constexpr int KS = 128;        // individuals per pipeline stage
constexpr int ND = 4;          // digit rows per trait: w, Y digits (3)
constexpr int ROUNDS = (TJ + 2) / 3;  // j rounds of the epilogue (3 j-SNPs per round)
constexpr uint32_t ACC_COL1 = N;
__host__ __device__ constexpr uint32_t acc_col(uint32_t buf) { return buf ? ACC_COL1 : 0u; }
// accumulator column of column type ty = 4b + s, j-SNP jj of the tile: digit rows s = 0, 1 in
// CTA 0's half, 2, 3 in CTA 1's; in each half the six local types q = 2b + s % 2 of a j-SNP
// are adjacent (column 6 jj + q)
__host__ __device__ constexpr int bq(int ty) { return 2 * (ty >> 2) + (ty & 1); }
__host__ __device__ constexpr int bcol(int ty, int jj) { return ((ty & 3) >> 1) * NH + 6 * jj + bq(ty); }
// the epilogue loads a round's three j-SNPs as 20 adjacent columns per half (five x4 loads)
constexpr int RCOLS = 20;
constexpr uint32_t TMEM_COLS = 512;
constexpr int A_STAGE = (M / 2) * KS;  // 16 KB
constexpr int B_STAGE = NH * KS;       // 16 KB
constexpr int A_BOX = 30;              // h3 rows per TMA box (10 i-SNPs x 3 genotypes)
constexpr uint32_t A_BYTES = 4 * A_BOX * KS;  // transaction bytes per A stage (one CTA)
constexpr uint32_t XB_BYTES = 6 * TJ * KS;     // the streamed-B variant: one CTA's B half (126 rows)
// raw stage: the j-tile's one-hot rows and the trait's digit rows, 1024-aligned sections
constexpr int RAW_J = 0, RAW_D = (TJ * KS + 1023) / 1024 * 1024;
constexpr int RAW_STAGE = 4 * 1024;
constexpr uint32_t RAW_BYTES = (TJ + ND) * KS;
// producer work items per stage: (j-SNP, 16-individual chunk); 128 producer threads take the
// first 128 and the threads below XTRA one more (the j-SNPs 16..20, same chunk)
constexpr int XTRA = TJ * 8 - 128;

constexpr uint32_t IDESC = tc::idesc_i8(M, N);
static_assert(RAW_D % 1024 == 0 && RAW_D + ND * KS <= RAW_STAGE, "raw layout");
static_assert(B_STAGE % 1024 == 0 && A_STAGE % 1024 == 0 && N % 32 == 0 && N <= 256 && NCOL <= N, "operand tiles");
static_assert(NTYPE % 2 == 0 && TYH * TJ <= NH && TYH == 6, "B split: six types per CTA");
static_assert(XTRA >= 0 && XTRA <= 128 && (XTRA % 8) == 0 && 16 + XTRA / 8 == TJ, "producer items");
static_assert(2 * N <= (int)TMEM_COLS, "TMEM layout: two accumulators");
// the accumulator loads of a round's three j-SNPs (18 columns per half) read two columns past
// them: within each half even for the last round
static_assert(6 * 3 * (ROUNDS - 1) + RCOLS <= NH && bcol(11, TJ - 1) < N && bcol(9, TJ - 1) < NH, "epilogue loads");

// Ring depths (a kernel variant, chosen by the autotuner): STAGES operand slots, each an A stage
// (TMA from L2 / DRAM) and a B stage (built from raw rows already in shared memory), and the raw
// ring (j one-hot and digit rows, by TMA), which lets the raw loader run ahead of the B
// producers. One barrier pair per operand slot keeps the MMA issuer's work per stage to one
// wait and one commit: the issuer is the pipeline's critical path (a barrier wait costs about a
// hundred cycles even when the barrier is ready).
//
// EPW epilogue warps per TMEM lane quarter: 2 (epilogue warps 0-3 and 8-11) or 3 (also 16-19).
// PW producer groups of 4 warps: 1 (warps 4-7) or 2 (also 16-19, the groups taking alternate
// stages, so each has two stage times for its loads, stores, proxy fence and arrivals: the
// producers' per-stage latency, not their throughput, bounds the pipeline). One group and two
// epilogue warps: 15 warps. Otherwise 20 warps (warp 15 idle), launched with 96 registers each
// and rebalanced by warpgroup (setmaxnreg): epilogue warpgroups to 128, producer warpgroups to
// 56 (EPW 3) or 88 (PW 2), the loaders and MMA issuer to 40 -- 3 x 128 x 128 + 128 x 56 +
// 128 x 40 = 61,440 and 2 x 128 x 128 + 2 x 128 x 88 + 128 x 40 = 60,416, within the launch's
// pool of 640 x 96 = 61,440.
//
// XF (the streamed-B variant, single traits and sizes whose expanded B rows fit in HBM): B is
// not built in shared memory but precomputed once per genotype and trait load into HBM (12
// bytes per SNP and individual: `hx`, rows ((t 2 + half) M + snp) 6 + q) and TMA-loaded with
// the A rows, one 126-row box per CTA half per stage; no producers or raw loader run (warps 4-7
// and 14 idle) and CTA 0's full barrier counts two arrivals (its loader, CTA 1's forward).
template <int S, int RSx, int EPW_ = 2, int PW_ = 1, bool XF_ = false>
struct Rings {
    static constexpr int STAGES = S, RSTAGES = RSx, EPW = EPW_, PW = PW_;
    static constexpr bool XF = XF_;
    static_assert(!XF || (EPW == 2 && PW == 1), "the streamed-B variant runs the 15-warp layout");
    static constexpr int NWARPS = (EPW == 2 && PW == 1) ? 15 : 20;
    static constexpr int NTHREADS = NWARPS * 32;
    static constexpr int PROD_REGS = PW == 2 ? 88 : 56;
    static_assert((EPW == 2 || EPW == 3) && (PW == 1 || PW == 2) && !(EPW == 3 && PW == 2), "warp roles");
    static_assert(NWARPS == 15 || EPW * 128 * 128 + PW * 128 * PROD_REGS + 128 * 40 <= NTHREADS * 96, "register split");
    struct Smem {
        uint8_t a[STAGES][A_STAGE];
        uint8_t b[STAGES][B_STAGE];
        uint8_t raw[RSTAGES][RAW_STAGE];
        // full: CTA 0 -- its A stage landed (its TMA), CTA 1's forward of its own, and both B
        // halves built (4 local + 4 remote producer warps): 10 arrivals; CTA 1 -- its A stage
        // landed (1). empty: the MMAs reading the slot are done (both CTAs, one commit)
        uint64_t full[STAGES], empty[STAGES], raw_full[RSTAGES], raw_empty[RSTAGES], acc_full[2], acc_empty[2],
            drain;
        uint64_t stall;  // never arrived at: the wait of the debug_stall test hook
        uint32_t tmem_base;
        int abort;
    };
};

// 16-byte chunk c of row r of a 128-byte-swizzled tile (1024-byte aligned base)
__device__ __forceinline__ uint4 ld_sw128(const uint8_t *base, int r, int c)
{
    return *reinterpret_cast<const uint4 *>(base + r * 128 + ((c ^ (r & 7)) << 4));
}

struct Unit {
    int block, trait, i0, j0;
    BlockDesc bd;
    bool skip;
};

// Unit u -> (trait, block, pair tile). Units run trait-fastest over the block's tiles. XF (the
// streamed-B variant): a block's tiles are walked in groups of xsi i-tiles, and within a group
// in chunks of xsj j-tiles, i-tile by i-tile inside a chunk, so the clusters working at the same
// time share a super-tile's A rows and expanded B rows in L2; otherwise i-tile by i-tile.
template <bool XF = false>
__device__ __forceinline__ Unit decode(const ScanArgs &a, long long u)
{
    Unit r;
    const long long tile = u / a.ntraits;
    r.trait = (int)(u % a.ntraits);
    r.block = find_block(a.blocks, a.nblocks, tile);
    r.bd = a.blocks[r.block];
    const long long lt = tile - r.bd.tile_base;
    int ti, tj;
    if (XF) {
        const long long grp_tiles = (long long)a.xsi * r.bd.tiles_j;
        const int grp = (int)(lt / grp_tiles);
        const int ni = min(a.xsi, r.bd.tiles_i - grp * a.xsi);
        const long long q = lt - (long long)grp * grp_tiles;
        const int jc = (int)(q / ((long long)ni * a.xsj));
        const int q2 = (int)(q - (long long)jc * ni * a.xsj);
        const int nj = min(a.xsj, r.bd.tiles_j - jc * a.xsj);
        ti = grp * a.xsi + q2 / nj;
        tj = jc * a.xsj + q2 % nj;
    } else {
        ti = (int)(lt / r.bd.tiles_j);
        tj = (int)(lt % r.bd.tiles_j);
    }
    r.i0 = ti * TIP;  // the pair tile's first i-SNP
    r.j0 = tj * TJ;
    r.skip = r.bd.start1 + min(r.i0 + TIP, r.bd.size1) - 1 <= r.bd.start2 + r.j0;
    return r;
}

template <class Smem>
__device__ __forceinline__ void fail(const ScanArgs &a, Smem &sm, int where)
{
    sm.abort = 1;
    if (atomicCAS(&a.counters[2], 0ull, 1ull) == 0ull) a.counters[3] = (unsigned long long)where;
}

__device__ __forceinline__ uint32_t sel3(const uint32_t v[3], int idx)
{
    return idx == 0 ? v[0] : (idx == 1 ? v[1] : v[2]);
}

template <class T>
__device__ __forceinline__ T pick3(T x0, T x1, T x2, int idx)
{
    return idx == 0 ? x0 : (idx == 1 ? x1 : x2);
}

// 1/x for x > 0: single-precision seed (__frcp_rn) refined by one Newton step in FP64,
// e = 1 - x r, r' = r + r e, which squares the seed's relative error (2^-24 -> ~2^-48).
__device__ __forceinline__ double rcp_d(double x)
{
    double r = (double)__frcp_rn((float)x);
    const double e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// num / den in FP64: by rcp_d when den is a normal single-precision magnitude (relative error
// ~2^-46), else by IEEE division (zero, tiny or huge denominators keep division's inf / NaN).
__device__ __forceinline__ double div_fast(double num, double den)
{
    const double ad = fabs(den);
    return (ad > 1e-30 && ad < 1e30) ? num * rcp_d(den) : num / den;
}

// The reference's 8 df / 4 df statistics (src/EpiOpenCL.c:231-247, :452-486) in FP64 from
// the exact integer cell counts n and digit sums si (S = si * sc), and Q = sum of y^2 over
// the pair's valid individuals. Same quantities as pair_stat, arranged to avoid division
// chains: reciprocals by rcp_d.
__device__ __forceinline__ PairStat pair_stat_exact(const int n[9], const double si[9], double sc, double Q,
                                                    bool want_int)
{
    // si are integers below 2^53 in magnitude (digit sums), so every sum of them is exact
    PairStat r;
    int N = 0, nfac = 0;
    double St_i = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        N += n[c];
        St_i += si[c];
        nfac += n[c] > 0;
    }
    const double St = St_i * sc;
    const double m = St * rcp_d((double)N);
    double mc[9], SSB = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        mc[c] = 0.0;
        if (n[c] > 0) {
            mc[c] = si[c] * sc * rcp_d((double)n[c]);
            const double d = mc[c] - m;
            SSB = fma((double)n[c] * d, d, SSB);
        }
    }
    const double SSW = ssw_floored(Q - St * m, SSB, SSW_FLOOR_EXACT);
    r.nfac = nfac;
    r.d1 = nfac - 1;
    r.d2 = N - nfac;
    r.F = div_fast(SSB * (double)r.d2, SSW * (double)r.d1);
    r.F2 = 0.0;
    if (want_int) {
        double row[3], col[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double rs = si[3 * i] + si[3 * i + 1] + si[3 * i + 2];
            const double cs = si[i] + si[i + 3] + si[i + 6];
            const int rn = n[3 * i] + n[3 * i + 1] + n[3 * i + 2];
            const int cn = n[i] + n[i + 3] + n[i + 6];
            row[i] = rn > 0 ? rs * sc * rcp_d((double)rn) : 0.0;
            col[i] = cn > 0 ? cs * sc * rcp_d((double)cn) : 0.0;
        }
        double SSI = 0.0;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            if (n[c] > 0) {
                const double t = mc[c] - row[c / 3] - col[c % 3] + m;
                SSI = fma((double)n[c] * t, t, SSI);
            }
        }
        r.F2 = div_fast(SSI * (double)r.d2, 4.0 * SSW);
    }
    return r;
}

// approximate reciprocal of the screen (one MUFU operation, relative error ~2^-23; 1/0 = +inf)
__device__ __forceinline__ float rcp_fast(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The same statistics in FP32, as a screen: relative error ~1e-6 for the centred trait and
// the exact integer cells this gets (no cancellation beyond SSW = Q - ... at large N).
// A pair whose screened F and F2 are clearly below every threshold and below the running
// maxima cannot be a hit or a new maximum, and keeps these values; every other pair is
// recomputed by pair_stat_exact.
__device__ __forceinline__ void pair_stat_f32(const int n[9], const float sd[9], float sc, float Q, bool want_int,
                                              float &F, float &F2)
{
    float N = 0.0f, St = 0.0f, nfac = 0.0f, sf[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        sf[c] = sd[c] * sc;
        N += (float)n[c];
        St += sf[c];
        nfac += n[c] > 0 ? 1.0f : 0.0f;
    }
    const float m = St * rcp_fast(N);
    float mc[9], SSB = 0.0f;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        mc[c] = n[c] > 0 ? sf[c] * rcp_fast((float)n[c]) : 0.0f;
        const float d = mc[c] - m;
        SSB = fmaf((float)n[c] * d, d, SSB);
    }
    const float SSY = Q - St * m;  // sum of squares about the pair's mean
    const float SSW = SSY - SSB;
    // SSW carries an absolute error of a few ulps of SSY; while SSW > 1e-3 SSY its relative
    // error stays below ~3e-4, inside the margin. A closer fit (or a negative SSW from
    // rounding) goes to the exact path: NaN fails every screen comparison.
    if (!(SSW > 1e-3f * SSY)) {
        F = F2 = __int_as_float(0x7fc00000);
        return;
    }
    const float d1 = nfac - 1.0f, d2 = N - nfac;
    F = (SSB * d2) * rcp_fast(SSW * d1);
    F2 = 0.0f;
    if (want_int) {
        float row[3], col[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float rn = (float)(n[3 * i] + n[3 * i + 1] + n[3 * i + 2]);
            const float cn = (float)(n[i] + n[i + 3] + n[i + 6]);
            row[i] = rn > 0.0f ? (sf[3 * i] + sf[3 * i + 1] + sf[3 * i + 2]) * rcp_fast(rn) : 0.0f;
            col[i] = cn > 0.0f ? (sf[i] + sf[i + 3] + sf[i + 6]) * rcp_fast(cn) : 0.0f;
        }
        float SSI = 0.0f;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const float t = mc[c] - row[c / 3] - col[c % 3] + m;
            SSI = n[c] > 0 ? fmaf((float)n[c] * t, t, SSI) : SSI;
        }
        F2 = (SSI * d2) * rcp_fast(4.0f * SSW);
    }
}

// x lowered by the screen's margin (relative 1e-3); -inf and NaN stay as they are
__device__ __forceinline__ float screen_lo(float x) { return x - 1e-3f * fabsf(x); }

template <int RING>
__device__ __forceinline__ void advance(uint32_t &slot, uint32_t &phase)
{
    if (++slot == RING) {
        slot = 0;
        phase ^= 1u;
    }
}

template <class C>
__global__ void __launch_bounds__(C::NTHREADS, 1) k_scan_mma(ScanArgs a, const __grid_constant__ MmaMaps maps)
{
    constexpr int STAGES = C::STAGES, RSTAGES = C::RSTAGES, EPW = C::EPW, PW = C::PW;
    using Smem = typename C::Smem;
    extern __shared__ uint8_t smem_raw[];
    // the operand stages need 1024-byte alignment (128-byte swizzle atoms); the offset is the
    // same in both CTAs of the pair, as the pair MMA and the remote arrivals require
    const uint32_t raw_s = tc::smem_u32(smem_raw);
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw + (((raw_s + 1023u) & ~1023u) - raw_s));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = tc::cluster_rank();  // 0: issues the MMAs
    const long long pair = tc::cluster_id(), npairs = tc::cluster_count();
    const long long units = a.ntiles * (long long)a.ntraits;
    const int nks = a.Np / KS;

    if (warp == 12) {
        tc::tmem_alloc_pair(&sm.tmem_base, TMEM_COLS);
        tc::tmem_relinquish_pair();
    }
    // each CTA's B half holds six column types in rows 0-125: rows 126-127 stay zero
    constexpr int ZR = NH - TYH * TJ;
    for (int w = threadIdx.x; w < STAGES * ZR * 8; w += blockDim.x) {
        const int st = w / (ZR * 8), n = TYH * TJ + (w / 8) % ZR, c = w % 8;
        *reinterpret_cast<uint4 *>(sm.b[st] + (n >> 3) * 1024 + (n & 7) * 128 + c * 16) = make_uint4(0, 0, 0, 0);
    }
    tc::fence_proxy_async_smem();
    // maxima of F and F2 per trait: per CTA in shared memory (flushed to global memory once,
    // at the end) up to SMAX_TRAITS traits, else the global maxima directly
    const bool smax_local = a.ntraits <= SMAX_TRAITS;
    unsigned int *smax = reinterpret_cast<unsigned int *>(reinterpret_cast<uint8_t *>(&sm) + sizeof(Smem));
    if (smax_local)
        for (int w = threadIdx.x; w < 2 * a.ntraits; w += blockDim.x) smax[w] = 0u;
    unsigned int *const mxf = smax_local ? smax : a.maxf;
    unsigned int *const mxf2 = smax_local ? smax + a.ntraits : a.maxf2;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tc::mbar_init(&sm.full[s], rank == 0 ? (C::XF ? 2 : 10) : 1);
            tc::mbar_init(&sm.empty[s], 1);
        }
        for (int r = 0; r < RSTAGES; ++r) {
            tc::mbar_init(&sm.raw_full[r], 1);
            tc::mbar_init(&sm.raw_empty[r], 4);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&sm.acc_full[b], 1);
            tc::mbar_init(&sm.acc_empty[b], 8 * EPW);  // every epilogue warp of both CTAs
        }
        tc::mbar_init(&sm.drain, 1);
        tc::mbar_init(&sm.stall, 1);
        sm.abort = 0;
        tc::fence_barrier_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // both CTAs' barriers exist before any remote arrival
    tc::tc_fence_after();
    const uint32_t tmem = sm.tmem_base;
    volatile int *abort = &sm.abort;

    // epilogue warps: 0-3, 8-11 (and 16-19 with three per lane quarter); producer warps: 4-7
    // (and 16-19 with two producer groups)
    const bool epi_warp = warp < 4 || (warp >= 8 && warp < 12) || (EPW == 3 && warp >= 16);
    const bool prod_warp = !C::XF && ((warp >= 4 && warp < 8) || (PW == 2 && warp >= 16));
    if constexpr (C::NWARPS == 20) {
        if (epi_warp) tc::setmaxnreg_inc<128>();
        else if (prod_warp) tc::setmaxnreg_dec<C::PROD_REGS>();
        else tc::setmaxnreg_dec<40>();
    }
    if (prod_warp) {
        // ---------------- B producers: thread -> (j-SNP, 16-individual chunk) ----------------
        // items (jj, c) with jj < 16 for every thread, and (16 + t/8, c) for t < XTRA; with two
        // groups, group pg builds the stages whose sequence number is pg modulo 2 (and follows
        // the ring positions of the others without touching them)
        const int pg = warp >= 16 ? 1 : 0;
        const int t = threadIdx.x - (pg ? 512 : 128), jj = t >> 3, c = t & 7;
        const bool xtra = t < XTRA;
        uint32_t stage = 0, phase = 0, rs = 0, rph = 0, seq = 0;
        bool ok = true;
        for (long long u = pair; u < units && ok; u += npairs) {
            const Unit un = decode<C::XF>(a, u);
            if (un.skip) continue;
            for (int ks = 0; ks < nks; ++ks) {
                if ((int)(seq++ % (uint32_t)PW) != pg) {
                    advance<STAGES>(stage, phase);
                    advance<RSTAGES>(rs, rph);
                    continue;
                }
                if (!tc::mbar_wait(&sm.raw_full[rs], rph, abort, a.wait_ns) || !tc::mbar_wait(&sm.empty[stage], phase ^ 1u, abort, a.wait_ns)) {
                    fail(a, sm, 2);
                    ok = false;
                    break;
                }
                const uint8_t *raw = sm.raw[rs];
                uint8_t *base = sm.b[stage];
                // this CTA's two digit rows: 2 rank and 2 rank + 1
                const uint4 d[2] = {ld_sw128(raw + RAW_D, 2 * (int)rank, c), ld_sw128(raw + RAW_D, 2 * (int)rank + 1, c)};
                // local type q = 2b + s' (genotype b, this CTA's digit row s') of j-SNP jx at
                // local row 6 jx + q
                auto put = [&](int q, int jx, const uint4 &m) {
                    const int n = 6 * jx + q;
                    const uint4 &dv = d[q & 1];
                    uint4 o;
                    o.x = m.x & dv.x;
                    o.y = m.y & dv.y;
                    o.z = m.z & dv.z;
                    o.w = m.w & dv.w;
                    *reinterpret_cast<uint4 *>(base + (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4)) = o;
                };
                // byte mask of genotype b: one-hot bit b of each byte spread to 0xFF
                auto gmask = [](const uint4 &h, int b) {
                    uint4 m;
                    m.x = ((h.x >> b) & 0x01010101u) * 0xFFu;
                    m.y = ((h.y >> b) & 0x01010101u) * 0xFFu;
                    m.z = ((h.z >> b) & 0x01010101u) * 0xFFu;
                    m.w = ((h.w >> b) & 0x01010101u) * 0xFFu;
                    return m;
                };
                auto build = [&](int jx) {
                    const uint4 h = ld_sw128(raw + RAW_J, jx, c);
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const uint4 m = gmask(h, b);
                        put(2 * b, jx, m);
                        put(2 * b + 1, jx, m);
                    }
                };
                build(jj);
                if (xtra) build(16 + jj);
                // the raw slot is released only after the stores above, which consume every
                // value loaded from it (an arrive right after the loads can overtake them)
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tc::mbar_arrive(&sm.raw_empty[rs]);
                    if (rank == 0) tc::mbar_arrive(&sm.full[stage]);
                    else tc::mbar_arrive_remote(&sm.full[stage], 0);
                }
                advance<STAGES>(stage, phase);
                advance<RSTAGES>(rs, rph);
            }
        }
    } else if (epi_warp) {
        // ---------------- epilogue: the j rounds split over the warps of each lane quarter ----------------
        // warps 0-3 (group 0), 8-11 (group 1), 16-19 (group 2): rounds [rb(g), rb(g + 1))
        const int e = warp & 3, grp = warp < 4 ? 0 : (warp < 12 ? 1 : 2);
        const int rho_begin = (grp * ROUNDS + EPW - 1) / EPW, rho_end = ((grp + 1) * ROUNDS + EPW - 1) / EPW;
        const int ii = 10 * e + lane / 3, ga = lane % 3, tbase = (lane / 3) * 3;
        const bool rowok = lane < 30;
        const uint32_t tl = tmem + ((uint32_t)(32 * e) << 16);
        uint32_t accph[2] = {0u, 0u};
        int buf = 0;
        for (long long u = pair; u < units; u += npairs) {
            Unit un = decode<C::XF>(a, u);
            if (un.skip) continue;
            un.i0 += TI * (int)rank;  // this CTA's i-SNPs
            const int t = un.trait;
            const double sc = a.yscale[t];
            const int di = un.i0 + ii;
            const bool ivalid = rowok && di < un.bd.size1;
            const int gi = un.bd.start1 + (ivalid ? di : 0);
            const size_t mi = (size_t)t * a.nsnp + gi;
            // sum of ytilde^2 over the valid individuals known at SNP i; and the quantities of
            // the individuals missing at i that the exact path needs
            const double pki = ivalid ? a.qtot[t] - a.qm[mi] : 0.0;
            const double smi = ivalid ? a.sm[mi] : 0.0, nmi_nv = ivalid ? a.nm[mi] - a.nvalid[t] : 0.0;
            const double ytot = a.ytot[t];
            if (!tc::mbar_wait(&sm.acc_full[buf], accph[buf], abort, a.wait_ns)) {
                fail(a, sm, 3);
                break;
            }
            tc::tc_fence_after();
            const uint32_t acc = tl + acc_col(buf);
            const bool report = a.report_trait < 0 || a.report_trait == t;
            const bool dumping = t == a.report_trait && (a.dump_counts || a.dump_F);
            const float t1c = screen_lo(a.t1), t2c = screen_lo(a.t2), scf = (float)sc;
            unsigned int fmx = 0u, f2mx = 0u;  // this thread's largest F, F2 of the tile (encoded)
            // screen against the CTA's maxima so far (exact values, a lower bound of the final
            // maxima): a pair that can raise a maximum always takes the exact path
            const unsigned int m1 = reinterpret_cast<volatile unsigned int *>(mxf)[t];
            const unsigned int m2 = reinterpret_cast<volatile unsigned int *>(mxf2)[t];
            float fmx_f = m1 ? ord2f(m1) : -INFINITY, f2mx_f = m2 ? ord2f(m2) : -INFINITY;
#pragma unroll 1
            for (int rho = rho_begin; rho < rho_end; ++rho) {
                const int jb = 3 * rho;
                const int jl = jb + ga;
                const int dj = un.j0 + jl;
                const bool valid = ivalid && (jl < TJ) && dj < un.bd.size2 &&
                                   (un.bd.start1 + di > un.bd.start2 + dj);
                const int gj = un.bd.start2 + (valid ? dj : 0);
                const size_t mj = (size_t)t * a.nsnp + gj;
                const double qmj = valid ? a.qm[mj] : 0.0;
                // the round's columns of both halves, then v[ty][c] = type ty of j-SNP jb + c
                uint32_t wv[2][RCOLS], v[NTYPE][3];
                auto load_round = [&]() {
#pragma unroll
                    for (int h = 0; h < 2; ++h)
#pragma unroll
                        for (int k = 0; k < RCOLS / 4; ++k)
                            tc::tmem_ld4(acc + h * NH + 6 * jb + 4 * k, wv[h][4 * k], wv[h][4 * k + 1], wv[h][4 * k + 2],
                                         wv[h][4 * k + 3]);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int ty = 0; ty < NTYPE; ++ty)
#pragma unroll
                        for (int c = 0; c < 3; ++c) v[ty][c] = wv[(ty & 3) >> 1][6 * c + bq(ty)];
                };
                load_round();
                // this lane's accumulator row (SNP i, genotype ga) folded per column c of the round
                // (j-SNP jb + c): three counts and three FP32 phenotype sums. Up to 131,072
                // individuals every digit sum is below 2^24 in magnitude, so the conversions are
                // exact and the two fmas round once each (beyond, the conversions round too:
                // relative 2^-24, far inside the screen's margin).
                int cn[3][3];
                float cs[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        cn[c][b] = (int)v[4 * b][c];
                        cs[c][b] = fmaf(65536.0f, (float)(int)v[4 * b + 3][c],
                                        fmaf(256.0f, (float)(int)v[4 * b + 2][c], (float)(int)v[4 * b + 1][c]));
                    }
                }
                // the pair (SNP i, j-SNP jb + ga) is this lane's: its own row directly, the rows of
                // the triplet's other two lanes by shuffle, each lane offering the column its reader
                // needs (the lane of genotype ga+1 offers its column (ga+1)+2 = ga, mod 3). Cells
                // row-major in this relative row order (own, ga+1, ga+2): F and F2 do not depend
                // on the order of the rows; only the count dump maps them back to genotypes.
                const int s1 = tbase + (ga + 1) % 3, s2 = tbase + (ga + 2) % 3;
                const int o1 = (ga + 2) % 3, o2 = (ga + 1) % 3;  // the columns this lane offers
                int n[9];
                float sfd[9];
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    n[b] = pick3(cn[0][b], cn[1][b], cn[2][b], ga);
                    n[3 + b] = __shfl_sync(0xffffffffu, pick3(cn[0][b], cn[1][b], cn[2][b], o1), s1);
                    n[6 + b] = __shfl_sync(0xffffffffu, pick3(cn[0][b], cn[1][b], cn[2][b], o2), s2);
                    sfd[b] = pick3(cs[0][b], cs[1][b], cs[2][b], ga);
                    sfd[3 + b] = __shfl_sync(0xffffffffu, pick3(cs[0][b], cs[1][b], cs[2][b], o1), s1);
                    sfd[6 + b] = __shfl_sync(0xffffffffu, pick3(cs[0][b], cs[1][b], cs[2][b], o2), s2);
                }
                PairStat s;
                s.nfac = s.d1 = s.d2 = 0;
                s.F = s.F2 = 0.0;
                int npair = 0;
                bool exact = false;
                if (valid) {
#pragma unroll
                    for (int c = 0; c < 9; ++c) npair += n[c];
                    // a lower bound of the pair's sum of squares (QMM_ij >= 0 left out), so the
                    // screened F and F2 bound the pair's values from above
                    const float Qf = (float)(pki - qmj);
                    float Ff, F2f;
                    pair_stat_f32(n, sfd, scf, Qf, a.test_int != 0, Ff, F2f);
                    exact = dumping || npair < 256 || !(Ff <= t1c) || !(Ff <= screen_lo(fmx_f)) ||
                            (a.test_int && (!(F2f <= t2c) || !(F2f <= screen_lo(f2mx_f))));
                    if (!exact) {
                        // below every threshold and both running maxima by more than the margin
                        int nfac = 0;
#pragma unroll
                        for (int c = 0; c < 9; ++c) nfac += n[c] > 0;
                        s.nfac = nfac;
                        s.d1 = nfac - 1;
                        s.d2 = npair - nfac;
                        s.F = Ff;
                        s.F2 = F2f;
                    }
                }
                if (__any_sync(0xffffffffu, exact)) {
                    // rare (pairs near a threshold or a running maximum, count dumps, small
                    // blocks): the exact digit sums of every cell, gathered again from the
                    // accumulator (still in TMEM until this warp releases it)
                    load_round();
                    uint32_t r1[NTYPE], r2[NTYPE];
#pragma unroll
                    for (int ty = 0; ty < NTYPE; ++ty) {
                        r1[ty] = __shfl_sync(0xffffffffu, sel3(v[ty], o1), s1);
                        r2[ty] = __shfl_sync(0xffffffffu, sel3(v[ty], o2), s2);
                    }
                    double si[9];  // digit sums as exact integers
                    double qmm = 0.0;
                    int nmm = 0;
                    if (exact) {
                        double st = 0.0;
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            const uint32_t c1[3] = {sel3(v[4 * b + 1], ga), r1[4 * b + 1], r2[4 * b + 1]};
                            const uint32_t c2[3] = {sel3(v[4 * b + 2], ga), r1[4 * b + 2], r2[4 * b + 2]};
                            const uint32_t c3[3] = {sel3(v[4 * b + 3], ga), r1[4 * b + 3], r2[4 * b + 3]};
#pragma unroll
                            for (int r = 0; r < 3; ++r) {
                                si[3 * r + b] = fma(65536.0, (double)(int)c3[r],
                                                    fma(256.0, (double)(int)c2[r], (double)(int)c1[r]));
                                st += si[3 * r + b];
                            }
                        }
                        // the individuals missing at both SNPs: their number, and for a single
                        // one its y^2 from the Y sums (every term an exact integer below 2^53)
                        nmm = npair + (int)(nmi_nv + a.nm[mj]);
                        if (nmm == 1) {
                            const double ymm = (st - ytot + smi + a.sm[mj]) * sc;
                            qmm = ymm * ymm;
                        }
                    }
                    // two or more: the whole warp intersects the two SNPs' missing bits for each
                    // such pair in turn and sums ytilde^2 over the intersection
                    unsigned int need = __ballot_sync(0xffffffffu, exact && nmm >= 2);
                    while (need) {
                        const int src = __ffs(need) - 1;
                        need &= need - 1;
                        const int si_ = __shfl_sync(0xffffffffu, gi, src), sj_ = __shfl_sync(0xffffffffu, gj, src);
                        const uint32_t *mbi = a.missbits + (size_t)si_ * a.Wp, *mbj = a.missbits + (size_t)sj_ * a.Wp;
                        const uint32_t *wm = a.wmask + (size_t)t * a.Wp;
                        const double *qdt = a.qd + (size_t)t * a.Np;
                        double part = 0.0;
                        for (int w = lane; w < a.Wp; w += 32) {
                            uint32_t bits = mbi[w] & mbj[w] & wm[w];
                            while (bits) {
                                part += qdt[32 * w + __ffs(bits) - 1];
                                bits &= bits - 1;
                            }
                        }
#pragma unroll
                        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
                        if (lane == src) qmm = part;
                    }
                    if (exact) s = pair_stat_exact(n, si, sc, pki - qmj + qmm, a.test_int != 0);
                }
                if (valid && dumping) {
                    const size_t o = (size_t)di * un.bd.size2 + dj;
                    if (a.dump_counts)
#pragma unroll
                        for (int c = 0; c < 9; ++c)  // relative row c/3 is genotype (ga + c/3) mod 3
                            a.dump_counts[9 * o + 3 * ((ga + c / 3) % 3) + c % 3] = n[c];
                    if (a.dump_F) a.dump_F[o] = (float)s.F;
                    if (a.dump_F2) a.dump_F2[o] = (float)s.F2;
                    if (a.dump_df1) a.dump_df1[o] = s.d1;
                    if (a.dump_df2) a.dump_df2[o] = s.d2;
                }
                const bool hit = valid && report && is_hit(a, s);
                emit_hit(a, hit, un.bd.start1 + di, un.bd.start2 + dj, s, t, un.block);
                if (valid && s.F == s.F) {
                    fmx = max(fmx, f2ord((float)s.F));
                    fmx_f = fmaxf(fmx_f, (float)s.F);
                }
                if (valid && s.F2 == s.F2) {
                    f2mx = max(f2mx, f2ord((float)s.F2));
                    f2mx_f = fmaxf(f2mx_f, (float)s.F2);
                }
            }
            fold_max_enc(&mxf[t], fmx);
            if (a.test_int) fold_max_enc(&mxf2[t], f2mx);
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (rank == 0) tc::mbar_arrive(&sm.acc_empty[buf]);
                else tc::mbar_arrive_remote(&sm.acc_empty[buf], 0);
            }
            accph[buf] ^= 1u;
            buf ^= 1;
        }
    } else if (warp == 13) {
        // ---------------- A loader: this CTA's indicator rows, one slot per operand stage ----
        if (lane == 0) {
            uint32_t as = 0, aph = 0, issued_a = 0;
            bool ok = true;
            for (long long u = pair; u < units && ok; u += npairs) {
                const Unit un = decode<C::XF>(a, u);
                if (un.skip) continue;
                const int arow = 3 * (un.bd.start1 + un.i0 + TI * (int)rank);
                const int xrow = ((un.trait * 2 + (int)rank) * a.nsnp + un.bd.start2 + un.j0) * 6;
                for (int ks = 0; ks < nks; ++ks) {
                    if (!tc::mbar_wait(&sm.empty[as], aph ^ 1u, abort, a.wait_ns)) {
                        fail(a, sm, 7);
                        ok = false;
                        break;
                    }
                    tc::mbar_arrive_expect_tx(&sm.full[as], C::XF ? A_BYTES + XB_BYTES : A_BYTES);
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        tc::tma_load_2d(sm.a[as] + 32 * w * KS, &maps.hi, ks * KS, arow + A_BOX * w, &sm.full[as]);
                    // the streamed-B variant: this CTA's half of the B stage, 126 expanded rows
                    if constexpr (C::XF) tc::tma_load_2d(sm.b[as], &maps.hx, ks * KS, xrow, &sm.full[as]);
                    ++issued_a;
                    advance<STAGES>(as, aph);
                }
            }
            // no TMA write may still be landing in shared memory when the CTA exits: wait for
            // the last loads issued into every slot. A stages of CTA 1 complete on its local
            // barrier; CTA 0's also need CTA 1's forward, so CTA 0 waits for its own bytes only
            // through the phases it can observe (all its issued phases complete on the normal
            // path; after an abort the bounded wait ends).
            int no_abort = 0;
            for (uint32_t back = 1; back <= STAGES && back <= issued_a; ++back) {
                const uint32_t slot = (as + STAGES - back) % STAGES, par = back > as ? (aph ^ 1u) : aph;
                if (!tc::mbar_wait(&sm.full[slot], par, &no_abort, a.wait_ns)) fail(a, sm, 8);
            }
        }
    } else if (warp == 14 && !C::XF) {
        // ---------------- raw loader: j one-hot rows and trait digit rows ----------------
        // gated only by the B producers' consumption, so it runs up to RSTAGES stages ahead
        // of them (the j rows come from DRAM once per pair tile)
        if (lane == 0) {
            uint32_t rs = 0, rph = 0, issued_r = 0;
            bool ok = true;
            for (long long u = pair; u < units && ok; u += npairs) {
                const Unit un = decode<C::XF>(a, u);
                if (un.skip) continue;
                for (int ks = 0; ks < nks; ++ks) {
                    if (!tc::mbar_wait(&sm.raw_empty[rs], rph ^ 1u, abort, a.wait_ns)) {
                        fail(a, sm, 10);
                        ok = false;
                        break;
                    }
                    uint8_t *raw = sm.raw[rs];
                    tc::mbar_arrive_expect_tx(&sm.raw_full[rs], RAW_BYTES);
                    tc::tma_load_2d(raw + RAW_J, &maps.hj, ks * KS, un.bd.start2 + un.j0, &sm.raw_full[rs]);
                    tc::tma_load_2d(raw + RAW_D, &maps.dg, ks * KS, ND * un.trait, &sm.raw_full[rs]);
                    ++issued_r;
                    advance<RSTAGES>(rs, rph);
                }
            }
            int no_abort = 0;
            for (uint32_t back = 1; back <= RSTAGES && back <= issued_r; ++back) {
                const uint32_t slot = (rs + RSTAGES - back) % RSTAGES, par = back > rs ? (rph ^ 1u) : rph;
                if (!tc::mbar_wait(&sm.raw_full[slot], par, &no_abort, a.wait_ns)) fail(a, sm, 11);
            }
        }
    } else if (warp == 12 && lane == 0 && rank == 1) {
        // ---------------- A forwarder (CTA 1, warp 12) ----------------
        // each of this CTA's A stages, once landed, counts as one arrival on CTA 0's full
        uint32_t as = 0, aph = 0;
        bool ok = true;
        for (long long u = pair; u < units && ok; u += npairs) {
            const Unit un = decode<C::XF>(a, u);
            if (un.skip) continue;
            for (int ks = 0; ks < nks; ++ks) {
                if (!tc::mbar_wait(&sm.full[as], aph, abort, a.wait_ns)) {
                    fail(a, sm, 9);
                    ok = false;
                    break;
                }
                tc::mbar_arrive_remote(&sm.full[as], 0);
                advance<STAGES>(as, aph);
            }
        }
    } else if (warp == 12 && lane == 0) {
        // ---------------- MMA issuer (CTA 0, warp 12) ----------------
        uint32_t as = 0, aph = 0, accph[2] = {0u, 0u};
        int buf = 0;
        bool ok = true;
        // test hook: the first CTA pair's issuer waits on a barrier that nothing arrives at, so
        // the wait runs out after wait_ns and the scan ends with a timeout status
        if (a.debug_stall && pair == 0 && !tc::mbar_wait(&sm.stall, 0, abort, a.wait_ns)) {
            fail(a, sm, 12);
            ok = false;
        }
        for (long long u = pair; u < units && ok; u += npairs) {
            const Unit un = decode<C::XF>(a, u);
            if (un.skip) continue;
            if (!tc::mbar_wait_cluster(&sm.acc_empty[buf], accph[buf] ^ 1u, abort, a.wait_ns)) {
                fail(a, sm, 4);
                break;
            }
            tc::tc_fence_after();
            const uint32_t d = tmem + acc_col(buf);
            for (int ks = 0; ks < nks; ++ks) {
                if (!tc::mbar_wait_cluster(&sm.full[as], aph, abort, a.wait_ns)) {
                    fail(a, sm, 5);
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t asb = tc::smem_u32(sm.a[as]), bsb = tc::smem_u32(sm.b[as]);
#pragma unroll
                for (int kk = 0; kk < KS / 32; ++kk)
                    tc::mma_i8_pair(d, tc::smem_desc_sw128(asb + 32 * kk), tc::smem_desc_sw128(bsb + 32 * kk), IDESC,
                                    (ks | kk) != 0);
                tc::mma_commit_pair_mc(&sm.empty[as], 0x3);
                advance<STAGES>(as, aph);
            }
            if (!ok) break;
            tc::mma_commit_pair_mc(&sm.acc_full[buf], 0x3);
            accph[buf] ^= 1u;
            buf ^= 1;
        }
        // every MMA issued above has completed once `drain` flips (waited for even after an
        // abort: the accumulators and both CTAs' operands must be idle before the TMEM and
        // shared memory are released)
        tc::mma_commit_pair(&sm.drain);
        int no_abort = 0;
        if (!tc::mbar_wait(&sm.drain, 0, &no_abort, a.wait_ns)) fail(a, sm, 6);
    }

    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // CTA 0's MMAs (which read CTA 1's shared memory) have drained
    if (warp == 12) {
        tc::tc_fence_after();
        tc::tmem_dealloc_pair(tmem, TMEM_COLS);
    }
    if (smax_local)
        for (int w = threadIdx.x; w < 2 * a.ntraits; w += blockDim.x)
            if (smax[w]) atomicMax(w < a.ntraits ? &a.maxf[w] : &a.maxf2[w - a.ntraits], smax[w]);
}

}  // namespace mma

// Tensor maps of the tensor form's TMA loads: the genotype-indicator rows h3 [3 nsnp][Np]
// with 30-row boxes (A), the one-hot genotype bytes [nsnp][Np] with 16-row boxes (j side) and
// the trait digit rows [7T][Np] with 7-row boxes; all 128 bytes wide, 128-byte swizzled,
// out-of-range rows read as zero.
static cudaError_t encode_2d(CUtensorMap *m, const void *base, uint64_t inner, uint64_t rows, uint32_t box_rows)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t dims[2] = {inner, rows};
    const cuuint64_t strides[1] = {inner};
    const cuuint32_t box[2] = {(cuuint32_t)mma::KS, box_rows};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t mma_encode_genotypes(MmaMaps *maps, const uint8_t *hcodes, const uint8_t *h3, int nsnp, int Np)
{
    cudaError_t e = encode_2d(&maps->hi, h3, (uint64_t)Np, 3 * (uint64_t)nsnp, mma::A_BOX);
    if (e == cudaSuccess) e = encode_2d(&maps->hj, hcodes, (uint64_t)Np, (uint64_t)nsnp, mma::TJ);
    return e;
}

cudaError_t mma_encode_traits(MmaMaps *maps, const int8_t *ydig, int ntraits, int Np)
{
    return encode_2d(&maps->dg, ydig, (uint64_t)Np, (uint64_t)mma::ND * ntraits, mma::ND);
}

// The streamed-B variant's expanded rows [ntraits][2][nsnp][6][Np], in boxes of one CTA half
// of a j tile (21 SNPs x 6 types = 126 rows)
cudaError_t mma_encode_x(MmaMaps *maps, const int8_t *x, int nsnp, int Np, int ntraits)
{
    return encode_2d(&maps->hx, x, (uint64_t)Np, 12 * (uint64_t)nsnp * ntraits, 6 * mma::TJ);
}

bool mma_available() { return true; }
int mma_tile_i() { return mma::TIP; }  // the host tiles blocks by CTA-pair tiles
int mma_tile_j() { return mma::TJ; }
int mma_min_nid() { return 256; }
int mma_max_nid() { return 1 << 24; }  // digit sums stay within int32
int mma_stage_individuals() { return mma::KS; }

// The variants the autotuner chooses among -- operand slots and raw stages (each ~200-216 KB
// of shared memory) and epilogue warps per TMEM lane quarter:
//   0  6 slots / 6 raw, 2 epilogue warps   1  5 / 10, 2   2  6 / 4, 2   3  6 / 6, 3
//   4  6 / 6, 2 epilogue warps, two producer groups on alternate stages
//   5  6 slots, streamed B (expanded rows TMA-loaded from HBM; no producers, no raw ring)
using Rings0 = mma::Rings<6, 6>;
using Rings1 = mma::Rings<5, 10>;
using Rings2 = mma::Rings<6, 4>;
using Rings3 = mma::Rings<6, 6, 3>;
using Rings4 = mma::Rings<6, 6, 2, 2>;
using Rings5 = mma::Rings<6, 1, 2, 1, true>;
constexpr int MMA_SHAPES = 6;

bool mma_needs_x(int v) { return v == 5; }

int mma_shapes() { return MMA_SHAPES; }

void mma_shape(int v, const char **desc)
{
    static const char *names[MMA_SHAPES] = {"6 operand slots / 6 raw stages, 8 epilogue warps",
                                            "5 operand slots / 10 raw stages, 8 epilogue warps",
                                            "6 operand slots / 4 raw stages, 8 epilogue warps",
                                            "6 operand slots / 6 raw stages, 12 epilogue warps (setmaxnreg)",
                                            "6 operand slots / 6 raw stages, 8 epilogue warps, 2 producer groups (setmaxnreg)",
                                            "6 operand slots, B streamed from HBM, 8 epilogue warps"};
    if (desc) *desc = names[v];
}

// Launch shape per (device, variant, dynamic shared memory size): the attribute set and the
// number of co-resident clusters, queried once (the occupancy query costs far more than a
// small scan's host work).
struct MmaShape {
    int device, variant;
    size_t smem;
    int clusters;
};

static std::mutex g_shape_mu;
static std::vector<MmaShape> g_shapes;

template <class C>
static cudaLaunchConfig_t mma_config(int ntraits, int grid, cudaStream_t stream, cudaLaunchAttribute *attr)
{
    cudaLaunchConfig_t cfg = {};
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(C::NTHREADS, 1, 1);
    // more than half of the SM's shared memory: one CTA per SM, which owns all 512 TMEM
    // columns; the tail holds the per-CTA maxima
    cfg.dynamicSmemBytes = sizeof(typename C::Smem) + 1024 + smax_bytes(ntraits);
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <class C>
static cudaError_t prepare(int v, int ntraits, int grid_request, int *grid)
{
    static_assert(sizeof(typename C::Smem) + 1024 > 116 * 1024, "one CTA per SM");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = mma_config<C>(ntraits, std::max(2, (grid_request + 1) & ~1), nullptr, attr);
    int clusters = 0;
    {
        std::lock_guard<std::mutex> lock(g_shape_mu);
        for (const MmaShape &sh : g_shapes)
            if (sh.device == device && sh.variant == v && sh.smem == cfg.dynamicSmemBytes) clusters = sh.clusters;
        if (clusters == 0) {
            // the attribute admits the largest size any trait count asks for
            e = cudaFuncSetAttribute(mma::k_scan_mma<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(typename C::Smem) + 1024 + smax_bytes(SMAX_TRAITS)));
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveClusters(&clusters, mma::k_scan_mma<C>, &cfg);
            if (e != cudaSuccess) return e;
            if (clusters < 1) return cudaErrorInvalidConfiguration;
            g_shapes.push_back({device, v, cfg.dynamicSmemBytes, clusters});
        }
    }
    *grid = std::min((int)cfg.gridDim.x, 2 * clusters);
    return cudaSuccess;
}

template <class C>
static cudaError_t enqueue(const ScanArgs &a, const MmaMaps &maps, int grid, cudaStream_t stream)
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = mma_config<C>(a.ntraits, grid, stream, attr);
    cudaError_t e = cudaLaunchKernelEx(&cfg, mma::k_scan_mma<C>, a, maps);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// The launch shape of a scan with variant v, resolved before any stream capture: the kernel's
// shared-memory attribute and the number of co-resident clusters, then whole clusters of two --
// at least one, never more than can be resident at once.
cudaError_t mma_prepare(int v, int ntraits, int grid_request, int *grid)
{
    switch (v) {
    case 0: return prepare<Rings0>(v, ntraits, grid_request, grid);
    case 1: return prepare<Rings1>(v, ntraits, grid_request, grid);
    case 2: return prepare<Rings2>(v, ntraits, grid_request, grid);
    case 3: return prepare<Rings3>(v, ntraits, grid_request, grid);
    case 4: return prepare<Rings4>(v, ntraits, grid_request, grid);
    case 5: return prepare<Rings5>(v, ntraits, grid_request, grid);
    }
    return cudaErrorInvalidValue;
}

// The launch itself (a stream operation only, so it can be captured into a CUDA graph).
cudaError_t mma_enqueue(int v, const ScanArgs &a, const MmaMaps &maps, int grid, cudaStream_t stream)
{
    switch (v) {
    case 0: return enqueue<Rings0>(a, maps, grid, stream);
    case 1: return enqueue<Rings1>(a, maps, grid, stream);
    case 2: return enqueue<Rings2>(a, maps, grid, stream);
    case 3: return enqueue<Rings3>(a, maps, grid, stream);
    case 4: return enqueue<Rings4>(a, maps, grid, stream);
    case 5: return enqueue<Rings5>(a, maps, grid, stream);
    }
    return cudaErrorInvalidValue;
}

}  // namespace epi
