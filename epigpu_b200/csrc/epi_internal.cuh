// epi_internal.cuh -- device-side structures shared by the scan kernels of libepigpu.so.
//
// Data layout in HBM (built once per epi_load_packed / epi_set_traits):
//   planes  uint4 [nsnp][Wp]      genotype bit-planes per 32 individuals:
//                                 x = [g==0], y = [g==1], z = [g==2], w = [g!=3]
//   codes   uint32 [nsnp][Wc]     2-bit codes, 16 individuals per word, LSB first,
//                                 padding individuals coded 3 (missing)
//   y       float [T][Np]         trait column centred by its valid mean, 0 where invalid
//   q       float [T][Np]         y^2 - qc[t] (qc = mean of y^2 over valid), 0 where invalid
//   wmask   uint32 [T][Wp]        phenotype-valid bits
//   maj     uint8 [nsnp]          most frequent genotype of each SNP (plain form)
//   pmC, pmN, pmQ                 plain form: per (trait, SNP) the sums of y and the counts by
//                                 genotype, and the sum of y^2 over the SNP's missing calls
// and for the tensor-core form
//   hcodes  uint8 [nsnp][Np]      one-hot genotype byte: 1 << g for g in 0..2, 0 if missing
//   missbits uint32 [nsnp][Wp]    missing-genotype bits
//   ydig    int8 [T][4][Np]       per individual: phenotype-valid flag and the three balanced
//                                 base-256 digits (low first) of Y = round(y * 2^sy)
//   qd      double [2][T][Np]     ytilde^2 (ytilde = Y 2^-sy, the quantised y), then Y itself;
//                                 0 where invalid; per trait qtot = sum of ytilde^2, ytot = sum
//                                 of Y, nvalid = count over the valid individuals
//   qm, sm, nm double [T][nsnp]   the sums of ytilde^2 and of Y, and the count, over the valid
//                                 individuals missing at that SNP
// Individuals are padded to Np = 32*Wp (a multiple of 128); padding carries no genotype
// and no phenotype.
#pragma once
#include <cstdint>
#include <cstring>
#include <cuda.h>
#include <cuda_runtime.h>

namespace epi {

// The scan kernels keep per-CTA maxima of F and F2 in shared memory (8 bytes per trait,
// flushed to global memory once per CTA) for up to this many traits; larger trait sets (a
// permutation run of thousands of phenotypes) fold straight into the global maxima.
constexpr int SMAX_TRAITS = 512;
__host__ __device__ constexpr size_t smax_bytes(int ntraits)
{
    return ntraits <= SMAX_TRAITS ? 8 * (size_t)ntraits : 0;
}

// One hit as written by a kernel; sorted into the reference's output order on the host.
struct DevHit {
    int32_t snp1, snp2, df1, df2;
    float F, F2;
    int32_t trait, block;
};

// A chromosome block of the scan and its tiling (tiles_i x tiles_j tiles of the
// kernel's tile shape); tile_base is the global index of the block's first tile.
struct BlockDesc {
    int32_t start1, size1, start2, size2;
    int32_t tiles_i, tiles_j;
    int64_t tile_base;
};

// The reference's 24-byte result row (src/id4117.h:14-21), as written on the device by the
// allocation-free entry point.
struct HitRow {
    int32_t snp1, snp2, df1, df2;
    float F, F2;
};

struct ScanArgs {
    // genotypes
    const uint4 *planes;
    const uint32_t *codes;
    const uint8_t *hcodes;
    const uint32_t *missbits;
    int32_t Wp, Wc, nid, nsnp;
    // traits
    const float *y, *q;
    const uint32_t *wmask;
    const double *qc;          // [T]
    const double *yscale;      // [T] (tensor form: 2^-sy)
    const double *qd, *qtot, *qm, *sm, *nm;  // tensor form (layout above)
    const double *ytot, *nvalid;             // [T] (tensor form)
    const int8_t *ydig;
    // plain form: per SNP the most frequent genotype; per (trait, SNP) the FP64 marginals by
    // genotype -- sum of y [T][nsnp][3], count [T][nsnp][3], sum of y^2 over the individuals
    // missing at the SNP [T][nsnp] -- and per trait the sum of y^2 over valid individuals
    const uint8_t *maj;
    const double *pmC;
    const int32_t *pmN;
    const double *pmQ, *ysq;
    int32_t Np, ntraits;
    // blocks / tiles
    const BlockDesc *blocks;
    int32_t nblocks;
    int64_t ntiles;
    // test
    int32_t test_int, safe, report_trait;
    float t1, t2;
    // tensor form: limit of every device-side wait (ns); test hook that makes one wait run out
    unsigned long long wait_ns;
    int32_t debug_stall;
    // tensor form, streamed-B variant: the unit order walks super-tiles of xsi x xsj pair
    // tiles, so that their A rows and expanded B rows stay in L2 together
    int32_t xsi, xsj;
    // outputs
    DevHit *hits;
    int64_t cap;
    unsigned long long *counters;  // [0] hits found, [1] tile queue, [2] error flag, [3] error site
    unsigned int *maxf, *maxf2;    // [T] order-preserving encoded floats
    // optional dump of one block (pair (gx, gy) at gx*size2 + gy)
    int32_t *dump_counts;
    float *dump_F, *dump_F2;
    int32_t *dump_df1, *dump_df2;
    // allocation-free entry point only: genotypes read straight from the reference's
    // packed words, hits written as 24-byte result rows
    const int32_t *gpack;
    int32_t npack, remain;
    HitRow *rows;
};


// TMA descriptors of the tensor form (kernel parameter, __grid_constant__)
struct MmaMaps {
    CUtensorMap hi, hj, dg, hx;  // hx: the expanded B rows of the streamed-B variant
};

// TMA descriptors of the plain form: the genotype plane words, in boxes of the tile's i-SNPs
// and of its j-SNPs
struct PopcMaps {
    CUtensorMap planes_i, planes_j;
};

// float -> unsigned with the same order (for atomicMax over possibly negative F)
__device__ __forceinline__ unsigned int f2ord(float f)
{
    unsigned int b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ inline float ord2f(unsigned int u)
{
    unsigned int b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

struct PairStat {
    int nfac, d1, d2;
    double F, F2;
};

// The reference's per-pair statistics (src/EpiOpenCL.c:231-247 and :452-486) in FP64
// from exact cell counts n[9], cell sums S[9] of the centred trait, and
// Qv = sum over valid individuals of y^2 (centred). With m the pair's valid mean:
//   SSY = Qv - N m^2, SSB = sum_c n_c (m_c - m)^2, d1 = nfac-1, d2 = N - nfac,
//   F = (SSB/d1) / ((SSY-SSB)/d2);  4 df: row/column means from raw sums (:466-467),
//   SSI = sum_c n_c (m_ab - r_a - c_b + m)^2, F2 = (SSI/4) / MSW.
// d1 == 0 gives SSB == 0 and F = 0/0 = NaN (never a hit).
//
// Resolution floor: SSW = SSY - SSB cancels when the pair's cells explain nearly all of the
// variance, and once SSW falls below the rounding error of the sums it came from, its value
// (and sign) is noise. The caller states that error as a fraction of SSY (ssw_floor); below
// it SSW is taken as ssw_floor * SSY, so F is a lower bound of the true F (which is larger
// still) and such a pair stays a hit; the relative error in F stays within the documented
// 1e-5 * SSY / SSW. NaN inputs stay NaN.
__device__ __forceinline__ double ssw_floored(double SSY, double SSB, double ssw_floor)
{
    const double SSW = SSY - SSB;
    return SSW < ssw_floor * SSY ? ssw_floor * SSY : SSW;
}

// floor for sums accumulated in FP32 over the individuals (the plain form)
constexpr double SSW_FLOOR_F32 = 1e-5;
// floor for the tensor form's exact integer sums (its Q carries the doubly-missing residual
// approximation, at most ~1e-8 of SSY)
constexpr double SSW_FLOOR_EXACT = 1e-7;

__device__ __forceinline__ PairStat pair_stat(const int n[9], const double S[9], double Qv, bool want_int)
{
    PairStat r;
    int N = 0, nfac = 0;
    double St = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        N += n[c];
        St += S[c];
        nfac += n[c] > 0;
    }
    const double m = St / (double)N;
    const double SSY = Qv - St * m;
    double mc[9], SSB = 0.0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        mc[c] = 0.0;
        if (n[c] > 0) {
            mc[c] = S[c] / (double)n[c];
            const double d = mc[c] - m;
            SSB += (double)n[c] * d * d;
        }
    }
    r.nfac = nfac;
    r.d1 = nfac - 1;
    r.d2 = N - nfac;
    const double MSW = ssw_floored(SSY, SSB, SSW_FLOOR_F32) / (double)r.d2;
    r.F = (SSB / (double)r.d1) / MSW;
    r.F2 = 0.0;
    if (want_int) {
        double row[3], col[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            col[i] = (S[i] + S[i + 3] + S[i + 6]) / (double)(n[i] + n[i + 3] + n[i + 6]);
            row[i] = (S[3 * i] + S[3 * i + 1] + S[3 * i + 2]) / (double)(n[3 * i] + n[3 * i + 1] + n[3 * i + 2]);
        }
        double SSI = 0.0;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            if (n[c] > 0) {
                const double t = mc[c] - row[c / 3] - col[c % 3] + m;
                SSI += (double)n[c] * t * t;
            }
        }
        r.F2 = (SSI / 4.0) / MSW;
    }
    return r;
}

// Hit rule: EpiOpenCL.c:251 (8 df), :487-489 (4 df, nfac > 6), :949 (safe 4 df, no filter).
__device__ __forceinline__ bool is_hit(const ScanArgs &a, const PairStat &s)
{
    if (!a.test_int) return s.F > (double)a.t1;
    return (s.F > (double)a.t1 || s.F2 > (double)a.t2) && (a.safe || s.nfac > 6);
}

// Warp-aggregated append of one candidate per lane. Every lane of the warp must call it.
__device__ __forceinline__ void emit_hit(const ScanArgs &a, bool hit, int snp1, int snp2,
                                         const PairStat &s, int trait, int block)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (mask == 0u) return;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(&a.counters[0], (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
        const unsigned long long idx = base + __popc(mask & ((1u << lane) - 1u));
        if ((long long)idx < a.cap) {
            DevHit h;
            h.snp1 = snp1;
            h.snp2 = snp2;
            h.df1 = s.d1;
            h.df2 = s.d2;
            h.F = (float)s.F;
            h.F2 = a.test_int ? (float)s.F2 : 0.0f;
            h.trait = trait;
            h.block = block;
            a.hits[idx] = h;
        }
    }
}

// Warp-aggregated append of 24-byte result rows (allocation-free entry point).
__device__ __forceinline__ void emit_row(const ScanArgs &a, bool hit, int snp1, int snp2, const PairStat &s)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (mask == 0u) return;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(&a.counters[0], (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
        const unsigned long long idx = base + __popc(mask & ((1u << lane) - 1u));
        if ((long long)idx < a.cap) {
            HitRow h;
            h.snp1 = snp1;
            h.snp2 = snp2;
            h.df1 = s.d1;
            h.df2 = s.d2;
            h.F = (float)s.F;
            h.F2 = a.test_int ? (float)s.F2 : 0.0f;
            a.rows[idx] = h;
        }
    }
}

// Warp max of F (NaN ignored) folded into the per-trait maximum. Every lane calls it.
// Warp maximum of already-encoded values, one atomicMax on `slot` (every lane must call it).
__device__ __forceinline__ void fold_max_enc(unsigned int *slot, unsigned int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31u) == 0u && v) atomicMax(slot, v);
}

__device__ __forceinline__ void fold_max(unsigned int *slot, bool valid, double F)
{
    unsigned int v = (valid && F == F) ? f2ord((float)F) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31u) == 0u && v) atomicMax(slot, v);
}

// Tile t -> block index (binary search over tile_base).
__device__ __forceinline__ int find_block(const BlockDesc *b, int nb, long long t)
{
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace epi
