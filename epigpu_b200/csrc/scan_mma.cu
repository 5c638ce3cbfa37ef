// scan_mma.cu -- tensor-core form of the pair scan (tcgen05, kind::i8, sm_100a).
//
// Per pair (i, j) the reference accumulates, over individuals k, the 3x3 genotype-cell
// counts and phenotype sums (src/EpiOpenCL.c:110-228). Both are contractions over k:
//     n_ab = sum_k [g_i(k)=a] [g_j(k)=b] w_k        S_ab = sum_k [g_i(k)=a] [g_j(k)=b] y_k
// so for a tile of 40 i-SNPs x 16 j-SNPs they are one integer GEMM
//     D[128 x 192] = A[128 x K] * B[K x 192]
//   A rows (TMEM lane 32w + l, l < 30): i-SNP 10w + l/3, genotype a = l%3: [g_i(k) == a]
//   B cols (type t = 4b + s, column 16t + j'): [g_j(k) == b] * D_s(k) with D_0 = w_k
//     (phenotype valid) and D_1..3 the balanced base-256 digits of the fixed-point
//     phenotype Y_k = round(y_k * 2^sy) (y centred, 0 when invalid).
// int8 operands, int32 accumulation: counts and digit sums are exact, so
//     S_ab = (D1 + 256 D2 + 65536 D3) * 2^-sy exactly for the quantised phenotype.
// The sum of y^2 over the pair's valid individuals comes from per-SNP FP64 terms and the
// (sparse) individuals missing on both SNPs:  Q_ij = Qtot - QM_i - QM_j + X_ij.
// The epilogue forms SSB / SSI / F / F2 in FP64 (pair_stat) from these exact inputs.
//
// Persistent kernel, one CTA per SM, warp-specialised, 14 warps:
//   warp 13     TMA loader (one thread): per 128-individual stage, three 2-D tiled loads
//               (no multicast) into a 6-deep raw ring: the i-tile's and j-tile's one-hot
//               genotype bytes (40 and 16 rows x 128 B) and the trait's 4 digit rows, all
//               128-byte swizzled; completion by mbarrier transaction bytes
//   warps 0-3   A producers: one TMEM lane each; expand the raw i rows into the stage's A
//               rows and store them into TMEM with tcgen05.st (the MMA reads A from TMEM)
//   warps 4-7   B producers: expand raw j rows x digits into the stage's B tile (K-major,
//               128-byte swizzle) in smem
//   warps 8-11  epilogue: tcgen05.ld of the accumulator, lane-triplet shuffles, FP64
//               statistics, warp-aggregated hit append, per-trait max F
//   warp 12     TMEM allocator and MMA issuer (one thread): 4 x tcgen05.mma per stage
// 4-stage operand pipeline, 2 TMEM accumulators (columns 0 and 192) so the epilogue of one
// tile overlaps the MMAs of the next. All waits are bounded (tc_ptx.cuh); a timeout sets
// counters[2] and every role leaves its loop.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "epi_internal.cuh"
#include "tc_ptx.cuh"

namespace epi {
namespace mma {

constexpr int TI = 40;         // i-SNPs per tile (4 warps x 10 lane triplets)
constexpr int TJ = 16;         // j-SNPs per tile
constexpr int NTYPE = 12;      // B column types per j-SNP: b (3) x {w, digit0, digit1, digit2}
constexpr int N = TJ * NTYPE;  // 192
constexpr int M = 128;
constexpr int KS = 128;        // individuals per pipeline stage
constexpr int STAGES = 4;
constexpr int ACC_COL1 = 192;  // second accumulator; first at column 0
constexpr int A_COL = 384;     // A stage s at TMEM columns A_COL + 32 s
constexpr uint32_t TMEM_COLS = 512;
constexpr int B_STAGE = N * KS;  // bytes per B stage (24 KB)
constexpr int RSTAGES = 6;       // raw (TMA) ring depth
constexpr int RAW_I = 0, RAW_J = TI * KS, RAW_D = RAW_I + 7 * 1024;  // 1024-aligned offsets in a raw stage
constexpr int RAW_STAGE = 8192;
constexpr uint32_t RAW_BYTES = (TI + TJ + 4) * KS;  // transaction bytes per raw stage
constexpr int NWARPS = 14;
constexpr int NTHREADS = NWARPS * 32;
constexpr uint32_t IDESC = tc::idesc_i8(M, N);
static_assert(RAW_J % 1024 == 0 && RAW_D >= RAW_J + TJ * KS && RAW_D + 4 * KS <= RAW_STAGE, "raw layout");

struct Smem {
    uint8_t b[STAGES][B_STAGE];
    uint8_t raw[RSTAGES][RAW_STAGE];
    uint64_t full[STAGES], empty[STAGES], raw_full[RSTAGES], raw_empty[RSTAGES], acc_full[2], acc_empty[2], drain;
    uint32_t tmem_base;
    int abort;
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

__device__ __forceinline__ Unit decode(const ScanArgs &a, long long u)
{
    Unit r;
    const long long tile = u / a.ntraits;
    r.trait = (int)(u % a.ntraits);
    r.block = find_block(a.blocks, a.nblocks, tile);
    r.bd = a.blocks[r.block];
    const long long lt = tile - r.bd.tile_base;
    r.i0 = (int)(lt / r.bd.tiles_j) * TI;
    r.j0 = (int)(lt % r.bd.tiles_j) * TJ;
    r.skip = r.bd.start1 + min(r.i0 + TI, r.bd.size1) - 1 <= r.bd.start2 + r.j0;
    return r;
}

__device__ __forceinline__ void fail(const ScanArgs &a, Smem &sm, int where)
{
    sm.abort = 1;
    if (atomicCAS(&a.counters[2], 0ull, 1ull) == 0ull) a.counters[3] = (unsigned long long)where;
}

__device__ __forceinline__ uint32_t sel3(const uint32_t v[4], int idx)
{
    return idx == 0 ? v[0] : (idx == 1 ? v[1] : v[2]);
}

// sum over individuals missing on both SNPs (and phenotype-valid) of y^2
__device__ __noinline__ double missing_both(const ScanArgs &a, int gi, int gj, int t)
{
    double x = 0.0;
    const uint32_t *si = a.misssum + (size_t)gi * a.Ws, *sj = a.misssum + (size_t)gj * a.Ws;
    const uint32_t *mi = a.missbits + (size_t)gi * a.Wp, *mj = a.missbits + (size_t)gj * a.Wp;
    const uint32_t *wt = a.wmask + (size_t)t * a.Wp;
    const double *qt = a.qd + (size_t)t * a.Np;
    for (int s = 0; s < a.Ws; ++s) {
        uint32_t m = si[s] & sj[s];
        while (m) {
            const int w = 32 * s + __ffs(m) - 1;
            m &= m - 1;
            uint32_t bits = mi[w] & mj[w] & wt[w];
            while (bits) {
                x += qt[32 * w + __ffs(bits) - 1];
                bits &= bits - 1;
            }
        }
    }
    return x;
}

struct PairIn {
    int n[9];
    long long s[9];
};

__device__ __noinline__ PairStat eval_pair(const ScanArgs &a, const PairIn in, int gi, int gj, int t, int di,
                                           int dj, int size2)
{
    double S[9];
    const double sc = a.yscale[t];
#pragma unroll
    for (int c = 0; c < 9; ++c) S[c] = (double)in.s[c] * sc;
    const double Q = a.qtot[t] - a.qm[(size_t)t * a.nsnp + gi] - a.qm[(size_t)t * a.nsnp + gj] +
                     missing_both(a, gi, gj, t);
    const PairStat s = pair_stat(in.n, S, Q, a.test_int != 0);
    if (t == a.report_trait && (a.dump_counts || a.dump_F)) {
        const size_t o = (size_t)di * size2 + dj;
        if (a.dump_counts)
            for (int c = 0; c < 9; ++c) a.dump_counts[9 * o + c] = in.n[c];
        if (a.dump_F) a.dump_F[o] = (float)s.F;
        if (a.dump_F2) a.dump_F2[o] = (float)s.F2;
        if (a.dump_df1) a.dump_df1[o] = s.d1;
        if (a.dump_df2) a.dump_df2[o] = s.d2;
    }
    return s;
}

__global__ void __launch_bounds__(NTHREADS, 1) k_scan_mma(ScanArgs a, const __grid_constant__ MmaMaps maps)
{
    extern __shared__ uint8_t smem_raw[];
    // the B stages need 1024-byte alignment (128-byte swizzle atoms)
    const uint32_t raw_s = tc::smem_u32(smem_raw);
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw + (((raw_s + 1023u) & ~1023u) - raw_s));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long units = a.ntiles * (long long)a.ntraits;
    const int nks = a.Np / KS;

    if (warp == 12) {
        tc::tmem_alloc(&sm.tmem_base, TMEM_COLS);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tc::mbar_init(&sm.full[s], 8);
            tc::mbar_init(&sm.empty[s], 1);
        }
        for (int r = 0; r < RSTAGES; ++r) {
            tc::mbar_init(&sm.raw_full[r], 1);
            tc::mbar_init(&sm.raw_empty[r], 8);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&sm.acc_full[b], 1);
            tc::mbar_init(&sm.acc_empty[b], 4);
        }
        tc::mbar_init(&sm.drain, 1);
        sm.abort = 0;
        tc::fence_barrier_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sm.tmem_base;
    volatile int *abort = &sm.abort;

    if (warp < 4) {
        // ---------------- A producers: TMEM lane = threadIdx.x ----------------
        const int ii = 10 * warp + lane / 3, ga = lane % 3;
        const bool rowok = lane < 30;
        const uint32_t taddr_lane = tmem + ((uint32_t)(32 * warp) << 16) + A_COL;
        uint32_t stage = 0, phase = 0, rs = 0, rph = 0;
        bool ok = true;
        for (long long u = blockIdx.x; u < units && ok; u += gridDim.x) {
            const Unit un = decode(a, u);
            if (un.skip) continue;
            for (int ks = 0; ks < nks; ++ks) {
                if (!tc::mbar_wait(&sm.raw_full[rs], rph, abort) || !tc::mbar_wait(&sm.empty[stage], phase ^ 1u, abort)) {
                    fail(a, sm, 1);
                    ok = false;
                    break;
                }
                uint32_t v[32];
                const uint8_t *ri = sm.raw[rs] + RAW_I;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const uint4 h = rowok ? ld_sw128(ri, ii, c) : make_uint4(0, 0, 0, 0);
                    v[4 * c + 0] = (h.x >> ga) & 0x01010101u;
                    v[4 * c + 1] = (h.y >> ga) & 0x01010101u;
                    v[4 * c + 2] = (h.z >> ga) & 0x01010101u;
                    v[4 * c + 3] = (h.w >> ga) & 0x01010101u;
                }
                tc::tmem_st32(taddr_lane + 32 * stage, v);
                tc::tmem_wait_st();
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    tc::mbar_arrive(&sm.full[stage]);
                    tc::mbar_arrive(&sm.raw_empty[rs]);
                }
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
                if (++rs == RSTAGES) {
                    rs = 0;
                    rph ^= 1u;
                }
            }
        }
    } else if (warp < 8) {
        // ---------------- B producers: thread -> (j-SNP, 16-individual chunk) ----------------
        const int t = threadIdx.x - 128, jj = t >> 3, c = t & 7;
        uint32_t stage = 0, phase = 0, rs = 0, rph = 0;
        bool ok = true;
        for (long long u = blockIdx.x; u < units && ok; u += gridDim.x) {
            const Unit un = decode(a, u);
            if (un.skip) continue;
            for (int ks = 0; ks < nks; ++ks) {
                if (!tc::mbar_wait(&sm.raw_full[rs], rph, abort) || !tc::mbar_wait(&sm.empty[stage], phase ^ 1u, abort)) {
                    fail(a, sm, 2);
                    ok = false;
                    break;
                }
                const uint8_t *raw = sm.raw[rs];
                const uint4 h = ld_sw128(raw + RAW_J, jj, c);
                uint4 d[4];
#pragma unroll
                for (int s2 = 0; s2 < 4; ++s2) d[s2] = ld_sw128(raw + RAW_D, s2, c);
                uint8_t *base = sm.b[stage];
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    uint4 m;
                    m.x = ((h.x >> b) & 0x01010101u) * 0xFFu;
                    m.y = ((h.y >> b) & 0x01010101u) * 0xFFu;
                    m.z = ((h.z >> b) & 0x01010101u) * 0xFFu;
                    m.w = ((h.w >> b) & 0x01010101u) * 0xFFu;
#pragma unroll
                    for (int s2 = 0; s2 < 4; ++s2) {
                        const int n = (4 * b + s2) * TJ + jj;
                        uint4 o;
                        o.x = m.x & d[s2].x;
                        o.y = m.y & d[s2].y;
                        o.z = m.z & d[s2].z;
                        o.w = m.w & d[s2].w;
                        *reinterpret_cast<uint4 *>(base + (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4)) = o;
                    }
                }
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tc::mbar_arrive(&sm.full[stage]);
                    tc::mbar_arrive(&sm.raw_empty[rs]);
                }
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
                if (++rs == RSTAGES) {
                    rs = 0;
                    rph ^= 1u;
                }
            }
        }
    } else if (warp < 12) {
        // ---------------- epilogue ----------------
        const int e = warp - 8;
        const int ii = 10 * e + lane / 3, ga = lane % 3, tbase = (lane / 3) * 3;
        const bool rowok = lane < 30;
        const uint32_t tl = tmem + ((uint32_t)(32 * e) << 16);
        uint32_t accph[2] = {0u, 0u};
        int buf = 0;
        for (long long u = blockIdx.x; u < units; u += gridDim.x) {
            const Unit un = decode(a, u);
            if (un.skip) continue;
            if (!tc::mbar_wait(&sm.acc_full[buf], accph[buf], abort)) {
                fail(a, sm, 3);
                break;
            }
            tc::tc_fence_after();
            const uint32_t acc = tl + (buf ? ACC_COL1 : 0);
            const int t = un.trait;
            const bool report = a.report_trait < 0 || a.report_trait == t;
            const int di = un.i0 + ii;
            const bool ivalid = rowok && di < un.bd.size1;
#pragma unroll 1
            for (int rho = 0; rho < (TJ + 2) / 3; ++rho) {
                const int jb = 3 * rho;
                uint32_t v[NTYPE][4];
#pragma unroll
                for (int ty = 0; ty < NTYPE; ++ty) tc::tmem_ld4(acc + ty * TJ + jb, v[ty][0], v[ty][1], v[ty][2], v[ty][3]);
                tc::tmem_wait_ld();
                // rows (ii, a') for my j-SNP jb + ga: own row directly, the others by shuffle
                uint32_t r1[NTYPE], r2[NTYPE];
#pragma unroll
                for (int ty = 0; ty < NTYPE; ++ty) {
                    r1[ty] = __shfl_sync(0xffffffffu, sel3(v[ty], (ga + 2) % 3), tbase + (ga + 1) % 3);
                    r2[ty] = __shfl_sync(0xffffffffu, sel3(v[ty], (ga + 1) % 3), tbase + (ga + 2) % 3);
                }
                const int dj = un.j0 + jb + ga;
                const bool valid = ivalid && (jb + ga < TJ) && dj < un.bd.size2 &&
                                   (un.bd.start1 + di > un.bd.start2 + dj);
                PairStat s;
                s.nfac = s.d1 = s.d2 = 0;
                s.F = s.F2 = 0.0;
                if (valid) {
                    PairIn in;
#pragma unroll
                    for (int ap = 0; ap < 3; ++ap) {
                        // row a' = ga + ap (mod 3): ap = 0 own, 1 from r1, 2 from r2
                        const int arow = (ga + ap) % 3;
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            uint32_t w0, w1, w2, w3;
                            if (ap == 0) {
                                w0 = sel3(v[4 * b], ga); w1 = sel3(v[4 * b + 1], ga);
                                w2 = sel3(v[4 * b + 2], ga); w3 = sel3(v[4 * b + 3], ga);
                            } else if (ap == 1) {
                                w0 = r1[4 * b]; w1 = r1[4 * b + 1]; w2 = r1[4 * b + 2]; w3 = r1[4 * b + 3];
                            } else {
                                w0 = r2[4 * b]; w1 = r2[4 * b + 1]; w2 = r2[4 * b + 2]; w3 = r2[4 * b + 3];
                            }
                            const int cell = 3 * arow + b;
                            in.n[cell] = (int)w0;
                            in.s[cell] = (long long)(int)w1 + 256LL * (long long)(int)w2 + 65536LL * (long long)(int)w3;
                        }
                    }
                    s = eval_pair(a, in, un.bd.start1 + di, un.bd.start2 + dj, t, di, dj, un.bd.size2);
                }
                const bool hit = valid && report && is_hit(a, s);
                emit_hit(a, hit, un.bd.start1 + di, un.bd.start2 + dj, s, t, un.block);
                fold_max(&a.maxf[t], valid, s.F);
                if (a.test_int) fold_max(&a.maxf2[t], valid, s.F2);
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sm.acc_empty[buf]);
            accph[buf] ^= 1u;
            buf ^= 1;
        }
    } else if (warp == 13) {
        // ---------------- TMA loader ----------------
        if (lane == 0) {
            uint32_t rs = 0, rph = 0, issued = 0;
            bool ok = true;
            for (long long u = blockIdx.x; u < units && ok; u += gridDim.x) {
                const Unit un = decode(a, u);
                if (un.skip) continue;
                for (int ks = 0; ks < nks; ++ks) {
                    if (!tc::mbar_wait(&sm.raw_empty[rs], rph ^ 1u, abort)) {
                        fail(a, sm, 7);
                        ok = false;
                        break;
                    }
                    uint8_t *raw = sm.raw[rs];
                    tc::mbar_arrive_expect_tx(&sm.raw_full[rs], RAW_BYTES);
                    tc::tma_load_2d(raw + RAW_I, &maps.hi, ks * KS, un.bd.start1 + un.i0, &sm.raw_full[rs]);
                    tc::tma_load_2d(raw + RAW_J, &maps.hj, ks * KS, un.bd.start2 + un.j0, &sm.raw_full[rs]);
                    tc::tma_load_2d(raw + RAW_D, &maps.dg, ks * KS, 4 * un.trait, &sm.raw_full[rs]);
                    ++issued;
                    if (++rs == RSTAGES) {
                        rs = 0;
                        rph ^= 1u;
                    }
                }
            }
            // no TMA write may still be landing in shared memory when the CTA exits: wait for
            // the last load issued into every ring slot (already complete on the normal path)
            int no_abort = 0;
            for (uint32_t k = 0; k < RSTAGES && k < issued; ++k) {
                // the slot used k+1 loads ago, and the parity its load completes
                const uint32_t back = k + 1;
                const uint32_t slot = (rs + RSTAGES - (back % RSTAGES)) % RSTAGES;
                const uint32_t par = (back > rs) ? (rph ^ 1u) : rph;
                if (!tc::mbar_wait(&sm.raw_full[slot], par, &no_abort)) fail(a, sm, 8);
            }
        }
    } else if (lane == 0) {
        // ---------------- MMA issuer ----------------
        uint32_t stage = 0, phase = 0, accph[2] = {0u, 0u};
        int buf = 0;
        bool ok = true;
        for (long long u = blockIdx.x; u < units && ok; u += gridDim.x) {
            const Unit un = decode(a, u);
            if (un.skip) continue;
            if (!tc::mbar_wait(&sm.acc_empty[buf], accph[buf] ^ 1u, abort)) {
                fail(a, sm, 4);
                break;
            }
            tc::tc_fence_after();
            const uint32_t d = tmem + (buf ? ACC_COL1 : 0);
            for (int ks = 0; ks < nks; ++ks) {
                if (!tc::mbar_wait(&sm.full[stage], phase, abort)) {
                    fail(a, sm, 5);
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t bs = tc::smem_u32(sm.b[stage]);
#pragma unroll
                for (int kk = 0; kk < KS / 32; ++kk)
                    tc::mma_i8_ts(d, tmem + A_COL + 32 * stage + 8 * kk, tc::smem_desc_sw128(bs + 32 * kk), IDESC,
                                  (ks | kk) != 0);
                tc::mma_commit(&sm.empty[stage]);
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
            if (!ok) break;
            tc::mma_commit(&sm.acc_full[buf]);
            accph[buf] ^= 1u;
            buf ^= 1;
        }
        // every MMA issued above has completed once `drain` flips (waited for even after an
        // abort: the accumulators and A stages must be idle before the TMEM is released)
        tc::mma_commit(&sm.drain);
        int no_abort = 0;
        if (!tc::mbar_wait(&sm.drain, 0, &no_abort)) fail(a, sm, 6);
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 12) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace mma

// Tensor maps of the tensor form's TMA loads: the one-hot genotype bytes [nsnp][Np] with
// boxes of 40 and 16 rows x 128 bytes, and the trait digit rows [4T][Np] with 4-row boxes;
// all 128-byte swizzled, out-of-range rows read as zero.
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

cudaError_t mma_encode_genotypes(MmaMaps *maps, const uint8_t *hcodes, int nsnp, int Np)
{
    cudaError_t e = encode_2d(&maps->hi, hcodes, (uint64_t)Np, (uint64_t)nsnp, mma::TI);
    if (e == cudaSuccess) e = encode_2d(&maps->hj, hcodes, (uint64_t)Np, (uint64_t)nsnp, mma::TJ);
    return e;
}

cudaError_t mma_encode_traits(MmaMaps *maps, const int8_t *ydig, int ntraits, int Np)
{
    return encode_2d(&maps->dg, ydig, (uint64_t)Np, (uint64_t)4 * ntraits, 4);
}

bool mma_available() { return true; }
int mma_tile_i() { return mma::TI; }
int mma_tile_j() { return mma::TJ; }
int mma_min_nid() { return 256; }
int mma_stage_individuals() { return mma::KS; }

cudaError_t launch_mma(const ScanArgs &a, const MmaMaps &maps, int grid, cudaStream_t stream)
{
    // more than half of the SM's shared memory: one CTA per SM, which owns all 512 TMEM columns
    const size_t smem = sizeof(mma::Smem) + 1024;
    static_assert(sizeof(mma::Smem) + 1024 > 116 * 1024, "one CTA per SM");
    cudaError_t e = cudaFuncSetAttribute(mma::k_scan_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    mma::k_scan_mma<<<grid, mma::NTHREADS, smem, stream>>>(a, maps);
    return cudaGetLastError();
}

}  // namespace epi
