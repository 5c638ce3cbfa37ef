// scan_noalloc.cu -- the allocation-free entry point (epi_scan_block_noalloc) and the
// kernel it runs: a popcount-form pair scan that reads the reference's packed genotype
// words directly (src/readplink.c:1066-1102) and writes 24-byte result rows, with all of its
// working memory in one fixed device array.
//
// The kernel is the reference's per-individual method (src/EpiOpenCL.c:110-228: unpack two
// SNPs, count the 3x3 genotype cells, add the phenotype into its cell) on the CUDA cores.
// Persistent, one 512-thread CTA per SM, pulling 64 x 32 SNP-pair tiles from a queue. Per
// tile it walks the individuals in stages of 64:
//   * stage expansion: the i-tile's genotype bits become U_a = [g_i==a]*y and U_V = [g_i valid]
//     as floats in shared memory (read by the whole warp: broadcast loads);
//   * cell counts: AND + __popc of 32-bit plane words (phenotype mask folded into the
//     i side), 16-bit packed counters;
//   * cell sums: each lane turns its own j-SNP's plane bits into F_b = [g_j==b] and
//     F_Q = [g_j valid]*q in registers, then S_ab += U_a*F_b (9 FP32 FMAs per pair and
//     individual) and Q += U_V*F_Q (sum of y^2 over valid individuals, q = y^2 - mean y^2).
// Each thread owns 4 whole pairs (the warp's four i-SNPs x the lane's j-SNP).
// Epilogue: FP64 SSB/SSI/F/F2 per pair, warp-aggregated atomic row append, maximum F.
#include "epi_internal.cuh"
#include "epigpu.h"

namespace epi {
namespace popc_raw {

constexpr int TI = 64;   // i-SNPs per tile (16 warps x 4, shared by the warp's lanes)
constexpr int TJ = 32;   // j-SNPs per tile (one per lane)
constexpr int NT = 512;
constexpr int KI = 64;   // individuals per stage
constexpr int KW = 2;    // 32-individual words per stage
constexpr int KP = 32;   // individual pairs per stage

struct __align__(16) Smem {
    float4 u[KP][2][TI];  // [0] = (U0a, U0b, U1a, U1b), [1] = (U2a, U2b, UVa, UVb)
    uint4 pi[KW][TI];     // i-side planes AND phenotype mask
    uint4 pj[KW][TJ];     // j-side planes
    float2 q[KP];         // q of the two individuals of each pair
    long long tile;
};

__device__ __forceinline__ float bitf(uint32_t w, int b) { return ((w >> b) & 1u) ? 1.0f : 0.0f; }
__device__ __forceinline__ float bitsel(uint32_t w, int b, float v) { return ((w >> b) & 1u) ? v : 0.0f; }

__device__ __forceinline__ void count9(uint32_t c[5], const uint4 &p, const uint4 &r)
{
    c[0] += __popc(p.x & r.x) + (__popc(p.x & r.y) << 16);
    c[1] += __popc(p.x & r.z) + (__popc(p.y & r.x) << 16);
    c[2] += __popc(p.y & r.y) + (__popc(p.y & r.z) << 16);
    c[3] += __popc(p.z & r.x) + (__popc(p.z & r.y) << 16);
    c[4] += __popc(p.z & r.z);
}

// Genotype bit-planes of 32 individuals (word w) of one SNP: from the library's plane array,
// or, in the allocation-free variant, decoded straight from the reference's packed row
// (src/readplink.c:1066-1102: MSB-first words, right-aligned tail word).
template <bool RAW>
__device__ __forceinline__ uint4 load_planes(const ScanArgs &a, int snp, int w)
{
    if (!RAW) return a.planes[(size_t)snp * a.Wp + w];
    const int npack1 = a.remain ? a.npack + 1 : a.npack;
    const uint32_t *row = reinterpret_cast<const uint32_t *>(a.gpack) + (size_t)snp * npack1;
    uint32_t p0 = 0, p1 = 0, p2 = 0;
#pragma unroll 4
    for (int t = 0; t < 32; ++t) {
        const int k = 32 * w + t;
        uint32_t c = 3u;
        if (k < 16 * a.npack) c = (__ldg(row + (k >> 4)) >> (30 - 2 * (k & 15))) & 3u;
        else if (k < a.nid) c = (__ldg(row + a.npack) >> (2 * (a.remain - 1 - (k - 16 * a.npack)))) & 3u;
        p0 |= (uint32_t)(c == 0u) << t;
        p1 |= (uint32_t)(c == 1u) << t;
        p2 |= (uint32_t)(c == 2u) << t;
    }
    return make_uint4(p0, p1, p2, p0 | p1 | p2);
}

struct PairAcc {
    uint32_t C[5];
    float S[9];
    float Q;
};

// FP64 statistics of one pair from its packed counts, FP32 cell sums and y^2 sum; also
// writes the optional per-pair dump. Kept out of line: the kernel's accumulators stay in
// registers and only this call's arguments go through the stack.
__device__ __noinline__ PairStat eval_pair(const ScanArgs &a, const PairAcc acc, double qc, int t, int gi, int gj,
                                           int size2)
{
    int n[9];
    double Sd[9];
    int N = 0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        n[c] = (int)((acc.C[c >> 1] >> (16 * (c & 1))) & 0xffffu);
        Sd[c] = (double)acc.S[c];
        N += n[c];
    }
    const PairStat s = pair_stat(n, Sd, (double)acc.Q + qc * (double)N, a.test_int != 0);
    if (t == a.report_trait) {
        const size_t o = (size_t)gi * size2 + gj;
        if (a.dump_counts)
#pragma unroll
            for (int c = 0; c < 9; ++c) a.dump_counts[9 * o + c] = n[c];
        if (a.dump_F) a.dump_F[o] = (float)s.F;
        if (a.dump_F2) a.dump_F2[o] = (float)s.F2;
        if (a.dump_df1) a.dump_df1[o] = s.d1;
        if (a.dump_df2) a.dump_df2[o] = s.d2;
    }
    return s;
}

// RAW = false: the library path (epi_scan). RAW = true: the allocation-free variant,
// reading the reference's packed words and writing 24-byte rows (epi_scan_block_noalloc).
template <bool RAW>
__global__ void __launch_bounds__(NT, 1) k_scan_popc(ScanArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nstages = a.Wp / KW;
    // maxima of F and F2 per trait: per CTA in shared memory (flushed to global memory once,
    // at the end) up to SMAX_TRAITS traits, else the global maxima directly
    const bool smax_local = a.ntraits <= SMAX_TRAITS;
    unsigned int *smax = reinterpret_cast<unsigned int *>(smem_raw + sizeof(Smem));
    if (smax_local)
        for (int w = tid; w < 2 * a.ntraits; w += NT) smax[w] = 0u;
    unsigned int *const mxf = smax_local ? smax : a.maxf;
    unsigned int *const mxf2 = smax_local ? smax + a.ntraits : a.maxf2;

    for (;;) {
        if (tid == 0) sm.tile = (long long)atomicAdd(&a.counters[1], 1ull);
        __syncthreads();
        const long long tile = sm.tile;
        __syncthreads();
        if (tile >= a.ntiles) break;
        const int b = find_block(a.blocks, a.nblocks, tile);
        const BlockDesc bd = a.blocks[b];
        const long long lt = tile - bd.tile_base;
        const int i0 = (int)(lt / bd.tiles_j) * TI, j0 = (int)(lt % bd.tiles_j) * TJ;
        // no pair with snp1 > snp2 in this tile (upper part of a diagonal block)
        if (bd.start1 + min(i0 + TI, bd.size1) - 1 <= bd.start2 + j0) continue;

        for (int t = 0; t < a.ntraits; ++t) {
            const float *yt = a.y + (size_t)t * a.Np;
            const float *qt = a.q + (size_t)t * a.Np;
            const uint32_t *wt = a.wmask + (size_t)t * a.Wp;
            float S[4][9];
            float Q[4];
            uint32_t C[4][5];
#pragma unroll
            for (int ii = 0; ii < 4; ++ii) {
#pragma unroll
                for (int c = 0; c < 9; ++c) S[ii][c] = 0.0f;
                Q[ii] = 0.0f;
#pragma unroll
                for (int c = 0; c < 5; ++c) C[ii][c] = 0u;
            }

            for (int st = 0; st < nstages; ++st) {
                const int w0 = st * KW, k0 = st * KI;
                __syncthreads();
                {   // i side: thread -> (i, 8 individuals)
                    const int i = tid >> 3, part = tid & 7;
                    const int gi = i0 + i;
                    uint4 P = make_uint4(0, 0, 0, 0);
                    if (gi < bd.size1) P = load_planes<RAW>(a, bd.start1 + gi, w0 + (part >> 2));
                    const float4 ya = *reinterpret_cast<const float4 *>(yt + k0 + 8 * part);
                    const float4 yb = *reinterpret_cast<const float4 *>(yt + k0 + 8 * part + 4);
                    const float yv[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
                    const int bit0 = 8 * (part & 3);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int bA = bit0 + 2 * e, bB = bA + 1;
                        const float yA = yv[2 * e], yB = yv[2 * e + 1];
                        sm.u[part * 4 + e][0][i] = make_float4(bitsel(P.x, bA, yA), bitsel(P.x, bB, yB),
                                                               bitsel(P.y, bA, yA), bitsel(P.y, bB, yB));
                        sm.u[part * 4 + e][1][i] = make_float4(bitsel(P.z, bA, yA), bitsel(P.z, bB, yB),
                                                               bitf(P.w, bA), bitf(P.w, bB));
                    }
                }
                if (tid < KW * TI) {
                    const int w = tid / TI, i = tid % TI, gi = i0 + i;
                    uint4 P = make_uint4(0, 0, 0, 0);
                    if (gi < bd.size1) P = load_planes<RAW>(a, bd.start1 + gi, w0 + w);
                    const uint32_t W = wt[w0 + w];
                    sm.pi[w][i] = make_uint4(P.x & W, P.y & W, P.z & W, 0u);
                } else if (tid < KW * TI + KW * TJ) {
                    const int idx = tid - KW * TI, w = idx / TJ, j = idx % TJ, gj = j0 + j;
                    uint4 P = make_uint4(0, 0, 0, 0);
                    if (gj < bd.size2) P = load_planes<RAW>(a, bd.start2 + gj, w0 + w);
                    sm.pj[w][j] = P;
                } else if (tid < KW * TI + KW * TJ + KP) {
                    const int kp = tid - KW * TI - KW * TJ;
                    sm.q[kp] = *reinterpret_cast<const float2 *>(qt + k0 + 2 * kp);
                }
                __syncthreads();

#pragma unroll
                for (int w = 0; w < KW; ++w) {
                    const uint4 r = sm.pj[w][lane];
#pragma unroll
                    for (int ii = 0; ii < 4; ++ii) count9(C[ii], sm.pi[w][warp * 4 + ii], r);
                }
#pragma unroll
                for (int w = 0; w < KW; ++w) {
                    // this lane's j-SNP: indicator floats from its plane bits
                    const uint4 r = sm.pj[w][lane];
#pragma unroll 1
                    for (int h = 0; h < 16; ++h) {
                        const int kp = 16 * w + h, bA = 2 * h, bB = bA + 1;
                        const float2 qq = sm.q[kp];
                        const float F[3][2] = {{bitf(r.x, bA), bitf(r.x, bB)},
                                               {bitf(r.y, bA), bitf(r.y, bB)},
                                               {bitf(r.z, bA), bitf(r.z, bB)}};
                        const float FQa = bitsel(r.w, bA, qq.x), FQb = bitsel(r.w, bB, qq.y);
#pragma unroll
                        for (int ii = 0; ii < 4; ++ii) {
                            const float4 ua = sm.u[kp][0][warp * 4 + ii], ub = sm.u[kp][1][warp * 4 + ii];
                            const float U[3][2] = {{ua.x, ua.y}, {ua.z, ua.w}, {ub.x, ub.y}};
#pragma unroll
                            for (int x = 0; x < 3; ++x)
#pragma unroll
                                for (int y = 0; y < 3; ++y) {
                                    S[ii][3 * x + y] = fmaf(U[x][0], F[y][0], S[ii][3 * x + y]);
                                    S[ii][3 * x + y] = fmaf(U[x][1], F[y][1], S[ii][3 * x + y]);
                                }
                            Q[ii] = fmaf(ub.z, FQa, Q[ii]);
                            Q[ii] = fmaf(ub.w, FQb, Q[ii]);
                        }
                    }
                }
            }

            // epilogue
            const double qc = a.qc[t];
            const bool report = a.report_trait < 0 || a.report_trait == t;
#pragma unroll
            for (int ii = 0; ii < 4; ++ii) {
                const int gi = i0 + warp * 4 + ii, gj = j0 + lane;
                const bool valid = gi < bd.size1 && gj < bd.size2 && (bd.start1 + gi > bd.start2 + gj);
                PairStat s;
                s.nfac = s.d1 = s.d2 = 0;
                s.F = s.F2 = 0.0;
                if (valid) {
                    PairAcc acc;
#pragma unroll
                    for (int c = 0; c < 5; ++c) acc.C[c] = C[ii][c];
#pragma unroll
                    for (int c = 0; c < 9; ++c) acc.S[c] = S[ii][c];
                    acc.Q = Q[ii];
                    s = eval_pair(a, acc, qc, t, gi, gj, bd.size2);
                }
                const bool hit = valid && report && is_hit(a, s);
                if (RAW) emit_row(a, hit, bd.start1 + gi, bd.start2 + gj, s);
                else emit_hit(a, hit, bd.start1 + gi, bd.start2 + gj, s, t, b);
                fold_max(&mxf[t], valid, s.F);
                if (a.test_int) fold_max(&mxf2[t], valid, s.F2);
            }
        }
    }
    __syncthreads();
    if (smax_local)
        for (int w = tid; w < 2 * a.ntraits; w += NT)
            if (smax[w]) atomicMax(w < a.ntraits ? &a.maxf[w] : &a.maxf2[w - a.ntraits], smax[w]);
}

}  // namespace popc_raw

}  // namespace epi

// ---------------------------------------------------------------------------------------
// Allocation-free entry point (epi_scan_block_noalloc).
//
// Some callers cannot allocate GPU memory: code that must not call cudaMalloc while it runs
// (a latency-critical service or a real-time loop after start-up), or a host framework
// that hands out device memory only from its own pool. They pass device buffers for every
// input and output, and the scan's working memory -- hit/tile counters, the block
// descriptor, the per-trait maxima and the centred phenotype arrays -- lives in the fixed
// array below, sized for at most EPI_NOALLOC_MAX_NID individuals (about 520 KiB, held by
// every GPU that loads the library until the process exits).
// ---------------------------------------------------------------------------------------
namespace epi {
namespace noalloc {

constexpr int NP_MAX = 65536;  // individuals, padded to a multiple of 128

struct Scratch {
    unsigned long long counters[4];  // hits found, tile queue, error flag, error site
    unsigned int maxf[2];            // order-encoded max F and max F2
    double qc;                       // mean of the centred phenotype's square
    BlockDesc block;
    float y[NP_MAX];                 // centred phenotype (0 where missing)
    float q[NP_MAX];                 // y^2 - qc (0 where missing)
    uint32_t wmask[NP_MAX / 32];     // phenotype-valid bits
};

// The scratch: one copy per device, shared by every call on that device. In host code this
// name only stands for the array; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[sizeof(Scratch)];

__device__ __forceinline__ void block_sum(double &v, long long &n, double *sv, long long *sn)
{
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sv[w] = v;
        sn[w] = n;
    }
    __syncthreads();
    v = 0.0;
    n = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
        v += sv[i];
        n += sn[i];
    }
}

__device__ __forceinline__ double block_max(double v, double *sv)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sv[w] = v;
    __syncthreads();
    v = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v = fmax(v, sv[i]);
    return v;
}

// One block: resets the counters and maxima (every call starts from zero), writes the block
// descriptor, then the centred phenotype as the library's epi_set_traits does on the host:
// centred by the valid mean and scaled by the power of two that brings its largest magnitude
// into [0.5, 1) (exact, so F and F2 are unchanged, and a trait in units of 1e20 or 1e-20
// neither overflows nor underflows the single-precision squares).
__global__ void __launch_bounds__(1024) k_prep(Scratch *s, const float *__restrict__ phen, int nid, int Np, int Wp,
                                               int safe, BlockDesc bd)
{
    __shared__ double sv[32];
    __shared__ long long sn[32];
    const int tid = threadIdx.x;
    if (tid < 4) s->counters[tid] = 0ull;
    if (tid < 2) s->maxf[tid] = 0x007fffffu;  // order-encoded -inf
    if (tid == 0) s->block = bd;
    double sum = 0.0;
    long long n = 0;
    for (int k = tid; k < nid; k += blockDim.x) {
        const float y = phen[k];
        if (safe || y != -9.0f) {
            sum += (double)y;
            ++n;
        }
    }
    block_sum(sum, n, sv, sn);
    const double mu = n ? sum / (double)n : 0.0;
    double mx = 0.0;
    for (int k = tid; k < nid; k += blockDim.x) {
        const float y = phen[k];
        if (safe || y != -9.0f) mx = fmax(mx, fabs((double)y - mu));
    }
    const double maxabs = block_max(mx, sv);
    const double p2 = (maxabs > 0.0 && isfinite(maxabs)) ? ldexp(1.0, -(ilogb(maxabs) + 1)) : 1.0;
    double s2 = 0.0;
    long long dummy = 0;
    for (int k = tid; k < Np; k += blockDim.x) {
        const float y = k < nid ? phen[k] : -9.0f;
        const bool ok = k < nid && (safe || y != -9.0f);
        const float yc = ok ? (float)(((double)y - mu) * p2) : 0.0f;
        s->y[k] = yc;
        if (ok) s2 += (double)yc * (double)yc;
    }
    block_sum(s2, dummy, sv, sn);
    const double c = n ? s2 / (double)n : 0.0;
    if (tid == 0) s->qc = c;
    for (int k = tid; k < Np; k += blockDim.x) {
        const float y = k < nid ? phen[k] : -9.0f;
        const bool ok = k < nid && (safe || y != -9.0f);
        const double yc = s->y[k];
        s->q[k] = ok ? (float)(yc * yc - c) : 0.0f;
    }
    for (int w = tid; w < Wp; w += blockDim.x) {
        uint32_t bits = 0;
        for (int t = 0; t < 32; ++t) {
            const int k = 32 * w + t;
            if (k < nid && (safe || phen[k] != -9.0f)) bits |= 1u << t;
        }
        s->wmask[w] = bits;
    }
}

__global__ void k_finish(const Scratch *s, int64_t *nhits, float *maxf, int test_int)
{
    if (threadIdx.x != 0) return;
    *nhits = (int64_t)s->counters[0];
    if (maxf) {
        maxf[0] = ord2f(s->maxf[0]);
        maxf[1] = test_int ? ord2f(s->maxf[1]) : 0.0f;
    }
}

constexpr int MAX_DEVICES = 64;
static int g_sms[MAX_DEVICES];  // per device: SM count, 0 until the device's set-up ran

}  // namespace noalloc
}  // namespace epi

extern "C" epi_status epi_scan_block_noalloc(const int32_t *d_gpack, int32_t nid, int32_t nsnp, const float *d_phen,
                                             const epi_block *block, const epi_scan_opts *opts, epi_hit *d_hits,
                                             int64_t cap, int64_t *d_nhits, float *d_maxf, void *stream)
{
    using namespace epi;
    if (!d_gpack || !d_phen || !block || !opts || !d_nhits || cap < 0 || (cap > 0 && !d_hits) || nsnp < 1 || nid < 1)
        return EPI_E_INVALID;
    if (nid > EPI_NOALLOC_MAX_NID) return EPI_E_UNSUPPORTED;  // beyond the fixed scratch
    if ((opts->test != 'f' && opts->test != 'i') || (opts->safe != 0 && opts->safe != 1)) return EPI_E_INVALID;
    if (block->start1 < 0 || block->start2 < 0 || block->size1 < 0 || block->size2 < 0 ||
        (int64_t)block->start1 + block->size1 > nsnp || (int64_t)block->start2 + block->size2 > nsnp)
        return EPI_E_INVALID;
    // an error left pending by the caller's earlier work is theirs: report it, do not clear it
    if (cudaPeekAtLastError() != cudaSuccess) return EPI_E_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= noalloc::MAX_DEVICES) return EPI_E_NODEVICE;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t smem = sizeof(popc_raw::Smem) + 8;  // + per-CTA maxima of one trait

    // set-up, once per device with that device current: the device check, the SM count and
    // the kernel's shared-memory attribute
    if (noalloc::g_sms[dev] == 0) {
        int major = 0, sms = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
            return EPI_E_NODEVICE;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            return EPI_E_CUDA;
        if (cudaFuncSetAttribute(popc_raw::k_scan_popc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return EPI_E_CUDA;
        noalloc::g_sms[dev] = sms;
    }
    // The scratch array's device address. In host code g_scratch only stands for the array;
    // the address comes from the runtime, for the current device. It is looked up on every
    // call (a host-side table lookup once the module is loaded), so that a device reset
    // between calls, which reloads the module, cannot leave a stale address behind.
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, noalloc::g_scratch) != cudaSuccess || ptr == nullptr) return EPI_E_CUDA;
    noalloc::Scratch *scr = (noalloc::Scratch *)ptr;

    const int Wp = ((nid + 31) / 32 + 3) / 4 * 4;
    const int Np = 32 * Wp;
    BlockDesc bd;
    bd.start1 = block->start1;
    bd.size1 = block->size1;
    bd.start2 = block->start2;
    bd.size2 = block->size2;
    bd.tiles_i = (block->size1 + popc_raw::TI - 1) / popc_raw::TI;
    bd.tiles_j = (block->size2 + popc_raw::TJ - 1) / popc_raw::TJ;
    bd.tile_base = 0;
    const long long ntiles = (long long)bd.tiles_i * bd.tiles_j;

    ScanArgs a;
    memset(&a, 0, sizeof(a));
    a.gpack = d_gpack;
    a.npack = nid / 16;
    a.remain = nid % 16;
    a.nid = nid;
    a.nsnp = nsnp;
    a.Wp = Wp;
    a.Np = Np;
    a.y = scr->y;
    a.q = scr->q;
    a.wmask = scr->wmask;
    a.qc = &scr->qc;
    a.ntraits = 1;
    a.blocks = &scr->block;
    a.nblocks = 1;
    a.ntiles = ntiles;
    a.test_int = opts->test == 'i';
    a.safe = opts->safe;
    a.report_trait = 0;
    a.t1 = opts->t1;
    a.t2 = opts->t2;
    a.rows = reinterpret_cast<HitRow *>(d_hits);
    a.cap = cap;
    a.counters = scr->counters;
    a.maxf = &scr->maxf[0];
    a.maxf2 = &scr->maxf[1];

    noalloc::k_prep<<<1, 1024, 0, st>>>(scr, d_phen, nid, Np, Wp, opts->safe, bd);
    if (ntiles > 0) {
        const int grid = (int)(ntiles < noalloc::g_sms[dev] ? ntiles : noalloc::g_sms[dev]);
        popc_raw::k_scan_popc<true><<<grid, popc_raw::NT, smem, st>>>(a);
    }
    noalloc::k_finish<<<1, 32, 0, st>>>(scr, d_nhits, d_maxf, a.test_int);
    if (cudaGetLastError() != cudaSuccess) return EPI_E_CUDA;
    unsigned long long found = 0ull;
    if (cudaMemcpyAsync(&found, &scr->counters[0], sizeof(found), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return EPI_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return EPI_E_CUDA;
    // as epi_scan: more hits than `cap` is reported (the first `cap` rows are written, and
    // *d_nhits holds the total)
    return (int64_t)found > cap ? EPI_E_OVERFLOW : EPI_OK;
}
