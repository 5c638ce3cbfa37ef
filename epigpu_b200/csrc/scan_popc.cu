// scan_popc.cu -- the plain form of the pair scan: the reference's per-individual method
// (src/EpiOpenCL.c:110-228: unpack two SNPs, count the 3x3 genotype cells, add the
// phenotype into its cell) redone for the B200's CUDA cores.
//
// Persistent kernel, one 512-thread CTA per SM, pulling 64 x 32 SNP-pair tiles from a
// queue over the triangular schedule of chromosome blocks. Per tile and trait it walks the
// individuals in stages of 64:
//   * stage expansion: the i-tile's bit-planes become U_a = [g_i==a]*y and U_V = [g_i valid]
//     as floats in shared memory (read by the whole warp: broadcast loads);
//   * cell counts: AND + __popc of 32-bit plane words (phenotype mask folded into the
//     i side), 16-bit packed counters;
//   * cell sums: each lane turns its own j-SNP's plane bits into F_b = [g_j==b] and
//     F_Q = [g_j valid]*q in registers, then S_ab += U_a*F_b (9 FP32 FMAs per pair and
//     individual) and Q += U_V*F_Q (sum of y^2 over valid individuals, q = y^2 - mean y^2).
// Each thread owns 4 whole pairs (the warp's four i-SNPs x the lane's j-SNP): no
// cross-lane reduction; ~100 registers so 16 warps per SM hide shared-memory latency.
// Epilogue: FP64 SSB/SSI/F/F2 per pair, warp-aggregated atomic hit append, per-trait max F.
#include "epi_internal.cuh"

namespace epi {
namespace popc {

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

__global__ void __launch_bounds__(NT, 1) k_scan_popc(ScanArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nstages = a.Wp / KW;

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
                    if (gi < bd.size1) P = a.planes[(size_t)(bd.start1 + gi) * a.Wp + w0 + (part >> 2)];
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
                    if (gi < bd.size1) P = a.planes[(size_t)(bd.start1 + gi) * a.Wp + w0 + w];
                    const uint32_t W = wt[w0 + w];
                    sm.pi[w][i] = make_uint4(P.x & W, P.y & W, P.z & W, 0u);
                } else if (tid < KW * TI + KW * TJ) {
                    const int idx = tid - KW * TI, w = idx / TJ, j = idx % TJ, gj = j0 + j;
                    uint4 P = make_uint4(0, 0, 0, 0);
                    if (gj < bd.size2) P = a.planes[(size_t)(bd.start2 + gj) * a.Wp + w0 + w];
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
                emit_hit(a, hit, bd.start1 + gi, bd.start2 + gj, s, t, b);
                fold_max(&a.maxf[t], valid, s.F);
                if (a.test_int) fold_max(&a.maxf2[t], valid, s.F2);
            }
        }
    }
}

}  // namespace popc

// Tile shape of this form (used by the host to build the tile schedule).
int popc_tile_i() { return popc::TI; }
int popc_tile_j() { return popc::TJ; }
int popc_words_multiple() { return popc::KW; }

cudaError_t launch_popc(const ScanArgs &a, int grid, cudaStream_t stream)
{
    const size_t smem = sizeof(popc::Smem);
    cudaError_t e = cudaFuncSetAttribute(popc::k_scan_popc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    popc::k_scan_popc<<<grid, popc::NT, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace epi
