// scan_popc.cu -- the plain form of the pair scan: the reference's per-individual method
// (src/EpiOpenCL.c:110-228: unpack two SNPs, count the 3x3 genotype cells, add the
// phenotype into its cell) redone for the B200's CUDA cores.
//
// Persistent kernel, one 512-thread CTA per SM, pulling (SNP-pair tile, trait) units from a
// queue over the tile schedule of the chromosome blocks (tile shapes: the table at the end of
// this file, chosen by the autotuner). The genotype bit-plane words of the tile's i-SNPs and
// j-SNPs (planes of g==0, g==1, g==2, g!=3 per 32 individuals)
// arrive by TMA, 64 individuals per stage, in a three-stage ring. Each SNP's two genotypes
// other than its most frequent one are its dense genotypes A and B. Per stage:
//   * expansion (all threads, double-buffered): for each i-SNP, U_A = [g_i==A]*y and
//     U_B = [g_i==B]*y floats in shared memory, two i-SNPs side by side, with the
//     phenotype-masked plane words of A, B and of the missing calls;
//   * cell counts of the dense 2x2 cells and of the individuals missing at j: AND + __popc of
//     32-bit plane words, 16-bit packed counters;
//   * cell sums S_{Ai,Aj}, S_{Ai,Bj}, S_{Bi,Aj}, S_{Bi,Bj}: each lane holds its own j-SNP's
//     plane words and adds the warp's broadcast U values into the cells its genotype bits
//     select (4 FP32 adds per pair and individual, predicated by the bits; the bit of the
//     lane's j-SNP is the same for two i-SNPs, so each predicated instruction is a packed
//     f32x2 add serving two pairs, rounded like two scalar adds);
//   * individuals missing at the j-SNP (per lane, sparse): their sums by the i genotype;
//   * individuals missing at the i-SNP (warp-uniform, sparse): their sums and counts by the
//     j genotype, and the sum of y^2 of individuals missing at both SNPs.
// The most frequent genotypes' row and column and the sum of squares come from per-(trait,
// SNP) FP64 marginals in the epilogue: S_{a,Mj} = R_a(i) - S_{a,Aj} - S_{a,Bj} - S_{a,3}
// (R_a(i) = sum of y over g_i = a), then S_{Mi,b} = C_b(j) - S_{Ai,b} - S_{Bi,b} - S_{3,b},
// likewise the counts, and Q = Qtot - QM_i - QM_j + QMM. Deriving the most frequent
// genotypes keeps the FP32 sums to the smaller cells. Each thread owns 8 whole pairs (the
// warp's 8 i-SNPs x the lane's j-SNP), so the reduction over individuals stays in registers.
// Epilogue: FP64 SSB/SSI/F/F2 per pair (src/EpiOpenCL.c:231-247, :452-486), warp-aggregated
// atomic hit append, per-trait maxima (warp-shuffle reductions).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "epi_internal.cuh"
#include "tc_ptx.cuh"

namespace epi {
namespace popc {

// A tile shape: WI x WJ warps, each warp PI i-SNPs x 32 j-SNPs (PI pairs per thread); the
// tile is TI = WI * PI i-SNPs by TJ = 32 * WJ j-SNPs. The autotuner picks one per device and
// workload from the table at the end of this file.
template <int WI_, int WJ_, int PI_>
struct Shape {
    static constexpr int WI = WI_, WJ = WJ_, PI = PI_;
    static constexpr int TI = WI * PI;        // i-SNPs per tile
    static constexpr int TJ = WJ * 32;        // j-SNPs per tile
    static constexpr int NT = WI * WJ * 32;   // threads
    static constexpr int KW = 2;              // 32-individual words per stage
    static constexpr int KI = 32 * KW;        // individuals per stage
    static constexpr int RS = 3;              // TMA ring depth
    static constexpr uint32_t STAGE_BYTES = (TI + TJ) * KW * 16;  // transaction bytes per stage
    static_assert(TI * KW <= NT - KI / 4 && TI <= 256 && TJ <= 256 && TI + TJ <= NT, "expansion roles");
    static_assert(PI % 2 == 0, "i-SNPs in pairs (packed FP32 adds)");

    struct Smem {
        uint4 raw_i[RS][TI][KW];  // TMA: plane words of the i-tile (row = SNP)
        uint4 raw_j[RS][TJ][KW];  // TMA: plane words of the j-tile
        float4 u[2][KI][TI / 2];  // (U_A, U_A', U_B, U_B') of i-SNPs 2p, 2p + 1 at individual k
        uint4 pm[2][KW][TI];      // (P_A & W, P_B & W, missing & W, W) of each i-SNP
        float y[2][KI];           // the stage's trait values (0 where invalid)
        float4 sps[PI][NT];       // per pair: sums over individuals missing at i by g_j: S_30..S_32, QMM
        uint2 spn[PI][NT];        // and counts: n_30 | n_31 << 16, n_32
        float2 spj[PI][NT];       // per pair: sums over individuals missing at j by g_i: S_{Ai,3}, S_{Bi,3}
        uint64_t full[RS];
        uint8_t maj[TI];          // most frequent genotype of each i-SNP
        uint8_t majj[TJ];         // and of each j-SNP
        long long unit;
        int never;                // always 0: the abort flag of the bounded waits
    };
};

// One pair's accumulators and the per-SNP values its statistics need, passed out of line.
struct PairIn {
    float S[4];    // S_{Ai,Aj}, S_{Ai,Bj}, S_{Bi,Aj}, S_{Bi,Bj}
    float SJ[2];   // S_{Ai,3}, S_{Bi,3}: individuals missing at j
    uint32_t C[3]; // n_{Ai,Aj} | n_{Ai,Bj} << 16, n_{Bi,Aj} | n_{Bi,Bj} << 16, n_{Ai,3} | n_{Bi,3} << 16
    float4 sp;     // individuals missing at i, by g_j: S_{3,0..2}, and QMM
    uint2 spn;     // n_{3,0} | n_{3,1} << 16, n_{3,2}
    int maj, majj, trait, si, sj, gi, gj, size2;
};

// FP64 statistics of one pair: the most frequent genotype's row from the marginals, then the
// reference's formulas (pair_stat); also writes the optional per-pair dump. Out of line, so the
// kernel's accumulators stay in registers.
__device__ __noinline__ PairStat eval_pair(const ScanArgs &a, const PairIn p)
{
    const int Ai = p.maj == 0 ? 1 : 0, Bi = p.maj == 2 ? 1 : 2, Mi = p.maj;
    const int Aj = p.majj == 0 ? 1 : 0, Bj = p.majj == 2 ? 1 : 2, Mj = p.majj;
    const size_t mi = (size_t)p.trait * a.nsnp + p.si, mj = (size_t)p.trait * a.nsnp + p.sj;
    int n[9];
    double S[9];
    // the dense 2 x 2 cells
    n[3 * Ai + Aj] = (int)(p.C[0] & 0xffffu);
    n[3 * Ai + Bj] = (int)(p.C[0] >> 16);
    n[3 * Bi + Aj] = (int)(p.C[1] & 0xffffu);
    n[3 * Bi + Bj] = (int)(p.C[1] >> 16);
    S[3 * Ai + Aj] = (double)p.S[0];
    S[3 * Ai + Bj] = (double)p.S[1];
    S[3 * Bi + Aj] = (double)p.S[2];
    S[3 * Bi + Bj] = (double)p.S[3];
    // the j-SNP's most frequent genotype, rows Ai and Bi: the i-SNP's marginal less the row's
    // other cells and its individuals missing at j
    n[3 * Ai + Mj] = a.pmN[3 * mi + Ai] - n[3 * Ai + Aj] - n[3 * Ai + Bj] - (int)(p.C[2] & 0xffffu);
    n[3 * Bi + Mj] = a.pmN[3 * mi + Bi] - n[3 * Bi + Aj] - n[3 * Bi + Bj] - (int)(p.C[2] >> 16);
    S[3 * Ai + Mj] = a.pmC[3 * mi + Ai] - S[3 * Ai + Aj] - S[3 * Ai + Bj] - (double)p.SJ[0];
    S[3 * Bi + Mj] = a.pmC[3 * mi + Bi] - S[3 * Bi + Aj] - S[3 * Bi + Bj] - (double)p.SJ[1];
    // the i-SNP's most frequent genotype, every column: the j-SNP's marginal less the column's
    // other cells and its individuals missing at i
    const int n3[3] = {(int)(p.spn.x & 0xffffu), (int)(p.spn.x >> 16), (int)p.spn.y};
    const double S3[3] = {(double)p.sp.x, (double)p.sp.y, (double)p.sp.z};
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        n[3 * Mi + b] = a.pmN[3 * mj + b] - n[3 * Ai + b] - n[3 * Bi + b] - n3[b];
        S[3 * Mi + b] = a.pmC[3 * mj + b] - S[3 * Ai + b] - S[3 * Bi + b] - S3[b];
    }
    // an empty cell's sum is 0: a derived sum of an empty cell holds only the rounding of the
    // FP32 sums it was formed from (so a pair without valid individuals keeps F = 0/0 = NaN)
#pragma unroll
    for (int c = 0; c < 9; ++c)
        if (n[c] == 0) S[c] = 0.0;
    const double Qv = a.ysq[p.trait] - a.pmQ[mi] - a.pmQ[mj] + (double)p.sp.w;
    const PairStat s = pair_stat(n, S, Qv, a.test_int != 0);
    if (p.trait == a.report_trait) {
        const size_t o = (size_t)p.gi * p.size2 + p.gj;
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

__device__ __forceinline__ bool bit(uint32_t w, int t) { return (w >> t) & 1u; }

template <class Sh>
__global__ void __launch_bounds__(Sh::NT, 1) k_scan_popc(ScanArgs a, const __grid_constant__ PopcMaps maps)
{
    constexpr int WI = Sh::WI, PI = Sh::PI, TI = Sh::TI, TJ = Sh::TJ, NT = Sh::NT, KW = Sh::KW, KI = Sh::KI;
    constexpr int RS = Sh::RS;
    using Smem = typename Sh::Smem;
    extern __shared__ uint8_t smem_raw[];
    // TMA destinations: 1024-byte aligned
    const uint32_t raw_s = tc::smem_u32(smem_raw);
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw + (((raw_s + 1023u) & ~1023u) - raw_s));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wi = warp % WI, wj = warp / WI;
    const int ib = wi * PI, jl = wj * 32 + lane;  // this thread's first i row, its j row
    const int nst = a.Wp / KW;
    const long long units = a.ntiles * (long long)a.ntraits;

    // maxima of F and F2 per trait: per CTA in shared memory (flushed once, at the end) up to
    // SMAX_TRAITS traits, else the global maxima directly
    const bool smax_local = a.ntraits <= SMAX_TRAITS;
    unsigned int *smax = reinterpret_cast<unsigned int *>(reinterpret_cast<uint8_t *>(&sm) + sizeof(Smem));
    if (smax_local)
        for (int w = tid; w < 2 * a.ntraits; w += NT) smax[w] = 0u;
    unsigned int *const mxf = smax_local ? smax : a.maxf;
    unsigned int *const mxf2 = smax_local ? smax + a.ntraits : a.maxf2;
    if (tid == 0) {
        for (int r = 0; r < RS; ++r) tc::mbar_init(&sm.full[r], 1);
        sm.never = 0;
        tc::fence_barrier_init();
    }
    __syncthreads();
    uint32_t par = 0u;  // parity of each ring slot's next phase (bit r), the same in every thread

    // every thread: wait for stage `st`'s words (bounded; a timeout is recorded, and the
    // control flow stays the same in every thread)
    auto wait_stage = [&](int st) {
        const int r = st % RS;
        if (!tc::mbar_wait(&sm.full[r], (par >> r) & 1u, &sm.never, a.wait_ns) && lane == 0 &&
            atomicCAS(&a.counters[2], 0ull, 1ull) == 0ull)
            a.counters[3] = 20ull;
        par ^= 1u << r;
    };

    for (;;) {
        if (tid == 0) sm.unit = (long long)atomicAdd(&a.counters[1], 1ull);
        __syncthreads();
        const long long u = sm.unit;
        __syncthreads();
        if (u >= units) break;
        const long long tile = u / a.ntraits;
        const int t = (int)(u % a.ntraits);
        const int blk = find_block(a.blocks, a.nblocks, tile);
        const BlockDesc bd = a.blocks[blk];
        const long long lt = tile - bd.tile_base;
        const int i0 = (int)(lt / bd.tiles_j) * TI, j0 = (int)(lt % bd.tiles_j) * TJ;
        // no pair with snp1 > snp2 in this tile (upper part of a diagonal block)
        if (bd.start1 + min(i0 + TI, bd.size1) - 1 <= bd.start2 + j0) continue;

        const float *yt = a.y + (size_t)t * a.Np;
        const uint32_t *wt = a.wmask + (size_t)t * a.Wp;
        if (tid < TI) sm.maj[tid] = i0 + tid < bd.size1 ? a.maj[bd.start1 + i0 + tid] : (uint8_t)0;
        else if (tid < TI + TJ)
            sm.majj[tid - TI] = j0 + tid - TI < bd.size2 ? a.maj[bd.start2 + j0 + tid - TI] : (uint8_t)0;
#pragma unroll
        for (int ii = 0; ii < PI; ++ii) {
            sm.sps[ii][tid] = make_float4(0.f, 0.f, 0.f, 0.f);
            sm.spn[ii][tid] = make_uint2(0u, 0u);
            sm.spj[ii][tid] = make_float2(0.f, 0.f);
        }
        auto issue = [&](int st) {  // thread 0: the TMA loads of stage st
            const int r = st % RS;
            tc::mbar_arrive_expect_tx(&sm.full[r], Sh::STAGE_BYTES);
            tc::tma_load_2d(&sm.raw_i[r][0][0], &maps.planes_i, 4 * KW * st, bd.start1 + i0, &sm.full[r]);
            tc::tma_load_2d(&sm.raw_j[r][0][0], &maps.planes_j, 4 * KW * st, bd.start2 + j0, &sm.full[r]);
        };
        if (tid == 0)
            for (int st = 0; st < min(RS, nst); ++st) issue(st);
        __syncthreads();  // maj

        // expansion of stage st into buffer b: work item -> (pair of i-SNPs, 4 individuals),
        // consecutive threads on consecutive i-SNP pairs (contiguous stores, the same trait
        // words in a warp)
        auto expand = [&](int st, int b) {
            const int r = st % RS;
            for (int it = tid; it < 8 * TI; it += NT) {
                const int p = it % (TI / 2), part = it / (TI / 2), w = part >> 3, k4 = 4 * (part & 7);
                const uint4 P0 = sm.raw_i[r][2 * p][w], P1 = sm.raw_i[r][2 * p + 1][w];
                const int m0 = sm.maj[2 * p], m1 = sm.maj[2 * p + 1];
                const uint32_t PA0 = m0 == 0 ? P0.y : P0.x, PB0 = m0 == 2 ? P0.y : P0.z;
                const uint32_t PA1 = m1 == 0 ? P1.y : P1.x, PB1 = m1 == 2 ? P1.y : P1.z;
                const float4 y4 = __ldg(reinterpret_cast<const float4 *>(yt + KI * st + 32 * w + k4));
                const float yv[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int k = k4 + e;
                    sm.u[b][32 * w + k][p] = make_float4(bit(PA0, k) ? yv[e] : 0.f, bit(PA1, k) ? yv[e] : 0.f,
                                                         bit(PB0, k) ? yv[e] : 0.f, bit(PB1, k) ? yv[e] : 0.f);
                }
            }
            if (tid < TI * KW) {
                const int i = tid % TI, w = tid / TI;
                const uint4 P = sm.raw_i[r][i][w];
                const int mj = sm.maj[i];
                const uint32_t W = __ldg(wt + KW * st + w);
                const uint32_t PA = mj == 0 ? P.y : P.x, PB = mj == 2 ? P.y : P.z;
                sm.pm[b][w][i] = make_uint4(PA & W, PB & W, ~P.w & W, W);
            } else if (tid >= NT - KI / 4) {
                const int q = tid - (NT - KI / 4);
                reinterpret_cast<float4 *>(sm.y[b])[q] = __ldg(reinterpret_cast<const float4 *>(yt + KI * st) + q);
            }
        };

        wait_stage(0);
        expand(0, 0);
        __syncthreads();

        float2 S[PI / 2][4];  // the cell sums of i-SNPs ib + 2p (x) and ib + 2p + 1 (y)
        uint32_t C[PI][3];
#pragma unroll
        for (int ii = 0; ii < PI; ++ii) {
            if (ii % 2 == 0)
#pragma unroll
                for (int c = 0; c < 4; ++c) S[ii / 2][c] = make_float2(0.f, 0.f);
            C[ii][0] = C[ii][1] = C[ii][2] = 0u;
        }
        const int mjj = sm.majj[jl];  // this lane's j-SNP: its dense genotypes' planes

        for (int st = 0; st < nst; ++st) {
            const int b = st & 1, r = st % RS;
            if (st + 1 < nst) {
                wait_stage(st + 1);
                expand(st + 1, b ^ 1);
            }
#pragma unroll 1
            for (int w = 0; w < KW; ++w) {
                const uint4 pj = sm.raw_j[r][jl][w];
                const uint32_t PAj = mjj == 0 ? pj.y : pj.x, PBj = mjj == 2 ? pj.y : pj.z, Mj = ~pj.w;
                // counts and the sparse individuals missing at i
#pragma unroll
                for (int ii = 0; ii < PI; ++ii) {
                    const uint4 pm = sm.pm[b][w][ib + ii];
                    C[ii][0] += __popc(pm.x & PAj) + (__popc(pm.x & PBj) << 16);
                    C[ii][1] += __popc(pm.y & PAj) + (__popc(pm.y & PBj) << 16);
                    C[ii][2] += __popc(pm.x & Mj) + (__popc(pm.y & Mj) << 16);
                    uint32_t m = pm.z;  // the same in every lane of the warp
                    while (m) {
                        const int k = __ffs(m) - 1;
                        m &= m - 1u;
                        const float yv = sm.y[b][32 * w + k];
                        const bool g0 = bit(pj.x, k), g1 = bit(pj.y, k), g2 = bit(pj.z, k);
                        float4 acc = sm.sps[ii][tid];
                        uint2 nn = sm.spn[ii][tid];
                        acc.x += g0 ? yv : 0.f;
                        acc.y += g1 ? yv : 0.f;
                        acc.z += g2 ? yv : 0.f;
                        acc.w += (g0 || g1 || g2) ? 0.f : yv * yv;
                        nn.x += (g0 ? 1u : 0u) + (g1 ? 0x10000u : 0u);
                        nn.y += g2 ? 1u : 0u;
                        sm.sps[ii][tid] = acc;
                        sm.spn[ii][tid] = nn;
                    }
                }
                // individuals missing at this lane's j-SNP (and phenotype-valid): their sums by
                // the i genotype (per lane; rare)
                uint32_t mj = Mj & sm.pm[b][w][ib].w;
                while (mj) {
                    const int k = __ffs(mj) - 1;
                    mj &= mj - 1u;
                    const float yv = sm.y[b][32 * w + k];
#pragma unroll
                    for (int ii = 0; ii < PI; ++ii) {
                        const uint2 pab = *reinterpret_cast<const uint2 *>(&sm.pm[b][w][ib + ii]);
                        float2 acc = sm.spj[ii][tid];
                        acc.x += bit(pab.x, k) ? yv : 0.f;
                        acc.y += bit(pab.y, k) ? yv : 0.f;
                        sm.spj[ii][tid] = acc;
                    }
                }
                // sums: this lane's j genotype bit of individual k selects the cells the U
                // values go to; one packed FP32 add serves two i-SNPs (the same j bit)
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const bool fA = bit(PAj, k), fB = bit(PBj, k);
#pragma unroll
                    for (int q = 0; q < PI / 2; ++q) {
                        const float4 uu = sm.u[b][32 * w + k][ib / 2 + q];
                        const float2 ua = make_float2(uu.x, uu.y), ub = make_float2(uu.z, uu.w);
                        if (fA) S[q][0] = __fadd2_rn(S[q][0], ua);
                        if (fB) S[q][1] = __fadd2_rn(S[q][1], ua);
                        if (fA) S[q][2] = __fadd2_rn(S[q][2], ub);
                        if (fB) S[q][3] = __fadd2_rn(S[q][3], ub);
                    }
                }
            }
            __syncthreads();  // stage st consumed (its ring slot and U buffer), st + 1 expanded
            if (tid == 0 && st + RS < nst) issue(st + RS);
        }

        // epilogue
        const bool report = a.report_trait < 0 || a.report_trait == t;
        // unrolled: S and C are indexed by constants only, so they stay in registers
#pragma unroll
        for (int ii = 0; ii < PI; ++ii) {
            const int gi = i0 + ib + ii, gj = j0 + jl;
            const bool valid = gi < bd.size1 && gj < bd.size2 && (bd.start1 + gi > bd.start2 + gj);
            PairStat s;
            s.nfac = s.d1 = s.d2 = 0;
            s.F = s.F2 = 0.0;
            if (valid) {
                PairIn p;
#pragma unroll
                for (int c = 0; c < 4; ++c) p.S[c] = ii % 2 ? S[ii / 2][c].y : S[ii / 2][c].x;
                const float2 sj = sm.spj[ii][tid];
                p.SJ[0] = sj.x;
                p.SJ[1] = sj.y;
#pragma unroll
                for (int c = 0; c < 3; ++c) p.C[c] = C[ii][c];
                p.sp = sm.sps[ii][tid];
                p.spn = sm.spn[ii][tid];
                p.maj = sm.maj[ib + ii];
                p.majj = sm.majj[jl];
                p.trait = t;
                p.si = bd.start1 + gi;
                p.sj = bd.start2 + gj;
                p.gi = gi;
                p.gj = gj;
                p.size2 = bd.size2;
                s = eval_pair(a, p);
            }
            const bool hit = valid && report && is_hit(a, s);
            emit_hit(a, hit, bd.start1 + gi, bd.start2 + gj, s, t, blk);
            fold_max(&mxf[t], valid, s.F);
            if (a.test_int) fold_max(&mxf2[t], valid, s.F2);
        }
    }
    __syncthreads();
    if (smax_local)
        for (int w = tid; w < 2 * a.ntraits; w += NT)
            if (smax[w]) atomicMax(w < a.ntraits ? &a.maxf[w] : &a.maxf2[w - a.ntraits], smax[w]);
}

}  // namespace popc

// The tile shapes the autotuner chooses among:
//   0  64 x 64 tile, 8 pairs per thread (8 x 2 warps): fewest shared-memory loads per add
//   1  64 x 32 tile, 4 pairs per thread (16 x 1 warps): fewest registers, most warps per i-SNP
//   2  32 x 128 tile, 8 pairs per thread (4 x 4 warps): the i-side expansion shared by more lanes
using Shape0 = popc::Shape<8, 2, 8>;
using Shape1 = popc::Shape<16, 1, 4>;
using Shape2 = popc::Shape<4, 4, 8>;
constexpr int POPC_SHAPES = 3;

int popc_shapes() { return POPC_SHAPES; }

// Tile size (i x j SNPs) and a description of shape v.
void popc_shape(int v, int *ti, int *tj, const char **desc)
{
    static const char *names[POPC_SHAPES] = {"64x64 tile, 8 pairs/thread, 8x2 warps",
                                             "64x32 tile, 4 pairs/thread, 16x1 warps",
                                             "32x128 tile, 8 pairs/thread, 4x4 warps"};
    const int tis[POPC_SHAPES] = {Shape0::TI, Shape1::TI, Shape2::TI};
    const int tjs[POPC_SHAPES] = {Shape0::TJ, Shape1::TJ, Shape2::TJ};
    *ti = tis[v];
    *tj = tjs[v];
    if (desc) *desc = names[v];
}

// The plane words [nsnp][Wp] (uint4) as a 2-D uint32 tensor [nsnp][4 Wp]; one box = the words
// of one stage (KW x 4 uint32 = 32 bytes) of `rows` SNPs; rows past the last SNP read as 0.
static cudaError_t encode_planes(CUtensorMap *m, const uint4 *planes, int nsnp, int Wp, int rows)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t dims[2] = {4 * (cuuint64_t)Wp, (cuuint64_t)nsnp};
    const cuuint64_t strides[1] = {16 * (cuuint64_t)Wp};
    const cuuint32_t box[2] = {4 * Shape0::KW, (cuuint32_t)rows};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint4 *>(planes), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t popc_encode_planes(int v, PopcMaps *maps, const uint4 *planes, int nsnp, int Wp)
{
    int ti = 0, tj = 0;
    popc_shape(v, &ti, &tj, nullptr);
    cudaError_t e = encode_planes(&maps->planes_i, planes, nsnp, Wp, ti);
    if (e == cudaSuccess) e = encode_planes(&maps->planes_j, planes, nsnp, Wp, tj);
    return e;
}

template <class C>
static size_t shape_smem(int ntraits)
{
    return sizeof(typename C::Smem) + 1024 + smax_bytes(ntraits);
}

template <class C>
static cudaError_t prepare(void)
{
    return cudaFuncSetAttribute(popc::k_scan_popc<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)shape_smem<C>(SMAX_TRAITS));
}

template <class C>
static cudaError_t enqueue(const ScanArgs &a, const PopcMaps &maps, int grid, cudaStream_t stream)
{
    popc::k_scan_popc<C><<<grid, C::NT, shape_smem<C>(a.ntraits), stream>>>(a, maps);
    return cudaGetLastError();
}

// Before any stream capture: the shape's kernel attribute (the largest shared-memory size any
// trait count asks for).
cudaError_t popc_prepare(int v)
{
    switch (v) {
    case 0: return prepare<Shape0>();
    case 1: return prepare<Shape1>();
    case 2: return prepare<Shape2>();
    }
    return cudaErrorInvalidValue;
}

// The launch itself (a stream operation only, so it can be captured into a CUDA graph).
cudaError_t popc_enqueue(int v, const ScanArgs &a, const PopcMaps &maps, int grid, cudaStream_t stream)
{
    switch (v) {
    case 0: return enqueue<Shape0>(a, maps, grid, stream);
    case 1: return enqueue<Shape1>(a, maps, grid, stream);
    case 2: return enqueue<Shape2>(a, maps, grid, stream);
    }
    return cudaErrorInvalidValue;
}

}  // namespace epi
