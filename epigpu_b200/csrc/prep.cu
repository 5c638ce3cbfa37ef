// prep.cu -- device-side genotype preparation.
//
// Turns the reference's packed rows (src/readplink.c:1066-1102: 16 codes per int32, first
// individual in bits 31:30, tail word right-aligned with `remain` codes) into
//   planes  uint4 [nsnp][Wp]: bits of [g==0], [g==1], [g==2], [g!=3] per 32 individuals
//   codes   uint32 [nsnp][Wc]: 2-bit codes, LSB first, padding individuals coded 3
// The decoding is the kernel's own (EpiOpenCL.c:116-228), done once per load instead of
// once per pair.
#include <cstdint>
#include <cuda_runtime.h>

namespace epi {

__device__ __forceinline__ uint32_t ref_code(const int32_t *row, int k, int nid, int npack, int remain)
{
    if (k >= nid) return 3u;
    if (k < 16 * npack) return ((uint32_t)row[k >> 4] >> (30 - 2 * (k & 15))) & 3u;
    const int t = k - 16 * npack;
    return ((uint32_t)row[npack] >> (2 * (remain - 1 - t))) & 3u;
}

// One thread per (SNP, 32-individual word). Also writes the tensor form's one-hot code
// bytes (1 << g, 0 when missing or padding), its genotype-indicator rows h3 (row 3s + a holds
// the byte [g == a] per individual) and the missing-genotype bits.
__global__ void k_unpack(const int32_t *__restrict__ raw, int nsnp, int nid, int npack, int remain,
                         int npack1, uint4 *__restrict__ planes, int Wp, uint32_t *__restrict__ codes, int Wc,
                         uint8_t *__restrict__ hcodes, uint8_t *__restrict__ h3, uint32_t *__restrict__ missbits)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)nsnp * Wp;
    if (gid >= total) return;
    const int s = (int)(gid / Wp), w = (int)(gid % Wp);
    const int32_t *row = raw + (size_t)s * npack1;
    uint32_t p0 = 0, p1 = 0, p2 = 0, c0 = 0, c1 = 0, miss = 0;
    uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int t = 0; t < 32; ++t) {
        const int k = 32 * w + t;
        const uint32_t c = ref_code(row, k, nid, npack, remain);
        p0 |= (uint32_t)(c == 0u) << t;
        p1 |= (uint32_t)(c == 1u) << t;
        p2 |= (uint32_t)(c == 2u) << t;
        miss |= (uint32_t)(c == 3u && k < nid) << t;
        h[t >> 2] |= (c < 3u ? (1u << c) : 0u) << (8 * (t & 3));
        if (t < 16) c0 |= c << (2 * t);
        else c1 |= c << (2 * (t - 16));
    }
    planes[(size_t)s * Wp + w] = make_uint4(p0, p1, p2, p0 | p1 | p2);
    if (hcodes != nullptr) {
        uint4 *dst = reinterpret_cast<uint4 *>(hcodes + ((size_t)s * Wp + w) * 32);
        dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
        dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
    if (h3 != nullptr) {
        const size_t Np = (size_t)Wp * 32;
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            uint32_t e[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) e[q] = (h[q] >> g) & 0x01010101u;
            uint4 *dst = reinterpret_cast<uint4 *>(h3 + (3 * (size_t)s + g) * Np + (size_t)w * 32);
            dst[0] = make_uint4(e[0], e[1], e[2], e[3]);
            dst[1] = make_uint4(e[4], e[5], e[6], e[7]);
        }
    }
    if (missbits != nullptr) missbits[(size_t)s * Wp + w] = miss;
    if (codes != nullptr) {
        if (2 * w < Wc) codes[(size_t)s * Wc + 2 * w] = c0;
        if (2 * w + 1 < Wc) codes[(size_t)s * Wc + 2 * w + 1] = c1;
    }
}

// Per trait t and SNP s, over the individuals missing at s (and phenotype-valid for t):
// qm[t][s] = sum of qd[t][k], rm[t][s] = sum of qr[t][k] and nm[t][s] = their number
__global__ void k_qmiss(const uint32_t *__restrict__ missbits, int nsnp, int Wp, const uint32_t *__restrict__ wmask,
                        const double *__restrict__ qd, const double *__restrict__ qr, int Np, int ntraits,
                        double *__restrict__ qm, double *__restrict__ rm, double *__restrict__ nm)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nsnp * ntraits) return;
    const int t = (int)(gid / nsnp), s = (int)(gid % nsnp);
    double x = 0.0, r = 0.0;
    int cnt = 0;
    const uint32_t *mb = missbits + (size_t)s * Wp;
    for (int w = 0; w < Wp; ++w) {
        uint32_t bits = mb[w] & wmask[(size_t)t * Wp + w];
        cnt += __popc(bits);
        while (bits) {
            const size_t k = (size_t)t * Np + 32 * w + __ffs(bits) - 1;
            x += qd[k];
            r += qr[k];
            bits &= bits - 1;
        }
    }
    qm[gid] = x;
    rm[gid] = r;
    nm[gid] = (double)cnt;
}

// The streamed-B variant's expanded B rows: for trait t, CTA half h, SNP s and local column
// type q = 2b + r (genotype b, digit row 2h + r of the trait: w, d0 for h = 0, d1, d2 for h = 1)
// row ((t 2 + h) nsnp + s) 6 + q holds [g_s(k) == b] * digit(k) for every individual k -- the
// rows the tensor form's producers otherwise build in shared memory. One thread per 16
// individuals of (t, h, s).
__global__ void k_expand(const uint8_t *__restrict__ hcodes, const int8_t *__restrict__ ydig, int nsnp, int Np,
                         int ntraits, int8_t *__restrict__ x)
{
    const int nc = Np / 16;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)ntraits * 2 * nsnp * nc) return;
    const int c = (int)(gid % nc);
    const long long rest = gid / nc;
    const int s = (int)(rest % nsnp);
    const int h = (int)((rest / nsnp) % 2), t = (int)(rest / nsnp / 2);
    const uint4 hc = reinterpret_cast<const uint4 *>(hcodes + (size_t)s * Np)[c];
    const uint4 d0 = reinterpret_cast<const uint4 *>(ydig + ((size_t)t * 4 + 2 * h) * Np)[c];
    const uint4 d1 = reinterpret_cast<const uint4 *>(ydig + ((size_t)t * 4 + 2 * h + 1) * Np)[c];
    uint4 *out = reinterpret_cast<uint4 *>(x + (((size_t)t * 2 + h) * nsnp + s) * 6 * (size_t)Np) + c;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        uint4 m;
        m.x = ((hc.x >> b) & 0x01010101u) * 0xFFu;
        m.y = ((hc.y >> b) & 0x01010101u) * 0xFFu;
        m.z = ((hc.z >> b) & 0x01010101u) * 0xFFu;
        m.w = ((hc.w >> b) & 0x01010101u) * 0xFFu;
        out[(size_t)(2 * b) * nc] = make_uint4(m.x & d0.x, m.y & d0.y, m.z & d0.z, m.w & d0.w);
        out[(size_t)(2 * b + 1) * nc] = make_uint4(m.x & d1.x, m.y & d1.y, m.z & d1.z, m.w & d1.w);
    }
}

// Per SNP the most frequent genotype (ties to the lower code), one warp per SNP: the plain
// form derives that genotype's row of the 3x3 table from the SNP's marginals.
__global__ void k_major(const uint4 *__restrict__ planes, int nsnp, int Wp, uint8_t *__restrict__ maj)
{
    const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= nsnp) return;
    int c0 = 0, c1 = 0, c2 = 0;
    for (int w = lane; w < Wp; w += 32) {
        const uint4 P = planes[(size_t)s * Wp + w];
        c0 += __popc(P.x);
        c1 += __popc(P.y);
        c2 += __popc(P.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(0xffffffffu, c0, o);
        c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        c2 += __shfl_xor_sync(0xffffffffu, c2, o);
    }
    if (lane == 0) maj[s] = (uint8_t)((c0 >= c1 && c0 >= c2) ? 0 : (c1 >= c2 ? 1 : 2));
}

// Plain-form marginals, one warp per (trait t, SNP s), lane = individual within each 32-word:
// pmC[t][s][b] = sum of y over g_s = b, pmN[t][s][b] = number of phenotype-valid individuals
// with g_s = b, pmQ[t][s] = sum of y^2 over the valid individuals missing at s. FP64 per lane,
// then a warp-shuffle reduction.
__global__ void k_marg(const uint4 *__restrict__ planes, int nsnp, int Wp, const float *__restrict__ y,
                       const uint32_t *__restrict__ wmask, int Np, int ntraits, double *__restrict__ pmC,
                       int32_t *__restrict__ pmN, double *__restrict__ pmQ)
{
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= (long long)nsnp * ntraits) return;
    const int t = (int)(gw / nsnp), s = (int)(gw % nsnp);
    double c0 = 0.0, c1 = 0.0, c2 = 0.0, q = 0.0;
    int n0 = 0, n1 = 0, n2 = 0;
    const float *yt = y + (size_t)t * Np;
    const uint32_t *wt = wmask + (size_t)t * Wp;
    for (int w = 0; w < Wp; ++w) {
        const uint4 P = planes[(size_t)s * Wp + w];
        const uint32_t W = wt[w];
        const double yv = (double)yt[32 * w + lane];
        const int ok = (W >> lane) & 1u;
        if ((P.x >> lane) & 1u) {
            c0 += yv;
            n0 += ok;
        } else if ((P.y >> lane) & 1u) {
            c1 += yv;
            n1 += ok;
        } else if ((P.z >> lane) & 1u) {
            c2 += yv;
            n2 += ok;
        } else if (ok) {
            q += yv * yv;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(0xffffffffu, c0, o);
        c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        c2 += __shfl_xor_sync(0xffffffffu, c2, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
        n0 += __shfl_xor_sync(0xffffffffu, n0, o);
        n1 += __shfl_xor_sync(0xffffffffu, n1, o);
        n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    }
    if (lane == 0) {
        const size_t o = (size_t)gw;
        pmC[3 * o] = c0;
        pmC[3 * o + 1] = c1;
        pmC[3 * o + 2] = c2;
        pmN[3 * o] = n0;
        pmN[3 * o + 1] = n1;
        pmN[3 * o + 2] = n2;
        pmQ[o] = q;
    }
}

cudaError_t launch_major(const uint4 *planes, int nsnp, int Wp, uint8_t *maj, cudaStream_t stream)
{
    const long long threads = 32LL * nsnp;
    k_major<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(planes, nsnp, Wp, maj);
    return cudaGetLastError();
}

cudaError_t launch_marg(const uint4 *planes, int nsnp, int Wp, const float *y, const uint32_t *wmask, int Np,
                        int ntraits, double *pmC, int32_t *pmN, double *pmQ, cudaStream_t stream)
{
    const long long threads = 32LL * nsnp * ntraits;
    k_marg<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(planes, nsnp, Wp, y, wmask, Np, ntraits, pmC, pmN,
                                                                 pmQ);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const int32_t *raw, int nsnp, int nid, int npack, int remain, uint4 *planes, int Wp,
                          uint32_t *codes, int Wc, uint8_t *hcodes, uint8_t *h3, uint32_t *missbits,
                          cudaStream_t stream)
{
    const int npack1 = remain ? npack + 1 : npack;
    const long long total = (long long)nsnp * Wp;
    const int nt = 256;
    const long long nb = (total + nt - 1) / nt;
    k_unpack<<<(unsigned)nb, nt, 0, stream>>>(raw, nsnp, nid, npack, remain, npack1, planes, Wp, codes, Wc, hcodes,
                                              h3, missbits);
    return cudaGetLastError();
}

cudaError_t launch_qmiss(const uint32_t *missbits, int nsnp, int Wp, const uint32_t *wmask, const double *qd,
                        const double *qr, int Np, int ntraits, double *qm, double *rm, double *nm,
                        cudaStream_t stream)
{
    const long long total = (long long)nsnp * ntraits;
    const int nt = 256;
    k_qmiss<<<(unsigned)((total + nt - 1) / nt), nt, 0, stream>>>(missbits, nsnp, Wp, wmask, qd, qr, Np, ntraits, qm,
                                                                     rm, nm);
    return cudaGetLastError();
}

cudaError_t launch_expand(const uint8_t *hcodes, const int8_t *ydig, int nsnp, int Np, int ntraits, int8_t *x,
                          cudaStream_t stream)
{
    const long long total = (long long)ntraits * 2 * nsnp * (Np / 16);
    const int nt = 256;
    k_expand<<<(unsigned)((total + nt - 1) / nt), nt, 0, stream>>>(hcodes, ydig, nsnp, Np, ntraits, x);
    return cudaGetLastError();
}

}  // namespace epi
