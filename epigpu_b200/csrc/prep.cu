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
// qm[t][s] = sum of qd[t][k] and, when qr is given, rm[t][s] = sum of qr[t][k]
__global__ void k_qmiss(const uint32_t *__restrict__ missbits, int nsnp, int Wp, const uint32_t *__restrict__ wmask,
                        const double *__restrict__ qd, const double *__restrict__ qr, int Np, int ntraits,
                        double *__restrict__ qm, double *__restrict__ rm)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nsnp * ntraits) return;
    const int t = (int)(gid / nsnp), s = (int)(gid % nsnp);
    double x = 0.0, r = 0.0;
    const uint32_t *mb = missbits + (size_t)s * Wp;
    for (int w = 0; w < Wp; ++w) {
        uint32_t bits = mb[w] & wmask[(size_t)t * Wp + w];
        while (bits) {
            const size_t k = (size_t)t * Np + 32 * w + __ffs(bits) - 1;
            x += qd[k];
            if (qr) r += qr[k];
            bits &= bits - 1;
        }
    }
    qm[gid] = x;
    if (rm) rm[gid] = r;
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
                        const double *qr, int Np, int ntraits, double *qm, double *rm, cudaStream_t stream)
{
    const long long total = (long long)nsnp * ntraits;
    const int nt = 256;
    k_qmiss<<<(unsigned)((total + nt - 1) / nt), nt, 0, stream>>>(missbits, nsnp, Wp, wmask, qd, qr, Np, ntraits, qm,
                                                                     rm);
    return cudaGetLastError();
}

}  // namespace epi
