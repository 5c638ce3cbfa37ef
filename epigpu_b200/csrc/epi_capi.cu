// epi_capi.cu -- the C ABI of libepigpu.so (include/epigpu.h).
//
// Host side of the scan: device selection, genotype and trait upload, the tile schedule
// over chromosome blocks, kernel dispatch (plain popcount form / tcgen05 tensor form),
// hit readback and ordering. It replaces the OpenCL host code of perform_scan
// (src/EpiOpenCL.c:1383-1627); the results file itself is written by the C host
// (epigpu_b200/host/scan_driver.c).
#include "epigpu.h"
#include "epi_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

namespace epi {
cudaError_t launch_unpack(const int32_t *raw, int nsnp, int nid, int npack, int remain, uint4 *planes, int Wp,
                          uint32_t *codes, int Wc, uint8_t *hcodes, uint8_t *h3, uint32_t *missbits,
                          cudaStream_t stream);
cudaError_t launch_qmiss(const uint32_t *missbits, int nsnp, int Wp, const uint32_t *wmask, const double *qd,
                        const double *qr, int Np, int ntraits, double *qm, double *rm, double *nm,
                        cudaStream_t stream);
cudaError_t launch_major(const uint4 *planes, int nsnp, int Wp, uint8_t *maj, cudaStream_t stream);
cudaError_t launch_marg(const uint4 *planes, int nsnp, int Wp, const float *y, const uint32_t *wmask, int Np,
                        int ntraits, double *pmC, int32_t *pmN, double *pmQ, cudaStream_t stream);
// plain form (scan_popc.cu)
int popc_shapes();
void popc_shape(int v, int *ti, int *tj, const char **desc);
cudaError_t popc_prepare(int v);
cudaError_t popc_enqueue(int v, const ScanArgs &a, const PopcMaps &maps, int grid, cudaStream_t stream);
cudaError_t popc_encode_planes(int v, PopcMaps *maps, const uint4 *planes, int nsnp, int Wp);
// tensor form (scan_mma.cu)
bool mma_available();
int mma_tile_i();
int mma_tile_j();
int mma_min_nid();
int mma_max_nid();
int mma_shapes();
void mma_shape(int v, const char **desc);
cudaError_t mma_prepare(int v, int ntraits, int grid_request, int *grid);
cudaError_t mma_enqueue(int v, const ScanArgs &a, const MmaMaps &maps, int grid, cudaStream_t stream);
cudaError_t mma_encode_genotypes(MmaMaps *maps, const uint8_t *hcodes, const uint8_t *h3, int nsnp, int Np);
cudaError_t mma_encode_traits(MmaMaps *maps, const int8_t *ydig, int ntraits, int Np);
cudaError_t mma_encode_x(MmaMaps *maps, const int8_t *x, int nsnp, int Np, int ntraits);
bool mma_needs_x(int v);
cudaError_t launch_expand(const uint8_t *hcodes, const int8_t *ydig, int nsnp, int Np, int ntraits, int8_t *x,
                          cudaStream_t stream);
// Start of a scan: counters (hits, tile queue, error flag and site) to zero, the per-trait
// maxima of F and F2 to the order-encoded -inf.
__global__ void k_scan_init(unsigned long long *counters, unsigned int *maxf, int n)
{
    if (threadIdx.x < 4) counters[threadIdx.x] = 0ull;
    for (int i = threadIdx.x; i < n; i += blockDim.x) maxf[i] = 0x007fffffu;
}
}  // namespace epi

using epi::BlockDesc;
using epi::DevHit;

struct epi_ctx {
    int device = -1;
    int sm_count = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // genotypes
    int nid = 0, nsnp = 0, npack = 0, remain = 0;
    int Wp = 0, Wc = 0, Np = 0;
    int32_t *d_raw = nullptr;
    size_t raw_cap = 0;
    uint4 *d_planes = nullptr;
    uint8_t *d_hcodes = nullptr, *d_h3 = nullptr;
    uint32_t *d_missbits = nullptr;
    uint8_t *d_maj = nullptr;
    size_t planes_cap = 0, hcodes_cap = 0, h3_cap = 0, missbits_cap = 0, maj_cap = 0;
    epi::PopcMaps pmaps;
    // traits
    int ntraits = 0, traits_nid = 0;
    float *d_y = nullptr, *d_q = nullptr;
    uint32_t *d_wmask = nullptr;
    double *d_qc = nullptr, *d_yscale = nullptr, *d_qd = nullptr, *d_qtot = nullptr, *d_qm = nullptr;
    int8_t *d_ydig = nullptr;
    size_t traits_cap = 0, ydig_cap = 0, qd_cap = 0, qm_cap = 0, wmask_cap = 0, qc_cap = 0, qtot_cap = 0,
           yscale_cap = 0;
    bool qm_valid = false;
    epi::MmaMaps maps;
    // tensor form, streamed-B variant: the expanded B rows of every SNP and trait (12 bytes per
    // SNP, individual and trait), built on first use after each genotype or trait load
    int8_t *d_x = nullptr;
    size_t x_cap = 0;
    bool x_valid = false;
    std::vector<double> qc;
    // plain form: marginals per (trait, SNP) and the sum of y^2 per trait
    double *d_pmC = nullptr, *d_pmQ = nullptr, *d_ysq = nullptr;
    int32_t *d_pmN = nullptr;
    size_t pmC_cap = 0, pmQ_cap = 0, pmN_cap = 0, ysq_cap = 0;
    bool pm_valid = false;
    // scan scratch
    DevHit *d_hits = nullptr;
    int64_t hit_cap = 0;
    unsigned long long *d_counters = nullptr;
    unsigned int *d_maxf = nullptr;
    int maxf_cap = 0;
    BlockDesc *d_blocks = nullptr;
    int blocks_cap = 0;
    // pinned host staging of the device part of a scan: the block schedule it uploads, the
    // counters and maxima it reads back
    BlockDesc *h_blocks = nullptr;
    int h_blocks_cap = 0;
    unsigned long long *h_state = nullptr;  // counters[4], then 2 x ntraits encoded maxima
    size_t h_state_cap = 0;
    // the device part of the last scan, captured as a CUDA graph, and what it was captured for
    cudaGraphExec_t gexec = nullptr;
    std::vector<unsigned char> gkey;
    // last scan
    double last_ms = 0.0;
    int64_t last_pairs = 0;
    int last_launches = 0;
    int last_form = 0;
    std::string last_config;  // form, kernel variant and how it was chosen
    std::string err;
};

static epi_status set_err(epi_ctx *ctx, epi_status s, const char *fmt, ...)
{
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return s;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            cudaGetLastError(); /* a failed call must not surface again at the next launch check */  \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? EPI_E_NOMEM : EPI_E_CUDA,          \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);      \
        }                                                                                             \
    } while (0)

template <class T>
static cudaError_t ensure(T **p, size_t *cap_bytes, size_t bytes)
{
    if (*p && *cap_bytes >= bytes) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap_bytes = 0;
    cudaError_t e = cudaMalloc((void **)p, bytes ? bytes : 16);
    if (e == cudaSuccess) *cap_bytes = bytes;
    return e;
}

extern "C" {

void epi_default_opts(epi_scan_opts *o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->test = 'f';
    o->safe = 0;
    o->chunk = 128;
    o->t1 = 6.5f;
    o->t2 = 10.5f;
    o->form = EPI_FORM_AUTO;
    o->report_trait = 0;
}

const char *epi_strerror(epi_status s)
{
    switch (s) {
    case EPI_OK: return "success";
    case EPI_E_INVALID: return "invalid argument";
    case EPI_E_CUDA: return "CUDA error";
    case EPI_E_NOMEM: return "out of device memory";
    case EPI_E_OVERFLOW: return "more hits than the output capacity";
    case EPI_E_STATE: return "genotypes or phenotypes not loaded";
    case EPI_E_TIMEOUT: return "device wait timed out";
    case EPI_E_NODEVICE: return "no suitable CUDA device";
    case EPI_E_UNSUPPORTED: return "unsupported option for this form";
    }
    return "unknown status";
}

const char *epi_last_error(const epi_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

epi_status epi_open(int32_t device, epi_ctx **out)
{
    if (!out) return EPI_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return EPI_E_NODEVICE;
    if (device < 0 || device >= n) return EPI_E_NODEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return EPI_E_NODEVICE;
    if (prop.major != 10) return EPI_E_NODEVICE;  // the library carries sm_100a code only
    epi_ctx *ctx = new epi_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    snprintf(ctx->name, sizeof(ctx->name), "%s", prop.name);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e == cudaSuccess) e = cudaMalloc((void **)&ctx->d_counters, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        epi_close(ctx);
        return EPI_E_CUDA;
    }
    *out = ctx;
    return EPI_OK;
}

epi_status epi_close(epi_ctx *ctx)
{
    if (!ctx) return EPI_OK;
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    void *bufs[] = {ctx->d_raw, ctx->d_planes, ctx->d_hcodes, ctx->d_h3, ctx->d_missbits, ctx->d_y, ctx->d_q,
                    ctx->d_wmask, ctx->d_qc, ctx->d_yscale, ctx->d_qd, ctx->d_qtot, ctx->d_qm, ctx->d_ydig,
                    ctx->d_hits, ctx->d_counters, ctx->d_maxf, ctx->d_blocks, ctx->d_maj, ctx->d_pmC,
                    ctx->d_pmQ, ctx->d_ysq, ctx->d_pmN, ctx->d_x};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->h_blocks) cudaFreeHost(ctx->h_blocks);
    if (ctx->h_state) cudaFreeHost(ctx->h_state);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return EPI_OK;
}

epi_status epi_device_info(const epi_ctx *ctx, char *name, int32_t name_len, int32_t *sm_count)
{
    if (!ctx) return EPI_E_INVALID;
    if (name && name_len > 0) snprintf(name, (size_t)name_len, "%s", ctx->name);
    if (sm_count) *sm_count = ctx->sm_count;
    return EPI_OK;
}

epi_status epi_load_packed(epi_ctx *ctx, const int32_t *gpack, int32_t nid, int32_t nsnp, int32_t npack,
                           int32_t remain)
{
    if (!ctx) return EPI_E_INVALID;
    if (!gpack || nid < 1 || nsnp < 1)
        return set_err(ctx, EPI_E_INVALID, "epi_load_packed: need gpack, nid >= 1, nsnp >= 1");
    if (npack != nid / 16 || remain != nid % 16)
        return set_err(ctx, EPI_E_INVALID, "epi_load_packed: npack/remain (%d/%d) inconsistent with nid %d "
                       "(src/readplink.c:1071-1072)", npack, remain, nid);
    CK(cudaSetDevice(ctx->device));
    const int npack1 = remain ? npack + 1 : npack;
    const int Wp = ((nid + 31) / 32 + 3) / 4 * 4;  // multiple of 4 words = 128 individuals
    const int Wc = 2 * Wp;
    CK(ensure(&ctx->d_raw, &ctx->raw_cap, (size_t)nsnp * npack1 * sizeof(int32_t)));
    CK(ensure(&ctx->d_planes, &ctx->planes_cap, (size_t)nsnp * Wp * sizeof(uint4)));
    CK(ensure(&ctx->d_hcodes, &ctx->hcodes_cap, (size_t)nsnp * Wp * 32));
    CK(ensure(&ctx->d_h3, &ctx->h3_cap, 3 * (size_t)nsnp * Wp * 32));
    CK(ensure(&ctx->d_missbits, &ctx->missbits_cap, (size_t)nsnp * Wp * sizeof(uint32_t)));
    CK(ensure(&ctx->d_maj, &ctx->maj_cap, (size_t)nsnp));
    CK(cudaMemcpyAsync(ctx->d_raw, gpack, (size_t)nsnp * npack1 * sizeof(int32_t), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(epi::launch_unpack(ctx->d_raw, nsnp, nid, npack, remain, ctx->d_planes, Wp, nullptr, Wc, ctx->d_hcodes,
                          ctx->d_h3, ctx->d_missbits, ctx->stream));
    CK(epi::launch_major(ctx->d_planes, nsnp, Wp, ctx->d_maj, ctx->stream));
    ctx->qm_valid = false;
    ctx->pm_valid = false;
    ctx->x_valid = false;
    CK(epi::mma_encode_genotypes(&ctx->maps, ctx->d_hcodes, ctx->d_h3, nsnp, 32 * Wp));
    if (ctx->traits_nid != nid) ctx->ntraits = 0;  // traits no longer match
    ctx->nid = nid;
    ctx->nsnp = nsnp;
    ctx->npack = npack;
    ctx->remain = remain;
    ctx->Wp = Wp;
    ctx->Wc = Wc;
    ctx->Np = 32 * Wp;
    return EPI_OK;
}

epi_status epi_set_traits(epi_ctx *ctx, const float *y, int32_t nid, int32_t ntraits, const uint8_t *valid)
{
    if (!ctx) return EPI_E_INVALID;
    if (!y || nid < 1 || ntraits < 1) return set_err(ctx, EPI_E_INVALID, "epi_set_traits: bad arguments");
    if (ctx->nid == 0) return set_err(ctx, EPI_E_STATE, "epi_set_traits: load genotypes first");
    if (nid != ctx->nid)
        return set_err(ctx, EPI_E_INVALID, "epi_set_traits: %d individuals, genotypes have %d", nid, ctx->nid);
    CK(cudaSetDevice(ctx->device));
    const int Np = ctx->Np, Wp = ctx->Wp;
    std::vector<float> hy((size_t)ntraits * Np, 0.0f), hq((size_t)ntraits * Np, 0.0f);
    std::vector<uint32_t> hw((size_t)ntraits * Wp, 0u);
    ctx->qc.assign(ntraits, 0.0);
    // Each centred trait is scaled by a power of two that brings its largest magnitude into
    // [0.5, 1). F and F2 do not depend on the trait's scale, and a power-of-two factor is
    // exact in binary floating point, so in the normal range every result is bit-identical
    // to the unscaled computation; a trait in units of 1e20 or 1e-20 no longer overflows or
    // underflows the single-precision sums of squares.
    std::vector<double> p2s(ntraits, 1.0), ysq(ntraits, 0.0);
    for (int t = 0; t < ntraits; ++t) {
        const float *yt = y + (size_t)t * nid;
        const uint8_t *vt = valid ? valid + (size_t)t * nid : nullptr;
        double sum = 0.0;
        long long nv = 0;
        for (int k = 0; k < nid; ++k) {
            const bool ok = vt ? vt[k] != 0 : yt[k] != -9.0f;
            if (ok) {
                sum += (double)yt[k];
                ++nv;
                hw[(size_t)t * Wp + k / 32] |= 1u << (k % 32);
            }
        }
        const double mu = nv ? sum / (double)nv : 0.0;
        double maxabs = 0.0;
        for (int k = 0; k < nid; ++k)
            if (hw[(size_t)t * Wp + k / 32] >> (k % 32) & 1u) maxabs = std::max(maxabs, std::fabs((double)yt[k] - mu));
        const double p2 = (maxabs > 0.0 && std::isfinite(maxabs)) ? std::ldexp(1.0, -(std::ilogb(maxabs) + 1)) : 1.0;
        p2s[t] = p2;
        double s2 = 0.0;
        for (int k = 0; k < nid; ++k) {
            if (hw[(size_t)t * Wp + k / 32] >> (k % 32) & 1u) {
                const float yc = (float)(((double)yt[k] - mu) * p2);
                hy[(size_t)t * Np + k] = yc;
                s2 += (double)yc * (double)yc;
            }
        }
        const double c = nv ? s2 / (double)nv : 0.0;
        ctx->qc[t] = c;
        ysq[t] = s2;
        for (int k = 0; k < nid; ++k) {
            if (hw[(size_t)t * Wp + k / 32] >> (k % 32) & 1u) {
                const double yc = hy[(size_t)t * Np + k];
                hq[(size_t)t * Np + k] = (float)(yc * yc - c);
            }
        }
    }
    // tensor form: per valid individual the flag and three balanced base-256 digits of
    // Y = round(y * 2^sy) (|Y| <= 8355711); hqd holds ytilde^2 = (Y 2^-sy)^2 (exact in FP64:
    // |Y| < 2^23) and Y; hsc per trait 2^-sy, the sum of Y and the number of valid individuals;
    // hqtot the sum of ytilde^2.
    constexpr int ND = 4;
    std::vector<int8_t> hd((size_t)ntraits * ND * Np, 0);
    std::vector<double> hqd(2 * (size_t)ntraits * Np, 0.0), hqtot(ntraits, 0.0), hsc(3 * (size_t)ntraits, 1.0);
    for (int t = 0; t < ntraits; ++t) {
        const float *yt = y + (size_t)t * nid;
        auto ok = [&](int k) { return (hw[(size_t)t * Wp + k / 32] >> (k % 32) & 1u) != 0; };
        double sum = 0.0;
        long long nv = 0;
        for (int k = 0; k < nid; ++k)
            if (ok(k)) {
                sum += (double)yt[k];
                ++nv;
            }
        const double mu = nv ? sum / (double)nv : 0.0;
        const double p2 = p2s[t];
        double maxabs = 0.0;
        for (int k = 0; k < nid; ++k)
            if (ok(k)) maxabs = std::max(maxabs, std::fabs(((double)yt[k] - mu) * p2));
        const int sy = (maxabs > 0.0 && std::isfinite(maxabs)) ? (int)std::floor(std::log2(8355000.0 / maxabs)) : 0;
        const double scale = std::ldexp(1.0, sy);
        hsc[t] = std::ldexp(1.0, -sy);
        int8_t *d0 = hd.data() + (size_t)t * ND * Np;
        long long ysum = 0;
        for (int k = 0; k < nid; ++k) {
            if (!ok(k)) continue;
            long long Y = std::llround(((double)yt[k] - mu) * p2 * scale);
            Y = std::min(8355711LL, std::max(-8355711LL, Y));
            const long long a0 = ((Y + 128) & 255) - 128, Y1 = (Y - a0) / 256;
            const long long a1 = ((Y1 + 128) & 255) - 128, a2 = (Y1 - a1) / 256;
            d0[k] = 1;
            d0[Np + k] = (int8_t)a0;
            d0[2 * (size_t)Np + k] = (int8_t)a1;
            d0[3 * (size_t)Np + k] = (int8_t)a2;
            const double yq = (double)Y * hsc[t];
            hqd[(size_t)t * Np + k] = yq * yq;
            hqd[((size_t)ntraits + t) * Np + k] = (double)Y;
            hqtot[t] += yq * yq;
            ysum += Y;
        }
        hsc[ntraits + t] = (double)ysum;
        hsc[2 * (size_t)ntraits + t] = (double)nv;
    }
    size_t need = (size_t)ntraits * Np * sizeof(float);
    size_t cap_y = ctx->traits_cap, cap_q = ctx->traits_cap;
    CK(ensure(&ctx->d_y, &cap_y, need));
    CK(ensure(&ctx->d_q, &cap_q, need));
    ctx->traits_cap = std::min(cap_y, cap_q);
    // buffers are kept across calls while they are large enough: a cudaFree would
    // synchronise the device on every trait upload
    CK(ensure(&ctx->d_wmask, &ctx->wmask_cap, (size_t)ntraits * Wp * sizeof(uint32_t)));
    CK(ensure(&ctx->d_qc, &ctx->qc_cap, (size_t)ntraits * sizeof(double)));
    CK(cudaMemcpyAsync(ctx->d_y, hy.data(), need, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_q, hq.data(), need, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_wmask, hw.data(), hw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_qc, ctx->qc.data(), ntraits * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(ensure(&ctx->d_ysq, &ctx->ysq_cap, (size_t)ntraits * sizeof(double)));
    CK(cudaMemcpyAsync(ctx->d_ysq, ysq.data(), ntraits * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(ensure(&ctx->d_ydig, &ctx->ydig_cap, hd.size()));
    CK(ensure(&ctx->d_qd, &ctx->qd_cap, hqd.size() * sizeof(double)));
    CK(ensure(&ctx->d_qtot, &ctx->qtot_cap, (size_t)ntraits * sizeof(double)));
    CK(ensure(&ctx->d_yscale, &ctx->yscale_cap, hsc.size() * sizeof(double)));
    CK(cudaMemcpyAsync(ctx->d_ydig, hd.data(), hd.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(epi::mma_encode_traits(&ctx->maps, ctx->d_ydig, ntraits, Np));
    CK(cudaMemcpyAsync(ctx->d_qd, hqd.data(), hqd.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_qtot, hqtot.data(), ntraits * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_yscale, hsc.data(), hsc.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->ntraits = ntraits;
    ctx->traits_nid = nid;
    ctx->qm_valid = false;
    ctx->pm_valid = false;
    ctx->x_valid = false;
    return EPI_OK;
}

epi_status epi_set_phenotype(epi_ctx *ctx, const float *phen, int32_t nid, int32_t safe)
{
    if (!ctx) return EPI_E_INVALID;
    if (!safe) return epi_set_traits(ctx, phen, nid, 1, nullptr);
    std::vector<uint8_t> v((size_t)(nid > 0 ? nid : 0), 1);
    return epi_set_traits(ctx, phen, nid, 1, v.data());
}

void epi_permute_phenotype(float *phen, int32_t nid, uint32_t seed)
{
    if (!phen) return;
    srand(seed);
    for (int i = nid; i > 1; i--) {
        const int r = rand() % i;
        const float t = phen[r];
        phen[r] = phen[i - 1];
        phen[i - 1] = t;
    }
}

}  // extern "C"

// number of pairs (gx, gy) of a block with start1+gx > start2+gy
static int64_t block_pairs(const epi_block &b)
{
    int64_t n = 0;
    const int64_t d = (int64_t)b.start1 - b.start2;
    for (int64_t gx = 0; gx < b.size1; ++gx) {
        int64_t lim = gx + d;
        if (lim > b.size2) lim = b.size2;
        if (lim > 0) n += lim;
    }
    return n;
}

namespace {

struct ScanRun {
    epi::ScanArgs args;
    int form;
    int variant;  // the form's kernel variant (tile shape or ring depths)
    int64_t ntiles;
    std::vector<BlockDesc> desc;
};

epi_status check_opts(epi_ctx *ctx, const epi_scan_opts *o)
{
    if (!o) return set_err(ctx, EPI_E_INVALID, "null options");
    if (o->test != 'f' && o->test != 'i') return set_err(ctx, EPI_E_INVALID, "test must be 'f' or 'i'");
    if (o->safe != 0 && o->safe != 1) return set_err(ctx, EPI_E_INVALID, "safe must be 0 or 1");
    if (o->chunk < 1) return set_err(ctx, EPI_E_INVALID, "chunk must be >= 1");
    if (o->form < EPI_FORM_AUTO || o->form > EPI_FORM_TENSOR) return set_err(ctx, EPI_E_INVALID, "bad form");
    if (o->report_trait < -1 || o->report_trait >= ctx->ntraits)
        return set_err(ctx, EPI_E_INVALID, "report_trait %d out of range", o->report_trait);
    if (o->wait_limit_ms < 0) return set_err(ctx, EPI_E_INVALID, "wait_limit_ms must be >= 0");
    if (o->debug != 0 && o->debug != EPI_DEBUG_STALL) return set_err(ctx, EPI_E_INVALID, "bad debug flags");
    if (o->no_graph != 0 && o->no_graph != 1) return set_err(ctx, EPI_E_INVALID, "no_graph must be 0 or 1");
    if (o->tile_config < 0) return set_err(ctx, EPI_E_INVALID, "tile_config must be >= 0");
    return EPI_OK;
}

int pick_form(const epi_ctx *ctx, const epi_scan_opts *o)
{
    if (o->form != EPI_FORM_AUTO) return o->form;
    if (epi::mma_available() && ctx->nid >= epi::mma_min_nid() && ctx->Np <= epi::mma_max_nid())
        return EPI_FORM_TENSOR;
    return EPI_FORM_POPC;
}

// Builds the kernel arguments and tile schedule for `blocks` and uploads the schedule.
// Bytes of the streamed-B variant's expanded rows, and whether they may be allocated: at most
// 32 GiB and half the device's free memory (beyond, that variant is not a candidate).
static size_t x_bytes(const epi_ctx *ctx) { return 12 * (size_t)ctx->nsnp * ctx->Np * ctx->ntraits; }
static bool x_usable(const epi_ctx *ctx)
{
    const size_t need = x_bytes(ctx);
    if (need <= ctx->x_cap) return true;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    return need <= (32ull << 30) && need <= fr / 2 + ctx->x_cap;
}

// The streamed-B variant as an autotuner candidate: only up to 6,144 padded individuals. Its
// expanded rows are 12 bytes per SNP and individual, and the DRAM traffic of its super-tiles
// grows with N per second of scanning; at N = 10,000 a full scan then runs into the 1 kW power
// cap (SM clock ~1,350 MHz against ~1,935 MHz for the shared-memory producers) and ends 12%
// slower, although the autotuner's short sample, run before the cap bites, ranks it 15% faster.
// At N = 4,000 it is 10-14% faster at full clock. tile_config can still force it.
static bool x_candidate(const epi_ctx *ctx) { return ctx->Np <= 6144 && x_usable(ctx); }

epi_status setup_run(epi_ctx *ctx, const epi_block *blocks, int nblocks, const epi_scan_opts *o, ScanRun &r,
                     int variant)
{
    r.form = pick_form(ctx, o);
    r.variant = variant;
    if (r.form == EPI_FORM_TENSOR && !epi::mma_available())
        return set_err(ctx, EPI_E_UNSUPPORTED, "tensor form not available in this library");
    if (r.form == EPI_FORM_TENSOR && ctx->Np > epi::mma_max_nid())
        return set_err(ctx, EPI_E_UNSUPPORTED, "tensor form: at most %d individuals", epi::mma_max_nid());
    if (r.form == EPI_FORM_POPC && ctx->nid > 65535)
        return set_err(ctx, EPI_E_UNSUPPORTED, "popcount form counts in 16 bits: at most 65535 individuals "
                       "(the reference's unsigned short counts, EpiOpenCL.c:68)");
    if (r.form == EPI_FORM_TENSOR && epi::mma_needs_x(variant)) {
        if (!x_usable(ctx))
            return set_err(ctx, EPI_E_UNSUPPORTED, "tensor variant %d: its %zu bytes of expanded B rows do not fit",
                           variant + 1, x_bytes(ctx));
        if (!ctx->x_valid) {
            CK(ensure(&ctx->d_x, &ctx->x_cap, x_bytes(ctx)));
            CK(epi::launch_expand(ctx->d_hcodes, ctx->d_ydig, ctx->nsnp, ctx->Np, ctx->ntraits, ctx->d_x,
                                  ctx->stream));
            CK(epi::mma_encode_x(&ctx->maps, ctx->d_x, ctx->nsnp, ctx->Np, ctx->ntraits));
            ctx->x_valid = true;
        }
    }
    int TI = epi::mma_tile_i(), TJ = epi::mma_tile_j();
    if (r.form == EPI_FORM_POPC) {
        epi::popc_shape(variant, &TI, &TJ, nullptr);
        CK(epi::popc_encode_planes(variant, &ctx->pmaps, ctx->d_planes, ctx->nsnp, ctx->Wp));
    }
    r.desc.resize(nblocks);
    int64_t base = 0;
    for (int b = 0; b < nblocks; ++b) {
        const epi_block &e = blocks[b];
        if (e.size1 < 0 || e.size2 < 0 || e.start1 < 0 || e.start2 < 0 ||
            (int64_t)e.start1 + e.size1 > ctx->nsnp || (int64_t)e.start2 + e.size2 > ctx->nsnp)
            return set_err(ctx, EPI_E_INVALID, "block %d out of range", b);
        BlockDesc &d = r.desc[b];
        d.start1 = e.start1;
        d.size1 = e.size1;
        d.start2 = e.start2;
        d.size2 = e.size2;
        d.tiles_i = (e.size1 + TI - 1) / TI;
        d.tiles_j = (e.size2 + TJ - 1) / TJ;
        d.tile_base = base;
        base += (int64_t)d.tiles_i * d.tiles_j;
    }
    r.ntiles = base;
    size_t bcap = (size_t)ctx->blocks_cap * sizeof(BlockDesc);
    CK(ensure(&ctx->d_blocks, &bcap, (size_t)std::max(nblocks, 1) * sizeof(BlockDesc)));
    ctx->blocks_cap = (int)(bcap / sizeof(BlockDesc));
    if (ctx->h_blocks_cap < nblocks) {
        if (ctx->h_blocks) cudaFreeHost(ctx->h_blocks);
        ctx->h_blocks = nullptr;
        ctx->h_blocks_cap = 0;
        CK(cudaHostAlloc((void **)&ctx->h_blocks, (size_t)nblocks * sizeof(BlockDesc), cudaHostAllocDefault));
        ctx->h_blocks_cap = nblocks;
    }
    const size_t state = 4 * sizeof(unsigned long long) + 2 * (size_t)ctx->ntraits * sizeof(unsigned int);
    if (ctx->h_state_cap < state) {
        if (ctx->h_state) cudaFreeHost(ctx->h_state);
        ctx->h_state = nullptr;
        ctx->h_state_cap = 0;
        CK(cudaHostAlloc((void **)&ctx->h_state, state, cudaHostAllocDefault));
        ctx->h_state_cap = state;
    }
    if (ctx->maxf_cap < 2 * ctx->ntraits) {
        if (ctx->d_maxf) cudaFree(ctx->d_maxf);
        ctx->d_maxf = nullptr;
        CK(cudaMalloc((void **)&ctx->d_maxf, 2 * ctx->ntraits * sizeof(unsigned int)));
        ctx->maxf_cap = 2 * ctx->ntraits;
    }
    if (r.form == EPI_FORM_TENSOR && !ctx->qm_valid) {
        const size_t tn = (size_t)ctx->ntraits * ctx->nsnp;
        CK(ensure(&ctx->d_qm, &ctx->qm_cap, 3 * tn * sizeof(double)));
        CK(epi::launch_qmiss(ctx->d_missbits, ctx->nsnp, ctx->Wp, ctx->d_wmask, ctx->d_qd,
                             ctx->d_qd + (size_t)ctx->ntraits * ctx->Np, ctx->Np, ctx->ntraits, ctx->d_qm,
                             ctx->d_qm + tn, ctx->d_qm + 2 * tn, ctx->stream));
        ctx->qm_valid = true;
    }
    if (r.form == EPI_FORM_POPC && !ctx->pm_valid) {
        const size_t tn = (size_t)ctx->ntraits * ctx->nsnp;
        CK(ensure(&ctx->d_pmC, &ctx->pmC_cap, 3 * tn * sizeof(double)));
        CK(ensure(&ctx->d_pmN, &ctx->pmN_cap, 3 * tn * sizeof(int32_t)));
        CK(ensure(&ctx->d_pmQ, &ctx->pmQ_cap, tn * sizeof(double)));
        CK(epi::launch_marg(ctx->d_planes, ctx->nsnp, ctx->Wp, ctx->d_y, ctx->d_wmask, ctx->Np, ctx->ntraits,
                            ctx->d_pmC, ctx->d_pmN, ctx->d_pmQ, ctx->stream));
        ctx->pm_valid = true;
    }
    epi::ScanArgs &a = r.args;
    memset(&a, 0, sizeof(a));
    a.planes = ctx->d_planes;
    a.hcodes = ctx->d_hcodes;
    a.missbits = ctx->d_missbits;
    a.Wp = ctx->Wp;
    a.Wc = ctx->Wc;
    a.nid = ctx->nid;
    a.nsnp = ctx->nsnp;
    a.yscale = ctx->d_yscale;
    a.ytot = ctx->d_yscale + ctx->ntraits;
    a.nvalid = ctx->d_yscale + 2 * (size_t)ctx->ntraits;
    a.qd = ctx->d_qd;
    a.qtot = ctx->d_qtot;
    a.qm = ctx->d_qm;
    a.sm = ctx->d_qm + (size_t)ctx->ntraits * ctx->nsnp;
    a.nm = ctx->d_qm + 2 * (size_t)ctx->ntraits * ctx->nsnp;
    a.ydig = ctx->d_ydig;
    a.maj = ctx->d_maj;
    a.pmC = ctx->d_pmC;
    a.pmN = ctx->d_pmN;
    a.pmQ = ctx->d_pmQ;
    a.ysq = ctx->d_ysq;
    a.y = ctx->d_y;
    a.q = ctx->d_q;
    a.wmask = ctx->d_wmask;
    a.qc = ctx->d_qc;
    a.Np = ctx->Np;
    a.ntraits = ctx->ntraits;
    a.blocks = ctx->d_blocks;
    a.nblocks = nblocks;
    a.ntiles = r.ntiles;
    a.test_int = o->test == 'i';
    a.safe = o->safe;
    a.report_trait = o->report_trait;
    a.t1 = o->t1;
    a.t2 = o->t2;
    a.wait_ns = o->wait_limit_ms > 0 ? (unsigned long long)o->wait_limit_ms * 1000000ull : 2000000000ull;
    a.debug_stall = o->debug == EPI_DEBUG_STALL;
    // streamed-B variant: super-tiles of about 40 MB of A rows (3 bytes per SNP and individual)
    // and expanded B rows (12 per SNP, individual and trait), equal sides in pair tiles
    {
        const double per = (3.0 * epi::mma_tile_i() + 12.0 * epi::mma_tile_j() * ctx->ntraits) * ctx->Np;
        a.xsi = a.xsj = std::max(1, (int)(40e6 / per));
    }
    a.counters = ctx->d_counters;
    a.maxf = ctx->d_maxf;
    a.maxf2 = ctx->d_maxf + ctx->ntraits;
    return EPI_OK;
}

// The device part of a scan, on the context's stream and nothing but stream operations (so it
// can be captured): counters and maxima reset, the block schedule uploaded from pinned memory,
// the selected form's persistent kernel between the timing events, and the counters and maxima
// read back into pinned memory.
cudaError_t enqueue_scan(epi_ctx *ctx, const ScanRun &r, int grid, int nblocks, bool capturing)
{
    cudaStream_t s = ctx->stream;
    // under stream capture the timing events are recorded as external records, which become
    // event nodes of the graph (so they time every replay); a direct launch records them plainly
    const unsigned int ev_flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    epi::k_scan_init<<<1, 256, 0, s>>>(ctx->d_counters, ctx->d_maxf, 2 * ctx->ntraits);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && nblocks)
        e = cudaMemcpyAsync(ctx->d_blocks, ctx->h_blocks, nblocks * sizeof(BlockDesc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev0, s, ev_flags);
    if (e == cudaSuccess && r.ntiles > 0)
        e = r.form == EPI_FORM_TENSOR ? epi::mma_enqueue(r.variant, r.args, ctx->maps, grid, s)
                                      : epi::popc_enqueue(r.variant, r.args, ctx->pmaps, grid, s);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev1, s, ev_flags);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->h_state, ctx->d_counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->h_state + 4, ctx->d_maxf, 2 * (size_t)ctx->ntraits * sizeof(unsigned int),
                            cudaMemcpyDeviceToHost, s);
    return e;
}

template <class T>
static void key_add(std::vector<unsigned char> &k, const T &v)
{
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// Runs the device part of a scan. With use_graph, a repeat of the previous scan's shape (same
// kernel arguments, tensor maps, schedule and launch shape) replays the CUDA graph captured for
// it with one launch; any other scan is captured anew first. Without, the operations are
// launched one by one.
epi_status launch_run(epi_ctx *ctx, ScanRun &r, int nblocks, bool use_graph)
{
    int grid = 0;
    if (r.ntiles > 0) {
        const int64_t units = r.ntiles * (int64_t)ctx->ntraits;
        if (r.form == EPI_FORM_TENSOR) {
            // one CTA pair per unit (tile x trait) up to every SM
            CK(epi::mma_prepare(r.variant, ctx->ntraits, (int)std::min<int64_t>(2 * units, ctx->sm_count), &grid));
        } else {
            // one CTA per unit up to every SM
            CK(epi::popc_prepare(r.variant));
            grid = (int)std::min<int64_t>(units, ctx->sm_count);
        }
    }
    if (nblocks) memcpy(ctx->h_blocks, r.desc.data(), nblocks * sizeof(BlockDesc));
    ctx->last_launches = r.ntiles > 0 ? 2 : 1;  // the state reset and the scan kernel
    ctx->last_form = r.form;
    if (!use_graph) {
        CK(enqueue_scan(ctx, r, grid, nblocks, false));
        return EPI_OK;
    }
    std::vector<unsigned char> key;
    key_add(key, r.args);
    key_add(key, r.form);
    key_add(key, r.variant);
    key_add(key, grid);
    key_add(key, ctx->ntraits);
    if (r.form == EPI_FORM_TENSOR) key_add(key, ctx->maps);
    else key_add(key, ctx->pmaps);
    key.insert(key.end(), reinterpret_cast<const unsigned char *>(r.desc.data()),
               reinterpret_cast<const unsigned char *>(r.desc.data() + nblocks));
    if (!ctx->gexec || key != ctx->gkey) {
        if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
        ctx->gexec = nullptr;
        ctx->gkey.clear();
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = enqueue_scan(ctx, r, grid, nblocks, true);
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);  // ends the capture in any case
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            CK(e != cudaSuccess ? e : e2);
        }
        const cudaError_t e3 = cudaGraphInstantiate(&ctx->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) ctx->gexec = nullptr;
        CK(e3);
        ctx->gkey = std::move(key);
    }
    CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    return EPI_OK;
}

// ---- autotuner: the kernel variant per (device, form, padded individuals, traits) ----
//
// Every candidate of the form's table (tile shapes of the plain form, ring depths of the
// tensor form) scans a sample block of the loaded genotypes and traits -- large enough for a
// few waves of tiles over every SM -- once to warm up and once timed with CUDA events; the
// fastest is kept for the process. The reference has one such knob, the chunk size of its
// launches (src/main.c:115-130, src/EpiOpenCL.c:1353-1362), set by hand.
struct TuneEntry {
    int device, form, Np, ntraits, variant;
    std::string how;
};
static std::mutex g_tune_mu;
static std::vector<TuneEntry> g_tune;

int form_variants(int form) { return form == EPI_FORM_TENSOR ? epi::mma_shapes() : epi::popc_shapes(); }

std::string variant_desc(int form, int v)
{
    const char *d = nullptr;
    int ti = 0, tj = 0;
    if (form == EPI_FORM_TENSOR) epi::mma_shape(v, &d);
    else epi::popc_shape(v, &ti, &tj, &d);
    return std::string(form == EPI_FORM_TENSOR ? "tensor form, " : "plain form, ") + d;
}

epi_status pick_variant(epi_ctx *ctx, const epi_scan_opts *o, int form, int *v, std::string *how)
{
    const int nv = form_variants(form);
    if (o->tile_config > 0) {
        if (o->tile_config > nv)
            return set_err(ctx, EPI_E_INVALID, "tile_config %d: this form has %d candidates", o->tile_config, nv);
        *v = o->tile_config - 1;
        *how = "requested";
        return EPI_OK;
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        // (a kept choice of the streamed-B variant holds only while this context's expanded rows
        // would fit: another context of the same shape may hold more SNPs)
        for (const TuneEntry &t : g_tune)
            if (t.device == ctx->device && t.form == form && t.Np == ctx->Np && t.ntraits == ctx->ntraits &&
                !(form == EPI_FORM_TENSOR && epi::mma_needs_x(t.variant) && !x_candidate(ctx))) {
                *v = t.variant;
                *how = t.how;
                return EPI_OK;
            }
    }
    if (nv == 1) {
        *v = 0;
        *how = "only candidate";
        return EPI_OK;
    }
    // sample: an off-diagonal s x s block (every pair valid) when the genome holds one, with
    // enough tiles for about sixteen waves over the SMs at this trait count, at least 1,024
    // SNPs a side (a smaller block ranked the tensor variants wrongly at 64 traits) unless that
    // makes more than 2^28 pair tests, and at most 2,048
    const int T = ctx->ntraits;
    int s = (int)std::ceil(std::sqrt(16.0 * ctx->sm_count * 4096.0 / T));
    const int lo = std::max(256, std::min(1024, (int)std::sqrt(268435456.0 / T)));
    s = std::max(lo, std::min(s, 2048));
    epi_block blk;
    if (ctx->nsnp >= 2 * s) blk = {s, s, 0, s};
    else blk = {0, ctx->nsnp, 0, ctx->nsnp};
    if (ctx->hit_cap == 0) {
        const int64_t initial = 1 << 20;
        CK(cudaMalloc((void **)&ctx->d_hits, initial * sizeof(DevHit)));
        ctx->hit_cap = initial;
    }
    epi_scan_opts o2 = *o;
    o2.report_trait = 0;
    std::vector<float> ms(nv, 0.0f);
    for (int c = 0; c < nv; ++c) {
        // the streamed-B variant is no candidate where its expanded rows would not fit or would
        // run into the power cap (x_candidate)
        if (form == EPI_FORM_TENSOR && epi::mma_needs_x(c) && !x_candidate(ctx)) {
            ms[c] = INFINITY;
            continue;
        }
        ScanRun r;
        epi_status st = setup_run(ctx, &blk, 1, &o2, r, c);
        if (st != EPI_OK) return st;
        r.args.hits = ctx->d_hits;
        r.args.cap = ctx->hit_cap;
        for (int rep = 0; rep < 2; ++rep) {
            st = launch_run(ctx, r, 1, false);
            if (st != EPI_OK) return st;
        }
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->h_state[2] != 0)
            return set_err(ctx, EPI_E_TIMEOUT, "a bounded device wait gave up while tuning (site %llu)",
                           ctx->h_state[3]);
        CK(cudaEventElapsedTime(&ms[c], ctx->ev0, ctx->ev1));
    }
    const int best = (int)(std::min_element(ms.begin(), ms.end()) - ms.begin());
    char buf[256];
    int len = snprintf(buf, sizeof(buf), "autotuned on a %d x %d-SNP block:", blk.size1, blk.size2);
    for (int c = 0; c < nv && len < (int)sizeof(buf); ++c)
        len += std::isfinite(ms[c]) ? snprintf(buf + len, sizeof(buf) - len, "%s %.3f ms", c ? " /" : "", ms[c])
                                    : snprintf(buf + len, sizeof(buf) - len, "%s n/a", c ? " /" : "");
    *v = best;
    *how = buf;
    // the streamed-B candidate's expanded rows (up to 32 GiB) are released when it lost
    if (form == EPI_FORM_TENSOR && !epi::mma_needs_x(best) && ctx->d_x) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->d_x);
        ctx->d_x = nullptr;
        ctx->x_cap = 0;
        ctx->x_valid = false;
    }
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.push_back({ctx->device, form, ctx->Np, ctx->ntraits, best, *how});
    return EPI_OK;
}

struct HitKey {
    int32_t trait, block, s, k, l, gx, gy;
    int64_t idx;
};

}  // namespace

extern "C" epi_status epi_scan(epi_ctx *ctx, const epi_block *blocks, int32_t nblocks, const epi_scan_opts *opts,
                               epi_hit *hits, int64_t cap, int64_t *nhits, int32_t *hit_block, int32_t *hit_trait,
                               float *max_f, float *max_f2)
{
    if (!ctx) return EPI_E_INVALID;
    ctx->err.clear();
    if (ctx->nid == 0 || ctx->ntraits == 0)
        return set_err(ctx, EPI_E_STATE, "epi_scan: load genotypes and traits first");
    if (nblocks < 0 || (nblocks > 0 && !blocks)) return set_err(ctx, EPI_E_INVALID, "epi_scan: bad blocks");
    if (cap < 0 || (cap > 0 && !hits)) return set_err(ctx, EPI_E_INVALID, "epi_scan: bad hit buffer");
    epi_status s = check_opts(ctx, opts);
    if (s != EPI_OK) return s;
    CK(cudaSetDevice(ctx->device));
    const int form = pick_form(ctx, opts);
    int variant = 0;
    std::string how;
    s = pick_variant(ctx, opts, form, &variant, &how);
    if (s != EPI_OK) return s;
    ScanRun r;
    s = setup_run(ctx, blocks, nblocks, opts, r, variant);
    if (s != EPI_OK) return s;
    if (ctx->hit_cap == 0) {
        const int64_t initial = 1 << 20;
        CK(cudaMalloc((void **)&ctx->d_hits, initial * sizeof(DevHit)));
        ctx->hit_cap = initial;
    }
    unsigned long long found = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        r.args.hits = ctx->d_hits;
        r.args.cap = ctx->hit_cap;
        // the rescan after a regrow is launched directly (a one-off shape)
        s = launch_run(ctx, r, nblocks, !opts->no_graph && attempt == 0);
        if (s != EPI_OK) return s;
        CK(cudaStreamSynchronize(ctx->stream));
        const unsigned long long *cnt = ctx->h_state;
        if (cnt[2] != 0)
            return set_err(ctx, EPI_E_TIMEOUT, "a bounded device wait of the scan kernel gave up (site %llu)",
                           cnt[3]);
        found = cnt[0];
        if ((int64_t)found <= ctx->hit_cap) break;
        // every hit is needed to put the first `cap` in output order: grow and rescan
        cudaFree(ctx->d_hits);
        ctx->d_hits = nullptr;
        ctx->hit_cap = 0;
        CK(cudaMalloc((void **)&ctx->d_hits, (size_t)found * sizeof(DevHit)));
        ctx->hit_cap = (int64_t)found;
    }
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms = ms;
    ctx->last_config = variant_desc(form, variant) + " (" + how + ")";
    int64_t pairs = 0;
    for (int b = 0; b < nblocks; ++b) pairs += block_pairs(blocks[b]);
    ctx->last_pairs = pairs * ctx->ntraits;

    const unsigned int *mx = reinterpret_cast<const unsigned int *>(ctx->h_state + 4);
    std::vector<DevHit> dh((size_t)found);
    if (found) {
        CK(cudaMemcpyAsync(dh.data(), ctx->d_hits, (size_t)found * sizeof(DevHit), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    for (int t = 0; t < ctx->ntraits; ++t) {
        if (max_f) max_f[t] = epi::ord2f(mx[t]);
        if (max_f2) max_f2[t] = opts->test == 'i' ? epi::ord2f(mx[ctx->ntraits + t]) : 0.0f;
    }

    // output order: (trait,) block, result slot, chunk k, chunk l, gx, gy (EpiOpenCL.c:1576-1627)
    const int L = opts->safe ? 8 : 16;
    const int chunk = opts->chunk;
    std::vector<HitKey> keys((size_t)found);
    for (size_t i = 0; i < keys.size(); ++i) {
        const DevHit &h = dh[i];
        const epi_block &b = blocks[h.block];
        HitKey &k = keys[i];
        k.trait = opts->report_trait < 0 ? h.trait : 0;
        k.block = h.block;
        k.gx = h.snp1 - b.start1;
        k.gy = h.snp2 - b.start2;
        k.s = (k.gx % L) * L + (k.gy % L);
        k.k = k.gx / chunk;
        k.l = k.gy / chunk;
        k.idx = (int64_t)i;
    }
    std::sort(keys.begin(), keys.end(), [](const HitKey &x, const HitKey &y) {
        if (x.trait != y.trait) return x.trait < y.trait;
        if (x.block != y.block) return x.block < y.block;
        if (x.s != y.s) return x.s < y.s;
        if (x.k != y.k) return x.k < y.k;
        if (x.l != y.l) return x.l < y.l;
        if (x.gx != y.gx) return x.gx < y.gx;
        return x.gy < y.gy;
    });
    const int64_t nout = std::min<int64_t>((int64_t)found, cap);
    for (int64_t i = 0; i < nout; ++i) {
        const DevHit &h = dh[(size_t)keys[(size_t)i].idx];
        hits[i].snp1 = h.snp1;
        hits[i].snp2 = h.snp2;
        hits[i].df1 = h.df1;
        hits[i].df2 = h.df2;
        hits[i].F = h.F;
        hits[i].F2 = h.F2;
        if (hit_block) hit_block[i] = h.block;
        if (hit_trait) hit_trait[i] = h.trait;
    }
    if (nhits) *nhits = (int64_t)found;
    if ((int64_t)found > cap) return set_err(ctx, EPI_E_OVERFLOW, "%llu hits, capacity %lld", found, (long long)cap);
    return EPI_OK;
}

extern "C" epi_status epi_scan_dump(epi_ctx *ctx, const epi_block *block, const epi_scan_opts *opts, int32_t trait,
                                    int32_t *counts, float *F, float *F2, int32_t *df1, int32_t *df2)
{
    if (!ctx) return EPI_E_INVALID;
    ctx->err.clear();
    if (ctx->nid == 0 || ctx->ntraits == 0) return set_err(ctx, EPI_E_STATE, "epi_scan_dump: nothing loaded");
    if (!block) return set_err(ctx, EPI_E_INVALID, "epi_scan_dump: null block");
    if (trait < 0 || trait >= ctx->ntraits) return set_err(ctx, EPI_E_INVALID, "trait out of range");
    epi_scan_opts o = *opts;
    o.report_trait = trait;
    epi_status s = check_opts(ctx, &o);
    if (s != EPI_OK) return s;
    CK(cudaSetDevice(ctx->device));
    const int form = pick_form(ctx, &o);
    int variant = 0;
    std::string how;
    s = pick_variant(ctx, &o, form, &variant, &how);
    if (s != EPI_OK) return s;
    ScanRun r;
    s = setup_run(ctx, block, 1, &o, r, variant);
    if (s != EPI_OK) return s;
    const size_t np = (size_t)block->size1 * block->size2;
    int32_t *dc = nullptr, *dd1 = nullptr, *dd2 = nullptr;
    float *dF = nullptr, *dF2 = nullptr;
    struct Out { void *host; void **dev; size_t bytes; };
    Out outs[] = {{counts, (void **)&dc, np * 9 * sizeof(int32_t)}, {F, (void **)&dF, np * sizeof(float)},
                  {F2, (void **)&dF2, np * sizeof(float)}, {df1, (void **)&dd1, np * sizeof(int32_t)},
                  {df2, (void **)&dd2, np * sizeof(int32_t)}};
    epi_status st = EPI_OK;
    for (Out &x : outs) {
        if (!x.host || !np) continue;
        cudaError_t e = cudaMalloc(x.dev, x.bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(*x.dev, x.host, x.bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) { st = set_err(ctx, EPI_E_CUDA, "dump buffers: %s", cudaGetErrorString(e)); break; }
    }
    if (st == EPI_OK) {
        r.args.dump_counts = dc;
        r.args.dump_F = dF;
        r.args.dump_F2 = dF2;
        r.args.dump_df1 = dd1;
        r.args.dump_df2 = dd2;
        r.args.hits = ctx->d_hits;
        r.args.cap = 0;
        st = launch_run(ctx, r, 1, false);
    }
    if (st == EPI_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = set_err(ctx, EPI_E_CUDA, "dump: %s", cudaGetErrorString(e));
        else if (ctx->h_state[2] != 0)
            st = set_err(ctx, EPI_E_TIMEOUT, "a bounded device wait gave up (site %llu)", ctx->h_state[3]);
    }
    if (st == EPI_OK) {
        for (Out &x : outs) {
            if (!x.host || !*x.dev) continue;
            cudaError_t e = cudaMemcpyAsync(x.host, *x.dev, x.bytes, cudaMemcpyDeviceToHost, ctx->stream);
            if (e != cudaSuccess) { st = set_err(ctx, EPI_E_CUDA, "dump readback: %s", cudaGetErrorString(e)); break; }
        }
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (st == EPI_OK && e != cudaSuccess) st = set_err(ctx, EPI_E_CUDA, "dump: %s", cudaGetErrorString(e));
    }
    for (Out &x : outs)
        if (*x.dev) cudaFree(*x.dev);
    return st;
}

extern "C" epi_status epi_scan_config(const epi_ctx *ctx, char *desc, int32_t len)
{
    if (!ctx || !desc || len < 1) return EPI_E_INVALID;
    snprintf(desc, (size_t)len, "%s", ctx->last_config.c_str());
    return EPI_OK;
}

extern "C" epi_status epi_get_stream(const epi_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return EPI_E_INVALID;
    *stream = (void *)ctx->stream;
    return EPI_OK;
}

extern "C" epi_status epi_last_timing(const epi_ctx *ctx, double *kernel_ms, int64_t *pairs, int32_t *launches,
                                      int32_t *form)
{
    if (!ctx) return EPI_E_INVALID;
    if (form) *form = ctx->last_form;
    if (kernel_ms) *kernel_ms = ctx->last_ms;
    if (pairs) *pairs = ctx->last_pairs;
    if (launches) *launches = ctx->last_launches;
    return EPI_OK;
}
