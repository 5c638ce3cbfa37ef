/*
 * epigpu.h -- C ABI of libepigpu.so, the B200 (sm_100a) exhaustive pairwise epistasis
 * scan.
 *
 * It replaces the device side of epiGPU's scan: the OpenCL pair kernels of
 * src/EpiOpenCL.c:45-963 and the platform/buffer/launch/readback code of perform_scan
 * (src/EpiOpenCL.c:1383-1436, :1473-1627). The host program keeps epiGPU's CLI, its
 * .epigpu input and its results file (the C host program in epigpu_b200/host). Only plain C types cross
 * this boundary: host pointers and sizes, no CUDA or torch types.
 *
 * Conventions
 *  - Every entry point returns an epi_status; none calls exit(). The reference exits
 *    through ereport() on any OpenCL error (src/EpiOpenCL.c:1159-1177); the host CLI
 *    keeps that behaviour on top of these codes.
 *  - The caller owns every host buffer. The library owns its device memory.
 *  - One context per host thread; a context is not thread-safe.
 *  - SNP indices are 0-based and global (position in the .epigpu SNP order), as in the
 *    reference's result rows before the +1 of the results file (EpiOpenCL.c:1633).
 */
#ifndef EPIGPU_H
#define EPIGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPI_ABI_VERSION 1

typedef enum epi_status {
    EPI_OK = 0,
    EPI_E_INVALID = 1,      /* bad argument (message in epi_last_error) */
    EPI_E_CUDA = 2,         /* CUDA runtime error */
    EPI_E_NOMEM = 3,        /* device allocation failed */
    EPI_E_OVERFLOW = 4,     /* more hits than `cap`: *nhits holds the total, `cap` rows written */
    EPI_E_STATE = 5,        /* genotypes or phenotypes not loaded yet */
    EPI_E_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    EPI_E_NODEVICE = 7,     /* no usable CUDA device at that index (ereport, EpiOpenCL.c:1161) */
    EPI_E_UNSUPPORTED = 8   /* option combination not supported by the selected form */
} epi_status;

typedef struct epi_ctx epi_ctx;

/* One result row: the reference's `table` struct (src/id4117.h:14-21), 24 bytes.
 * F2 is 0 in the 8 df test (EpiOpenCL.c:261). */
typedef struct epi_hit {
    int32_t snp1, snp2, df1, df2;
    float F, F2;
} epi_hit;

/* A chromosome x chromosome block: SNP1 in [start1, start1+size1), SNP2 in
 * [start2, start2+size2). Pairs are tested when snp1 > snp2 (EpiOpenCL.c:97-98);
 * perform_scan visits blocks (i, j <= i) (EpiOpenCL.c:1527-1540). */
typedef struct epi_block {
    int32_t start1, size1, start2, size2;
} epi_block;

enum { EPI_FORM_AUTO = 0, EPI_FORM_POPC = 1, EPI_FORM_TENSOR = 2 };

/* Scan options: the analysis-mode flags of src/main.c:58-188 that reach the kernel. */
typedef struct epi_scan_opts {
    int32_t test;          /* 'f' = 8 df test, 'i' = 8 df + 4 df test (-t) */
    int32_t safe;          /* -s: 1 = safe-mode rules (no nfac>6 filter in 'i', 8x8 slots) */
    int32_t chunk;         /* -i iteration size (multiple of 16): only changes the output order */
    float t1;              /* -F threshold for F (8 df) */
    float t2;              /* -I threshold for F2 (4 df) */
    int32_t form;          /* EPI_FORM_AUTO / _POPC (plain popcount form, up to 65,535 individuals)
                            * / _TENSOR (tcgen05, up to 2^24 individuals); AUTO takes the tensor
                            * form from 256 individuals on */
    int32_t report_trait;  /* trait whose hits are returned; -1 = every trait */
    int32_t wait_limit_ms; /* tensor form: every device-side wait gives up after this many
                            * milliseconds and the scan returns EPI_E_TIMEOUT; 0 = 2000 */
    int32_t debug;         /* 0; EPI_DEBUG_STALL (tests of the timeout path only): one wait of
                            * the tensor form is on a barrier nothing arrives at, so it runs
                            * out after wait_limit_ms and the scan returns EPI_E_TIMEOUT */
    int32_t no_graph;      /* 0: the scan's device work is captured as a CUDA graph and a repeat of
                            * the same scan shape (kernel arguments, blocks) replays it with one
                            * launch; 1: every operation is launched directly */
    int32_t tile_config;   /* 0: the kernel variant (plain form: tile shape, 3 candidates;
                            * tensor form: ring depths, epilogue warps, producer groups and
                            * streamed B, 6 candidates, streamed B only up to 6,144 padded
                            * individuals) is chosen by the autotuner, which times every
                            * candidate on a sample block once per device, form, individual
                            * count and trait count; k >= 1: candidate k (epi_scan_config
                            * names it) */
    int32_t reserved[5];   /* set to 0 */
} epi_scan_opts;

#define EPI_DEBUG_STALL 1

/* Fills `o` with the reference defaults: 'f', normal mode, chunk 128, F 6.5, I 10.5
 * (src/main.c:244-249), AUTO form, trait 0. */
void epi_default_opts(epi_scan_opts *o);

/* Replaces the OpenCL platform/device/context/queue set-up of perform_scan
 * (src/EpiOpenCL.c:1383-1481); `device` is the -d index (src/main.c:132-143). */
epi_status epi_open(int32_t device, epi_ctx **out);
epi_status epi_close(epi_ctx *ctx);

const char *epi_strerror(epi_status s);
/* Message of the last error on this context ("" if none). */
const char *epi_last_error(const epi_ctx *ctx);
/* Device name and SM count of the context's GPU. */
epi_status epi_device_info(const epi_ctx *ctx, char *name, int32_t name_len, int32_t *sm_count);

/*
 * Genotypes in the reference's packed layout (src/readplink.c:1066-1102, read by
 * readpackedbinary, :1183-1273): nsnp rows of npack1 = npack + (remain > 0) int32
 * words; 16 codes per full word, first individual in bits 31:30; the tail word holds
 * `remain` codes right-aligned. Codes 0/1/2, 3 = missing. Replaces the per-chromosome
 * uploads g_chr1/g_chr2 (EpiOpenCL.c:1530-1545): the whole genome is kept on the GPU as
 * 2-bit code rows and genotype bit-planes built on the device.
 */
epi_status epi_load_packed(epi_ctx *ctx, const int32_t *gpack, int32_t nid, int32_t nsnp,
                           int32_t npack, int32_t remain);

/*
 * Phenotype columns ("traits"), column-major nid x ntraits floats. `valid` (nullable,
 * nid x ntraits bytes, column-major) marks usable values; when NULL a value of -9 is
 * missing (EpiOpenCL.c:135). Replaces g_phen, mY and SSY (EpiOpenCL.c:1364-1376,
 * :1507-1515). Safe mode (-s 1) uses -9 as a value: pass an all-ones `valid`.
 */
epi_status epi_set_traits(epi_ctx *ctx, const float *y, int32_t nid, int32_t ntraits,
                          const uint8_t *valid);

/* One trait; safe != 0 uses every value (no -9 test, EpiOpenCL.c:597). */
epi_status epi_set_phenotype(epi_ctx *ctx, const float *phen, int32_t nid, int32_t safe);

/*
 * Scans every pair of the given blocks for the loaded traits and returns the pairs
 * above threshold -- the hit test of EpiOpenCL.c:251 ('f') or :487-489 ('i';
 * :949 in safe mode) -- in the order perform_scan writes them: block by block in the
 * given order, inside a block by result slot (EpiOpenCL.c:1621), then chunk and
 * work-group order (trait-major first when several traits are reported).
 * Replaces the chunk loop, launches and hit readback of EpiOpenCL.c:1527-1627.
 *
 *   hits, cap    output rows (may be NULL when cap == 0 to count only)
 *   nhits        total number of hits (even beyond cap -> EPI_E_OVERFLOW)
 *   hit_block    nullable, cap entries: index into `blocks` of each row
 *   hit_trait    nullable, cap entries: trait of each row
 *   max_f        nullable, ntraits entries: largest 8 df F over all scanned pairs
 *   max_f2       nullable, ntraits entries: largest 4 df F2 (test 'i' only)
 */
epi_status epi_scan(epi_ctx *ctx, const epi_block *blocks, int32_t nblocks,
                    const epi_scan_opts *opts, epi_hit *hits, int64_t cap, int64_t *nhits,
                    int32_t *hit_block, int32_t *hit_trait, float *max_f, float *max_f2);

/*
 * Per-pair statistics of one block for one trait, from the same kernels as epi_scan
 * (a test and inspection aid). Outputs are size1 x size2 arrays, pair (gx, gy) at
 * gx*size2 + gy; pairs with snp1 <= snp2 are left untouched. counts: 9 cells per pair,
 * cell 3*g1 + g2 (EpiOpenCL.c:140). Any output may be NULL.
 */
epi_status epi_scan_dump(epi_ctx *ctx, const epi_block *block, const epi_scan_opts *opts,
                         int32_t trait, int32_t *counts, float *F, float *F2,
                         int32_t *df1, int32_t *df2);

/* Device time of the last epi_scan's pair kernels (CUDA events on the scan stream),
 * the pair tests they made (pairs x traits), how many kernels were launched and which
 * form ran (EPI_FORM_POPC or EPI_FORM_TENSOR). Any output may be NULL. */
epi_status epi_last_timing(const epi_ctx *ctx, double *kernel_ms, int64_t *pairs,
                           int32_t *launches, int32_t *form);

/* The form and kernel variant the last epi_scan ran, and how the variant was chosen (the
 * autotuner's timings of every candidate, or "requested"), as text. No counterpart in the
 * reference, whose only tuning knob is the chunk size of its launches (src/main.c:115-130). */
epi_status epi_scan_config(const epi_ctx *ctx, char *desc, int32_t len);

/* The context's CUDA stream (a cudaStream_t, returned as an opaque pointer): every copy
 * and kernel of the context runs on it, so a caller can order or time its own work
 * against the scan. */
epi_status epi_get_stream(const epi_ctx *ctx, void **stream);

/*
 * Allocation-free scan of one block (no counterpart in the reference).
 *
 * For callers that cannot allocate GPU memory while they run: a service or real-time loop
 * that forbids cudaMalloc after start-up, or a host framework that hands out device memory
 * only from its own pool. Every input and output is a device buffer the caller owns; the
 * call makes no cudaMalloc, cudaFree or other allocating call. The plain popcount form
 * runs on the calling thread's current device, on `stream` (a cudaStream_t; NULL = the
 * default stream), and the call returns once the scan has finished.
 *
 *   d_gpack  device, nsnp x (nid/16 + (nid%16 > 0)) int32: the reference's packed words
 *   d_phen   device, nid floats; -9 = missing unless opts->safe
 *   block    the pairs to scan (snp1 in block 1 > snp2 in block 2), as for epi_scan
 *   opts     test, safe, t1, t2 as for epi_scan (form and chunk are ignored)
 *   d_hits   device, cap rows: the hits, in no particular order (epi_scan gives the
 *            reference's order; sort by (snp1, snp2) to compare)
 *   d_nhits  device, one int64: the number of hits; when it exceeds cap the first cap
 *            rows are written and the call returns EPI_E_OVERFLOW, as epi_scan does
 *   d_maxf   device, nullable, 2 floats: largest F and F2 over the block
 *
 * Working memory is a fixed array of about 520 KiB in this library, one per device, held
 * until the process exits: it limits nid to EPI_NOALLOC_MAX_NID (larger returns
 * EPI_E_UNSUPPORTED). The first call on each device does that device's set-up (device
 * check, SM count, kernel attribute). No call may be made while `stream` is being captured
 * into a CUDA graph: every call copies the hit count to the host and synchronises.
 * Every call looks up the array's device address for the current device. All calls on a
 * device share the array and each call clears what it needs, so results never carry over,
 * but calls that overlap on the GPU (other host threads, other streams) race and must be
 * serialised by the caller. The call waits for the scan to finish (it synchronises
 * `stream`) before it returns. A CUDA error already pending from the caller's earlier work
 * makes it return EPI_E_CUDA at once, leaving that error pending.
 */
#define EPI_NOALLOC_MAX_NID 65535
epi_status epi_scan_block_noalloc(const int32_t *d_gpack, int32_t nid, int32_t nsnp,
                                  const float *d_phen, const epi_block *block,
                                  const epi_scan_opts *opts, epi_hit *d_hits, int64_t cap,
                                  int64_t *d_nhits, float *d_maxf, void *stream);

/* The permutation of src/main.c:336-348 applied to a phenotype vector: srand(seed), then
 * glibc rand() Fisher-Yates from the end. Matches `epiGPU -A ... -p seed`. */
void epi_permute_phenotype(float *phen, int32_t nid, uint32_t seed);

#ifdef __cplusplus
}
#endif

#endif /* EPIGPU_H */
