/*
 * ndrange_emu.c -- TEST INFRASTRUCTURE (oracle A). Never linked into the product.
 *
 * Drives the reference's own OpenCL pair kernels, extracted at build time from
 * src/EpiOpenCL.c:45-963 and compiled as C (ref_prelude.h, build_ref.py), through an
 * emulation of perform_scan's launch loop (src/EpiOpenCL.c:1540-1607):
 *
 *   - work-group 16x16, or 8x8 in safe mode (EpiOpenCL.c:1353-1362);
 *   - global size rounded up to the work-group (EpiOpenCL.c:1559-1560);
 *   - chunk x chunk launches, chunk l <= k on a diagonal block (EpiOpenCL.c:1564-1607);
 *   - kernel arguments 0-20 exactly as perform_scan sets them (EpiOpenCL.c:1512-1596).
 *
 * Each work-group runs with freshly zeroed hit counters, so every result slot holds at
 * most one hit per group and nothing overflows the reference's 200-row slots
 * (EpiOpenCL.c:255). Hits are then put in the order perform_scan writes them for a
 * serial execution: result slot s = lx*L + ly ascending (EpiOpenCL.c:1621), then launch
 * (chunk k, chunk l), then work-group (x-major). Running the launches on several threads
 * therefore gives the same output as running them on one.
 *
 * The phenotype mean/sum of squares are computed as perform_scan does it
 * (EpiOpenCL.c:1367-1376), in float, over all individuals including -9 values.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "ref_prelude.h"
#ifdef _OPENMP
#include <omp.h>
#endif

__thread size_t epi_emu_global_id[2];
__thread size_t epi_emu_local_id[2];
__thread size_t epi_emu_local_size[2];
__thread size_t epi_emu_global_size[2];

/* the reference's result row, src/id4117.h:14-21 (24 bytes) */
typedef struct table { int snp1, snp2, df1, df2; float F, F2; } table;

#define KARGS_HEAD int *gchr1, int *gchr2, const float *phen, table *results, \
    const float mY, const float SSY, const float threshold1, const float threshold2, \
    const int nid, const int nsnp, const int npack, const int remain, float *mY_fac
#define KARGS_TAIL int *nhits, const int chr1, const int chr2, const int chr1g, \
    const int chr2g, const int chr1m, const int chr2m

void ref_kernelfull(KARGS_HEAD, unsigned short *factor_count, KARGS_TAIL);
void ref_kernelint(KARGS_HEAD, unsigned short *factor_count, KARGS_TAIL);
void ref_kernelfullsafe(KARGS_HEAD, unsigned int *factor_count, KARGS_TAIL);
void ref_kernelintsafe(KARGS_HEAD, unsigned int *factor_count, KARGS_TAIL);

#define SLOT_ROWS 200  /* MAX2, src/id4117.h:9 */

typedef struct { int32_t s, k, l, gx, gy; table t; } keyed_hit;

typedef struct { keyed_hit *v; int64_t n, cap; } hit_list;

static void list_push(hit_list *L, const keyed_hit *h)
{
    if (L->n == L->cap) {
        L->cap = L->cap ? 2 * L->cap : 1024;
        L->v = (keyed_hit *)realloc(L->v, (size_t)L->cap * sizeof(keyed_hit));
    }
    L->v[L->n++] = *h;
}

static int cmp_key(const void *a, const void *b)
{
    const keyed_hit *x = (const keyed_hit *)a, *y = (const keyed_hit *)b;
    if (x->s != y->s) return x->s < y->s ? -1 : 1;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    if (x->l != y->l) return x->l < y->l ? -1 : 1;
    if (x->gx != y->gx) return x->gx < y->gx ? -1 : 1;
    if (x->gy != y->gy) return x->gy < y->gy ? -1 : 1;
    return 0;
}

/* EpiOpenCL.c:1364-1376: float mean and sum of squares over all nid values */
void ref_phen_stats(const float *phen, int nid, float *mY_out, float *SSY_out)
{
    float mY = 0, SSY = 0;
    int i;
    for (i = 0; i < nid; i++) mY += phen[i];
    mY /= nid;
    for (i = 0; i < nid; i++) SSY += (phen[i] - mY) * (phen[i] - mY);
    *mY_out = mY;
    *SSY_out = SSY;
}

typedef struct { int k, l, chr1, chr2, w0, w1; } launch_t;

/*
 * Scans chromosome block (i, j) -- SNPs [chr1g, chr1g+chr1m) x [chr2g, chr2g+chr2m) --
 * as perform_scan does for one iteration of its `for(j ...)` loop. `same_chr` is (i == j).
 * Returns the total number of hits; writes the first `cap` of them, in output order, to
 * `hits` with global 0-based SNP indices (the 4 df kernels store chromosome-local
 * indices, which the reference host shifts back, EpiOpenCL.c:1644-1648).
 * Optional dumps (chr1m*chr2m*9 entries, pair (gx,gy) at (gx*chr2m+gy)*9): the cell counts
 * and the float cell values the kernel leaves in local memory (cell means where the count
 * is positive), written only for pairs the kernel computes.
 */
int64_t ref_scan_block(int test, int safe, int chunk,
                       const int32_t *geno, int npack, int remain, int nid,
                       const float *phen, float mY, float SSY, float t1, float t2,
                       int chr1g, int chr1m, int chr2g, int chr2m, int same_chr,
                       table *hits, int64_t cap,
                       uint32_t *dump_counts, float *dump_means, int nthreads)
{
    const int L = safe ? 8 : 16;
    const int npack1 = remain ? npack + 1 : npack;
    int *g1 = (int *)(geno + (size_t)npack1 * chr1g);
    int *g2 = (int *)(geno + (size_t)npack1 * chr2g);
    size_t gws0 = (size_t)ceil((double)chr1m / L) * L;
    size_t gws1 = (size_t)ceil((double)chr2m / L) * L;
    int nit0 = (int)ceil((double)gws0 / chunk), nit1 = (int)ceil((double)gws1 / chunk);
    launch_t *launches = (launch_t *)malloc(sizeof(launch_t) * (size_t)nit0 * nit1 + 1);
    int nl = 0, k, l;
    int64_t total = 0, i;

    for (k = 0; k < nit0; k++) {
        int flag = same_chr ? k + 1 : nit1;
        int w0 = (k == nit0 - 1 && gws0 % chunk) ? (int)(gws0 % chunk) : chunk;
        for (l = 0; l < flag; l++) {
            int w1 = (l == nit1 - 1 && gws1 % chunk) ? (int)(gws1 % chunk) : chunk;
            launch_t la = { k, l, k * chunk, l * chunk, w0, w1 };
            launches[nl++] = la;
        }
    }

    if (nthreads < 1) nthreads = 1;
    hit_list *lists = (hit_list *)calloc((size_t)nthreads, sizeof(hit_list));

#pragma omp parallel num_threads(nthreads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        float *mY_fac = (float *)calloc((size_t)L * L * 9, sizeof(float));
        unsigned short *fc16 = (unsigned short *)calloc((size_t)L * L * 9, sizeof(unsigned short));
        unsigned int *fc32 = (unsigned int *)calloc((size_t)L * L * 9, sizeof(unsigned int));
        int *nh = (int *)calloc((size_t)L * L, sizeof(int));
        table *res = (table *)calloc((size_t)SLOT_ROWS * L * L, sizeof(table));
        int li;
#pragma omp for schedule(dynamic, 1)
        for (li = 0; li < nl; li++) {
            launch_t la = launches[li];
            int gx0, gy0, lx, ly;
            epi_emu_local_size[0] = epi_emu_local_size[1] = (size_t)L;
            epi_emu_global_size[0] = (size_t)la.w0;
            epi_emu_global_size[1] = (size_t)la.w1;
            for (gx0 = 0; gx0 < la.w0; gx0 += L) {
                for (gy0 = 0; gy0 < la.w1; gy0 += L) {
                    memset(nh, 0, sizeof(int) * (size_t)L * L);
                    for (lx = 0; lx < L; lx++) {
                        for (ly = 0; ly < L; ly++) {
                            int gx = gx0 + lx + la.chr1, gy = gy0 + ly + la.chr2;
                            epi_emu_global_id[0] = (size_t)(gx0 + lx);
                            epi_emu_global_id[1] = (size_t)(gy0 + ly);
                            epi_emu_local_id[0] = (size_t)lx;
                            epi_emu_local_id[1] = (size_t)ly;
                            if (test == 'f' && !safe)
                                ref_kernelfull(g1, g2, phen, res, mY, SSY, t1, t2, nid, 0, npack, remain,
                                               mY_fac, fc16, nh, la.chr1, la.chr2, chr1g, chr2g, chr1m, chr2m);
                            else if (test == 'f')
                                ref_kernelfullsafe(g1, g2, phen, res, mY, SSY, t1, t2, nid, 0, npack, remain,
                                                   mY_fac, fc32, nh, la.chr1, la.chr2, chr1g, chr2g, chr1m, chr2m);
                            else if (!safe)
                                ref_kernelint(g1, g2, phen, res, mY, SSY, t1, t2, nid, 0, npack, remain,
                                              mY_fac, fc16, nh, la.chr1, la.chr2, chr1g, chr2g, chr1m, chr2m);
                            else
                                ref_kernelintsafe(g1, g2, phen, res, mY, SSY, t1, t2, nid, 0, npack, remain,
                                                  mY_fac, fc32, nh, la.chr1, la.chr2, chr1g, chr2g, chr1m, chr2m);
                            if ((dump_counts || dump_means) && gx + chr1g > gy + chr2g && gx < chr1m && gy < chr2m) {
                                int lad = 9 * (lx * L + ly), c;
                                size_t o = ((size_t)gx * chr2m + gy) * 9;
                                for (c = 0; c < 9; c++) {
                                    if (dump_counts) dump_counts[o + c] = safe ? fc32[lad + c] : fc16[lad + c];
                                    if (dump_means) dump_means[o + c] = mY_fac[lad + c];
                                }
                            }
                        }
                    }
                    for (lx = 0; lx < L; lx++) {
                        for (ly = 0; ly < L; ly++) {
                            int s = lx * L + ly;
                            if (nh[s]) {
                                keyed_hit h;
                                h.s = s; h.k = la.k; h.l = la.l;
                                h.gx = gx0 + lx + la.chr1; h.gy = gy0 + ly + la.chr2;
                                h.t = res[SLOT_ROWS * s];
                                if (test != 'f') { h.t.snp1 += chr1g; h.t.snp2 += chr2g; }
                                list_push(&lists[tid], &h);
                            }
                        }
                    }
                }
            }
        }
        free(mY_fac); free(fc16); free(fc32); free(nh); free(res);
    }

    for (k = 0; k < nthreads; k++) total += lists[k].n;
    {
        keyed_hit *all = (keyed_hit *)malloc(sizeof(keyed_hit) * (size_t)(total + 1));
        int64_t off = 0;
        for (k = 0; k < nthreads; k++) {
            if (lists[k].n) memcpy(all + off, lists[k].v, sizeof(keyed_hit) * (size_t)lists[k].n);
            off += lists[k].n;
            free(lists[k].v);
        }
        qsort(all, (size_t)total, sizeof(keyed_hit), cmp_key);
        for (i = 0; i < total && i < cap; i++) hits[i] = all[i].t;
        free(all);
    }
    free(lists);
    free(launches);
    return total;
}

/* Number of pairs the kernel computes in a block (the reference's triangle/square). */
int64_t ref_block_pairs(int chr1g, int chr1m, int chr2g, int chr2m)
{
    int64_t n = 0;
    int gx;
    for (gx = 0; gx < chr1m; gx++) {
        int64_t lim = (int64_t)gx + chr1g - chr2g;  /* gy < lim */
        if (lim > chr2m) lim = chr2m;
        if (lim > 0) n += lim;
    }
    return n;
}
