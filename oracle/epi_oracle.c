/*
 * epi_oracle.c -- TEST INFRASTRUCTURE (oracle B). Never linked into the product.
 *
 * Independent FP64 restatement of the reference's per-pair statistics, the accuracy
 * oracle for F and F2. It follows the reference's algorithm step by step but in double
 * precision and from raw genotypes, with no online mean/SS downdate:
 *
 *   unpacking         src/readplink.c:1104-1143 (MSB-first words, right-aligned tail)
 *                     = the kernel's unpacking, src/EpiOpenCL.c:110-228
 *   validity          genotype code 3 = missing on either SNP, phenotype -9 = missing
 *                     (EpiOpenCL.c:135); safe mode has no phenotype test (:597, :824)
 *   cell counts/sums  EpiOpenCL.c:140-142
 *   mean, SSY         mean and sum of squares over the valid individuals: what the
 *                     Welford-style downdate of EpiOpenCL.c:145-147 computes from the
 *                     all-individual values of EpiOpenCL.c:1367-1376
 *   SSB, d1, d2, F    EpiOpenCL.c:231-247
 *   SSI, F2           EpiOpenCL.c:452-486 (row/column means from raw sums, :466-467)
 *   hit rule          F > T1 (:251); (F > T1 || F2 > T2) && nfac > 6 (:487-489);
 *                     safe 4 df has no nfac filter (:949)
 *   output order      result slot s = (gx mod L)*L + (gy mod L) ascending (:1621), then
 *                     chunk k = gx/chunk, chunk l = gy/chunk, then gx, gy -- the order
 *                     perform_scan writes a block in for a serial execution.
 *   permutation       src/main.c:336-348 (glibc srand/rand Fisher-Yates)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef struct oracle_hit { int32_t snp1, snp2, df1, df2; double F, F2; } oracle_hit;

/* readplink.c:1104-1143: codes 0/1/2/3, one byte per genotype, SNP-major */
void oracle_unpack(const int32_t *gpack, int nid, int nsnp, int npack, int remain, uint8_t *geno)
{
    int npack1 = remain ? npack + 1 : npack;
    for (int s = 0; s < nsnp; s++) {
        const uint32_t *w = (const uint32_t *)gpack + (size_t)s * npack1;
        uint8_t *g = geno + (size_t)s * nid;
        for (int p = 0; p < npack; p++)
            for (int t = 0; t < 16; t++)
                g[16 * p + t] = (uint8_t)((w[p] >> (30 - 2 * t)) & 3u);
        for (int t = 0; t < remain; t++)
            g[16 * npack + t] = (uint8_t)((w[npack] >> (2 * (remain - 1 - t))) & 3u);
    }
}

/* readplink.c:1066-1102: the inverse (16 codes per word, first individual in bits 31:30;
 * the tail word holds `remain` codes right-aligned). */
void oracle_pack(const uint8_t *geno, int nid, int nsnp, int32_t *gpack)
{
    int npack = nid / 16, remain = nid % 16, npack1 = remain ? npack + 1 : npack;
    for (int s = 0; s < nsnp; s++) {
        const uint8_t *g = geno + (size_t)s * nid;
        uint32_t *w = (uint32_t *)gpack + (size_t)s * npack1;
        for (int p = 0; p < npack; p++) {
            uint32_t v = 0;
            for (int t = 0; t < 16; t++) v = (v << 2) | (g[16 * p + t] & 3u);
            w[p] = v;
        }
        if (remain) {
            uint32_t v = 0;
            for (int t = 0; t < remain; t++) v = (v << 2) | (g[16 * npack + t] & 3u);
            w[npack] = v;
        }
    }
}

/* One pair in FP64. Returns nfac. */
int oracle_pair(const uint8_t *g1, const uint8_t *g2, const float *phen, int nid, int safe,
                int32_t counts[9], double sums[9], double *F, double *F2, int *df1, int *df2)
{
    int64_t n[9] = {0};
    double S[9] = {0};
    int64_t N = 0;
    double St = 0;
    for (int k = 0; k < nid; k++) {
        int a = g1[k], b = g2[k];
        float y = phen[k];
        if (a != 3 && b != 3 && (safe || y != -9.0f)) {
            n[3 * a + b]++;
            S[3 * a + b] += (double)y;
            N++;
            St += (double)y;
        }
    }
    double m = St / (double)N, SSY = 0;
    for (int k = 0; k < nid; k++) {
        int a = g1[k], b = g2[k];
        float y = phen[k];
        if (a != 3 && b != 3 && (safe || y != -9.0f)) {
            double d = (double)y - m;
            SSY += d * d;
        }
    }
    int nfac = 0;
    double SSB = 0, mc[9];
    for (int c = 0; c < 9; c++) {
        mc[c] = 0;
        if (n[c] > 0) {
            nfac++;
            mc[c] = S[c] / (double)n[c];
            SSB += (double)n[c] * (mc[c] - m) * (mc[c] - m);
        }
    }
    double row[3], col[3], SSI = 0;
    for (int i = 0; i < 3; i++) {
        col[i] = (S[i] + S[i + 3] + S[i + 6]) / (double)(n[i] + n[i + 3] + n[i + 6]);
        row[i] = (S[3 * i] + S[3 * i + 1] + S[3 * i + 2]) / (double)(n[3 * i] + n[3 * i + 1] + n[3 * i + 2]);
    }
    for (int c = 0; c < 9; c++) {
        if (n[c] > 0) {
            double t = mc[c] - row[c / 3] - col[c % 3] + m;
            SSI += (double)n[c] * t * t;
        }
    }
    int d1 = nfac - 1, d2 = (int)(N - nfac);
    double MSW = (SSY - SSB) / (double)d2;
    *F = (SSB / (double)d1) / MSW;
    *F2 = (SSI / 4.0) / MSW;
    *df1 = d1;
    *df2 = d2;
    for (int c = 0; c < 9; c++) {
        if (counts) counts[c] = (int32_t)n[c];
        if (sums) sums[c] = S[c];
    }
    return nfac;
}

typedef struct { int32_t s, k, l, gx, gy; oracle_hit h; } okey_hit;

static int okey_cmp(const void *a, const void *b)
{
    const okey_hit *x = (const okey_hit *)a, *y = (const okey_hit *)b;
    if (x->s != y->s) return x->s < y->s ? -1 : 1;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    if (x->l != y->l) return x->l < y->l ? -1 : 1;
    if (x->gx != y->gx) return x->gx < y->gx ? -1 : 1;
    if (x->gy != y->gy) return x->gy < y->gy ? -1 : 1;
    return 0;
}

/*
 * All pairs of block [chr1g, chr1g+chr1m) x [chr2g, chr2g+chr2m) with global
 * snp1 > snp2 (EpiOpenCL.c:97-98). `geno` is the unpacked genome (nsnp x nid).
 * Hits go to `hits` (first cap, output order); returns the hit count. Optional
 * per-pair outputs in (gx*chr2m + gy) layout: counts (9 each), F, F2, df1, df2;
 * untouched for pairs outside the triangle.
 */
int64_t oracle_scan_block(int test, int safe, int chunk, const uint8_t *geno, int nid,
                          const float *phen, float t1, float t2,
                          int chr1g, int chr1m, int chr2g, int chr2m,
                          oracle_hit *hits, int64_t cap,
                          int32_t *out_counts, double *out_F, double *out_F2,
                          int32_t *out_df1, int32_t *out_df2)
{
    const int L = safe ? 8 : 16;
    const size_t np = (size_t)chr1m * (size_t)chr2m;
    /* pass 1, rows in parallel: every pair's statistics (into the caller's arrays, or
     * scratch ones); pass 2, serial: the hit rule and the output order */
    double *pF = out_F ? out_F : (double *)malloc(sizeof(double) * (np ? np : 1));
    double *pF2 = out_F2 ? out_F2 : (double *)malloc(sizeof(double) * (np ? np : 1));
    int32_t *pd1 = out_df1 ? out_df1 : (int32_t *)malloc(sizeof(int32_t) * (np ? np : 1));
    int32_t *pd2 = out_df2 ? out_df2 : (int32_t *)malloc(sizeof(int32_t) * (np ? np : 1));
#pragma omp parallel for schedule(dynamic, 1)
    for (int gx = 0; gx < chr1m; gx++) {
        for (int gy = 0; gy < chr2m; gy++) {
            if (!(gx + chr1g > gy + chr2g)) continue;
            int32_t cnt[9];
            double F, F2;
            int d1, d2;
            oracle_pair(geno + (size_t)(gx + chr1g) * nid, geno + (size_t)(gy + chr2g) * nid, phen, nid, safe, cnt,
                        NULL, &F, &F2, &d1, &d2);
            size_t o = (size_t)gx * chr2m + gy;
            if (out_counts) memcpy(out_counts + 9 * o, cnt, sizeof(cnt));
            pF[o] = F;
            pF2[o] = F2;
            pd1[o] = d1;
            pd2[o] = d2;
        }
    }
    int64_t nh = 0, capk = 1024;
    okey_hit *kh = (okey_hit *)malloc(sizeof(okey_hit) * (size_t)capk);
    for (int gx = 0; gx < chr1m; gx++) {
        for (int gy = 0; gy < chr2m; gy++) {
            if (!(gx + chr1g > gy + chr2g)) continue;
            size_t o = (size_t)gx * chr2m + gy;
            const double F = pF[o], F2 = pF2[o];
            const int d1 = pd1[o], d2 = pd2[o], nfac = d1 + 1;
            int hit;
            if (test == 'f') hit = F > (double)t1;
            else hit = (F > (double)t1 || F2 > (double)t2) && (safe || nfac > 6);
            if (!hit) continue;
            if (nh == capk) {
                capk *= 2;
                kh = (okey_hit *)realloc(kh, sizeof(okey_hit) * (size_t)capk);
            }
            okey_hit *e = &kh[nh++];
            e->s = (gx % L) * L + (gy % L);
            e->k = gx / chunk;
            e->l = gy / chunk;
            e->gx = gx;
            e->gy = gy;
            e->h.snp1 = gx + chr1g;
            e->h.snp2 = gy + chr2g;
            e->h.df1 = d1;
            e->h.df2 = d2;
            e->h.F = F;
            e->h.F2 = (test == 'f') ? 0.0 : F2;
        }
    }
    qsort(kh, (size_t)nh, sizeof(okey_hit), okey_cmp);
    for (int64_t i = 0; i < nh && i < cap; i++) hits[i] = kh[i].h;
    free(kh);
    if (!out_F) free(pF);
    if (!out_F2) free(pF2);
    if (!out_df1) free(pd1);
    if (!out_df2) free(pd2);
    return nh;
}

/* main.c:336-348 applied to a phenotype vector (the ped records carry the phenotype). */
void oracle_permute(float *phen, int nid, unsigned int seed)
{
    srand(seed);
    for (int i = nid; i > 1; i--) {
        int r = rand() % i;
        float t = phen[r];
        phen[r] = phen[i - 1];
        phen[i - 1] = t;
    }
}
