/*
 * scan_driver.c -- perform_scan on the B200: the drop-in for src/EpiOpenCL.c:1312-1686.
 *
 * Same signature, same globals, same results file:
 *   header (EpiOpenCL.c:1459-1470), then per chromosome block (i, j <= i) in order a line
 *   "# i x j : n interactions" (:1618) and n rows (:1632-1653):
 *     SNP1 (1-based) SNP1name Chr1 SNP2 SNP2name Chr2 df1 df2 F [F2]
 * and the same checkpoint/resume rule: an existing results file is validated against the
 * data and the scan restarts after its last complete block (resume, :1187-1274).
 * The OpenCL set-up, buffers and chunk launches are replaced by libepigpu.so: all the
 * remaining blocks go to the GPU in batches, each batch in one persistent launch; every
 * block's section is appended as soon as its batch returns.
 *
 * Differences from the reference, on purpose:
 *  - a resumed scan restarts at column s2 only in row s1; the reference starts every later
 *    row at s2 as well (EpiOpenCL.c:1540) and so skips blocks (i > s1, j < s2);
 *  - hits are counted with atomics and returned in the reference's serial order instead
 *    of 200-row slots written without synchronisation (EpiOpenCL.c:253-255), so no hit is
 *    lost or overwritten whatever the count;
 *  - a results file cut inside a block (interrupted write) is truncated back to the end of
 *    its last complete block before the scan resumes; the reference appends after the
 *    partial rows;
 *  - errors print the library's message and exit with its status (ereport, :1159-1177).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "epigpu_host.h"

#define PAIR_BATCH ((long long)1 << 34) /* pairs per launch batch between checkpoints */

/* Settings this scan driver adds to the reference's globals (src/epiopencl.h:9-16, which the
 * caller's main.c defines). They are defined here, with their defaults, so that the
 * reference's own main.c links against this file unchanged: the GPU form (-g), the
 * permutation-threshold count (-N) and the reference's resume rule (-R). */
int UFORM = EPI_FORM_AUTO;
int UNPERM = 0;
int UREFRESUME = 0;

static void fail(epi_ctx *ctx, epi_status st, const char *what)
{
    if (st == EPI_E_NODEVICE) {
        printf("\n\nError:\nThere is no suitable GPU on this computer.\nThis program requires an NVIDIA B200 "
               "(sm_100a) device; -d selects it.\n\n");
        exit(1);
    }
    printf("\n\nThere was an error.\n%s: %s\n%s\n", what, epi_strerror(st), ctx ? epi_last_error(ctx) : "");
    exit((int)st);
}

/* src/EpiOpenCL.c:1187-1274. Returns 0 = fresh start, 1 = resume, exits on mismatch. */
int resume_point(const char *filename, int *chr1, int *chr2, int *tothits, int nid, int nsnp)
{
    char line[512], name[300];
    int v = 0, c1 = 0, c2 = 0, k = 0, blocks = 0;
    float th1 = 0, th2 = 0;
    char x = 0;
    *chr1 = *chr2 = 0;
    FILE *in = fopen(filename, "rt");
    if (!in) return 0;
    name[0] = 0;
    if (!fgets(line, sizeof(line), in) || sscanf(line, "Datafile: %299s", name) != 1 || strcmp(name, plinkbin) != 0) {
        printf("Can't resume analysis with different datafile!\n");
        exit(1);
    }
    if (!fgets(line, sizeof(line), in) || sscanf(line, "Number of individuals: %d", &v) != 1 || v != nid) {
        printf("Can't resume analysis with different data!\n");
        exit(1);
    }
    if (!fgets(line, sizeof(line), in) || sscanf(line, "Number of SNPs: %d", &v) != 1 || v != nsnp) {
        printf("Can't resume analysis with different data!\n");
        exit(1);
    }
    if (!fgets(line, sizeof(line), in) || sscanf(line, "Permutation: %d", &v) != 1 || v != UPERM) {
        printf("Can't resume analysis with different permutation!\n");
        exit(1);
    }
    if (fgets(line, sizeof(line), in) && sscanf(line, "Threshold: %f %f", &th1, &th2) == 2) {
        if (th1 != UTHRESHOLD1)
            printf("Warning: Resuming analysis with different full threshold, changed from %f to %f\n", th1,
                   UTHRESHOLD1);
        if (th2 != UTHRESHOLD2)
            printf("Warning: Resuming analysis with different interaction threshold, changed from %f to %f\n", th2,
                   UTHRESHOLD2);
    }
    if (!fgets(line, sizeof(line), in) || sscanf(line, "Test: %c", &x) != 1 || x != UTEST) {
        printf("Can't resume analysis performing a different test!\n");
        exit(1);
    }
    if (!fgets(line, sizeof(line), in) || !fgets(line, sizeof(line), in)) { /* blank line, column names */
        fclose(in);
        return 1;
    }
    /* count complete blocks: a block header followed by all of its rows */
    long good_end = ftell(in);
    while (fgets(line, sizeof(line), in)) {
        int a, b, n;
        if (sscanf(line, "# %d x %d : %d interactions", &a, &b, &n) != 3) break;
        int rows = 0;
        while (rows < n && fgets(line, sizeof(line), in)) ++rows;
        if (rows < n) break; /* a block cut short is rescanned */
        c1 = a;
        c2 = b;
        k = n;
        *tothits += k;
        ++blocks;
        good_end = ftell(in);
    }
    fseek(in, 0, SEEK_END);
    const long size = ftell(in);
    fclose(in);
    if (blocks && size > good_end && truncate(filename, good_end) != 0) {
        printf("Cannot truncate the partial block at the end of %s\n", filename);
        exit(1);
    }
    if (blocks) {
        if (c1 == c2) {
            *chr1 = c1 + 1;
            *chr2 = 0;
        } else {
            *chr1 = c1;
            *chr2 = c2 + 1;
        }
    }
    return 1;
}

/* EpiOpenCL.c:1459-1470 */
static void write_header_full(const char *filename, int nid, int nsnp)
{
    FILE *out = fopen(filename, "wt");
    if (!out) {
        printf("Cannot write %s\n", filename);
        exit(1);
    }
    fprintf(out, "Datafile: %s %s\n", plinkbin, UPHEN);
    fprintf(out, "Number of individuals: %d\nNumber of SNPs: %d\nPermutation: %d\nThreshold: %f %f\n", nid, nsnp,
            UPERM, UTHRESHOLD1, UTHRESHOLD2);
    if (UTEST == 'f') {
        fprintf(out, "Test: full\n\n");
        fprintf(out, "SNP1\tSNP1name\tChr1\tSNP2\tSNP2name\tChr2\tdf1\tdf2\tFval\n");
    } else {
        fprintf(out, "Test: interactions + full\n\n");
        fprintf(out, "SNP1\tSNP1name\tChr1\tSNP2\tSNP2name\tChr2\tdf1\tdf2\tFval\tFint\n");
    }
    fclose(out);
}

static int cmp_float(const void *a, const void *b)
{
    const float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

/* Empirical family-wise threshold at level alpha: the ceil((1 - alpha) K)-th smallest of the
 * K permutation maxima (sorted ascending). */
static float fw_threshold(const float *sorted, int K, double alpha)
{
    int k = (int)ceil((1.0 - alpha) * K);
    if (k < 1) k = 1;
    if (k > K) k = K;
    return sorted[k - 1];
}

/* <filename>.perm: the largest F (and F2) over all pairs of every permuted phenotype, the
 * family-wise thresholds they give, and the family-wise p-value of the observed largest F. */
static void write_permutation_summary(const char *filename, int ntraits, const float *maxf, const float *maxf2)
{
    const int K = ntraits - 1;
    char fn[1200];
    snprintf(fn, sizeof(fn), "%s.perm", filename);
    FILE *f = fopen(fn, "w");
    if (!f) {
        printf("Cannot write %s\n", fn);
        exit(1);
    }
    float *s1 = (float *)malloc(sizeof(float) * (size_t)K), *s2 = (float *)malloc(sizeof(float) * (size_t)K);
    int above = 0, above2 = 0;
    for (int p = 0; p < K; p++) {
        s1[p] = maxf[p + 1];
        s2[p] = maxf2[p + 1];
        above += s1[p] >= maxf[0];
        above2 += s2[p] >= maxf2[0];
    }
    qsort(s1, (size_t)K, sizeof(float), cmp_float);
    qsort(s2, (size_t)K, sizeof(float), cmp_float);
    const int inter = UTEST == 'i';
    fprintf(f, "Datafile: %s %s\n", plinkbin, UPHEN);
    fprintf(f, "Permutations: %d (phenotype shuffled as by -p p, p = 1..%d)\n", K, K);
    fprintf(f, "Test: %s\n", inter ? "interactions + full" : "full");
    fprintf(f, "Observed largest F: %f\n", maxf[0]);
    fprintf(f, "Family-wise p-value of the observed largest F: %f\n", (1.0 + above) / (K + 1.0));
    fprintf(f, "Family-wise 5%% threshold for F: %f\n", fw_threshold(s1, K, 0.05));
    fprintf(f, "Family-wise 1%% threshold for F: %f\n", fw_threshold(s1, K, 0.01));
    if (inter) {
        fprintf(f, "Observed largest Fint: %f\n", maxf2[0]);
        fprintf(f, "Family-wise p-value of the observed largest Fint: %f\n", (1.0 + above2) / (K + 1.0));
        fprintf(f, "Family-wise 5%% threshold for Fint: %f\n", fw_threshold(s2, K, 0.05));
        fprintf(f, "Family-wise 1%% threshold for Fint: %f\n", fw_threshold(s2, K, 0.01));
    }
    fprintf(f, "\nPerm\tmaxF%s\n", inter ? "\tmaxFint" : "");
    for (int p = 1; p <= K; p++) {
        if (inter) fprintf(f, "%d\t%f\t%f\n", p, maxf[p], maxf2[p]);
        else fprintf(f, "%d\t%f\n", p, maxf[p]);
    }
    fclose(f);
    free(s1);
    free(s2);
    printf("Permutation maxima and family-wise thresholds written to %s\n", fn);
}

int perform_scan(int *geno, chromosome *chrstat, ped *dat, map *genmap, int nid, int nsnp, int npack, int remain,
                 int nchr, char *filename)
{
    const double t_start = wall_seconds();
    epi_ctx *ctx = NULL;
    epi_status st = epi_open(UDEVICE, &ctx);
    if (st != EPI_OK) fail(NULL, st, "opening the GPU");
    {
        char name[256];
        int sms = 0;
        epi_device_info(ctx, name, sizeof(name), &sms);
        printf("\nUsing device %d: %s (%d SMs)\n\n", UDEVICE, name, sms);
    }

    int s1 = 0, s2 = 0, tothits = 0;
    const int chrint = nchr * (nchr + 1) / 2;
    int ccount = 0;
    if (resume_point(filename, &s1, &s2, &tothits, nid, nsnp) && (s1 != 0 || s2 != 0)) {
        ccount = s1 * (s1 + 1) / 2 + s2;
        if (ccount == chrint) {
            printf("Scan already completed!\n\n");
            epi_close(ctx);
            return tothits;
        } else if (ccount > chrint) {
            printf("The initial analysis was performed with a different dataset!\nPlease use a different "
                   "filename.\n");
            exit(1);
        }
        if (UNPERM > 0) {
            printf("A permutation threshold (-N) needs every block scanned in one run; %s already holds part of "
                   "a scan. Please use a different filename.\n", filename);
            exit(1);
        }
        printf("Resuming from %d/%d, %d hits found so far...\n\n", ccount + 1, chrint, tothits);
    } else {
        write_header_full(filename, nid, nsnp);
    }

    st = epi_load_packed(ctx, (const int32_t *)geno, nid, nsnp, npack, remain);
    if (st != EPI_OK) fail(ctx, st, "loading genotypes");
    /* trait 0 is the phenotype; with -N, traits 1..UNPERM are its permutations p = 1..UNPERM
     * by the -p rule (src/main.c:336-357), scanned in the same launches */
    const int ntraits = 1 + UNPERM;
    float *phen = (float *)malloc(sizeof(float) * (size_t)nid * ntraits);
    uint8_t *valid = (uint8_t *)malloc((size_t)nid * ntraits);
    if (!phen || !valid) {
        printf("Out of host memory for %d phenotype columns\n", ntraits);
        exit(1);
    }
    for (int i = 0; i < nid; i++) phen[i] = dat[i].phen;
    for (int t = 1; t < ntraits; t++) {
        memcpy(phen + (size_t)t * nid, phen, sizeof(float) * (size_t)nid);
        epi_permute_phenotype(phen + (size_t)t * nid, nid, (uint32_t)t);
    }
    if (UNPERM == 0) {
        st = epi_set_phenotype(ctx, phen, nid, USAFE);
    } else {
        for (size_t k = 0; k < (size_t)nid * ntraits; k++) valid[k] = USAFE ? 1 : (phen[k] != -9.0f);
        st = epi_set_traits(ctx, phen, nid, ntraits, valid);
    }
    if (st != EPI_OK) fail(ctx, st, "loading the phenotype");
    free(phen);
    free(valid);
    float *maxf = (float *)malloc(sizeof(float) * (size_t)ntraits * 4);
    float *maxf2 = maxf + ntraits, *accf = maxf + 2 * ntraits, *accf2 = maxf + 3 * ntraits;
    for (int t = 0; t < ntraits; t++) accf[t] = accf2[t] = -INFINITY;

    epi_scan_opts opts;
    epi_default_opts(&opts);
    opts.test = UTEST;
    opts.safe = USAFE;
    opts.chunk = UCHUNKSIZE;
    opts.t1 = UTHRESHOLD1;
    opts.t2 = UTHRESHOLD2;
    opts.form = UFORM;
    opts.report_trait = 0;

    /* remaining blocks in perform_scan's order */
    epi_block *blocks = (epi_block *)malloc(sizeof(epi_block) * (size_t)(chrint > 0 ? chrint : 1));
    int *bi = (int *)malloc(sizeof(int) * (size_t)(chrint > 0 ? chrint : 1));
    int *bj = (int *)malloc(sizeof(int) * (size_t)(chrint > 0 ? chrint : 1));
    int nb = 0;
    for (int i = s1; i < nchr; i++) {
        /* the reference restarts every later chromosome at column s2 as well
         * (src/EpiOpenCL.c:1540), skipping blocks (i > s1, j < s2); -R 1 keeps that for
         * comparisons with its output, the default rescans them */
        for (int j = (i == s1 || UREFRESUME) ? s2 : 0; j <= i; j++) {
            blocks[nb].start1 = chrstat[i].chrstart;
            blocks[nb].size1 = chrstat[i].chrsize;
            blocks[nb].start2 = chrstat[j].chrstart;
            blocks[nb].size2 = chrstat[j].chrsize;
            bi[nb] = i;
            bj[nb] = j;
            ++nb;
        }
    }

    int64_t cap = 1 << 20;
    epi_hit *hits = (epi_hit *)malloc(sizeof(epi_hit) * (size_t)cap);
    int32_t *hblock = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
    double gpu_ms = 0.0;
    int b0 = 0;
    while (b0 < nb) {
        /* batch of whole blocks up to PAIR_BATCH pairs */
        long long pairs = 0;
        int b1 = b0;
        while (b1 < nb && (b1 == b0 || pairs + (long long)blocks[b1].size1 * blocks[b1].size2 <= PAIR_BATCH)) {
            pairs += (long long)blocks[b1].size1 * blocks[b1].size2;
            ++b1;
        }
        for (int b = b0; b < b1; ++b)
            printf("%d/%d\tScanning %s vs %s\n", ++ccount, chrint, chrstat[bi[b]].chrname, chrstat[bj[b]].chrname);
        fflush(stdout);
        int64_t n = 0;
        st = epi_scan(ctx, blocks + b0, b1 - b0, &opts, hits, cap, &n, hblock, NULL, maxf, maxf2);
        if (st == EPI_E_OVERFLOW) {
            free(hits);
            free(hblock);
            cap = n;
            hits = (epi_hit *)malloc(sizeof(epi_hit) * (size_t)cap);
            hblock = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
            if (!hits || !hblock) {
                printf("Out of host memory for %lld results\n", (long long)n);
                exit(1);
            }
            st = epi_scan(ctx, blocks + b0, b1 - b0, &opts, hits, cap, &n, hblock, NULL, maxf, maxf2);
        }
        if (st != EPI_OK) fail(ctx, st, "scanning");
        for (int t = 0; t < ntraits; t++) {
            if (maxf[t] > accf[t]) accf[t] = maxf[t];
            if (maxf2[t] > accf2[t]) accf2[t] = maxf2[t];
        }
        double ms = 0.0;
        epi_last_timing(ctx, &ms, NULL, NULL, NULL);
        gpu_ms += ms;

        FILE *out = fopen(filename, "a");
        if (!out) {
            printf("Cannot append to %s\n", filename);
            exit(1);
        }
        int64_t h = 0;
        for (int b = b0; b < b1; ++b) {
            const int i = bi[b], j = bj[b];
            int64_t h_end = h;
            while (h_end < n && hblock[h_end] == b - b0) ++h_end;
            const int tn = (int)(h_end - h);
            printf("\n\t%d interactions found in %s vs %s\n", tn, chrstat[i].chrname, chrstat[j].chrname);
            fprintf(out, "# %d x %d : %d interactions\n", i, j, tn);
            for (; h < h_end; ++h) {
                const epi_hit *r = &hits[h];
                if (UTEST == 'f')
                    fprintf(out, "%d\t%s\t%s\t%d\t%s\t%s\t%d\t%d\t%f\n", r->snp1 + 1, genmap[r->snp1].snpname,
                            chrstat[i].chrname, r->snp2 + 1, genmap[r->snp2].snpname, chrstat[j].chrname, r->df1,
                            r->df2, r->F);
                else
                    fprintf(out, "%d\t%s\t%s\t%d\t%s\t%s\t%d\t%d\t%f\t%f\n", r->snp1 + 1, genmap[r->snp1].snpname,
                            chrstat[i].chrname, r->snp2 + 1, genmap[r->snp2].snpname, chrstat[j].chrname, r->df1,
                            r->df2, r->F, r->F2);
                ++tothits;
            }
        }
        fclose(out);
        char tt[64];
        format_duration(tt, sizeof(tt), ms / 1000.0);
        printf("\n\t%d blocks scanned on the GPU in %s (%.3f s)\n\n", b1 - b0, tt, ms / 1000.0);
        b0 = b1;
    }
    if (UNPERM > 0) write_permutation_summary(filename, ntraits, accf, accf2);
    free(maxf);
    free(hits);
    free(hblock);
    free(blocks);
    free(bi);
    free(bj);
    epi_close(ctx);

    char tt[64];
    format_duration(tt, sizeof(tt), wall_seconds() - t_start);
    printf("\nProgramme finished in %s (GPU %.3f s)\n%d epistatic interactions discovered\n", tt, gpu_ms / 1000.0,
           tothits);
    return tothits;
}
