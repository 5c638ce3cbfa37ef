/*
 * epifile.c -- the .epigpu packed binary file and the separate phenotype file.
 *
 * File layout (src/readplink.c:1145-1181): "epiGPU" (6 bytes), int nid, nsnp, npack,
 * remain, nchr, ped[nid], map[nsnp], chromosome[nchr], int[npack1*nsnp] genotype words
 * (npack1 = npack + (remain > 0)). The reader checks what readpackedbinary
 * (src/readplink.c:1183-1273) does not: header consistency and truncation, so that a
 * corrupt file is reported instead of scanned.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "epigpu_host.h"

void free_epigpu(epigpu_data *d)
{
    free(d->dat);
    free(d->genmap);
    free(d->chrstat);
    free(d->gpack);
    memset(d, 0, sizeof(*d));
}

int read_epigpu(const char *filename, epigpu_data *d, char *err, size_t errlen)
{
    memset(d, 0, sizeof(*d));
    FILE *f = fopen(filename, "rb");
    if (!f) {
        snprintf(err, errlen, "No input file found");
        return 1;
    }
    char sig[7] = {0};
    int hdr[5];
    if (fread(sig, 1, 6, f) != 6 || strcmp(sig, "epiGPU") != 0) {
        snprintf(err, errlen, "Invalid input file!\nPlease convert plink .ped and .map data files to the "
                 "epiGPU format.");
        fclose(f);
        return 1;
    }
    if (fread(hdr, sizeof(int), 5, f) != 5) {
        snprintf(err, errlen, "Invalid input file: truncated header");
        fclose(f);
        return 1;
    }
    d->nid = hdr[0];
    d->nsnp = hdr[1];
    d->npack = hdr[2];
    d->remain = hdr[3];
    d->nchr = hdr[4];
    if (d->nid < 1 || d->nsnp < 1 || d->nchr < 1 || d->npack != d->nid / 16 || d->remain != d->nid % 16) {
        snprintf(err, errlen, "Invalid input file: inconsistent header (nid %d, nsnp %d, npack %d, remain %d, "
                 "nchr %d)", d->nid, d->nsnp, d->npack, d->remain, d->nchr);
        fclose(f);
        return 1;
    }
    const size_t npack1 = (size_t)d->npack + (d->remain ? 1 : 0);
    d->dat = (ped *)malloc(sizeof(ped) * (size_t)d->nid);
    d->genmap = (map *)malloc(sizeof(map) * (size_t)d->nsnp);
    d->chrstat = (chromosome *)malloc(sizeof(chromosome) * (size_t)d->nchr);
    d->gpack = (int32_t *)malloc(sizeof(int32_t) * npack1 * (size_t)d->nsnp);
    if (!d->dat || !d->genmap || !d->chrstat || !d->gpack) {
        snprintf(err, errlen, "Out of host memory reading %s", filename);
        fclose(f);
        free_epigpu(d);
        return 1;
    }
    if (fread(d->dat, sizeof(ped), (size_t)d->nid, f) != (size_t)d->nid ||
        fread(d->genmap, sizeof(map), (size_t)d->nsnp, f) != (size_t)d->nsnp ||
        fread(d->chrstat, sizeof(chromosome), (size_t)d->nchr, f) != (size_t)d->nchr ||
        fread(d->gpack, sizeof(int32_t), npack1 * d->nsnp, f) != npack1 * (size_t)d->nsnp) {
        snprintf(err, errlen, "Invalid input file: truncated");
        fclose(f);
        free_epigpu(d);
        return 1;
    }
    fclose(f);
    for (int c = 0; c < d->nchr; ++c) {
        const chromosome *ch = &d->chrstat[c];
        if (ch->chrsize < 0 || ch->chrstart < 0 || (long long)ch->chrstart + ch->chrsize > d->nsnp) {
            snprintf(err, errlen, "Invalid input file: chromosome %d spans SNPs %d..%d of %d", c, ch->chrstart,
                     ch->chrstart + ch->chrsize, d->nsnp);
            free_epigpu(d);
            return 1;
        }
    }
    return 0;
}

int write_epigpu(const char *filename, const epigpu_data *d)
{
    FILE *f = fopen(filename, "wb");
    if (!f) return 1;
    const int hdr[5] = {d->nid, d->nsnp, d->npack, d->remain, d->nchr};
    const size_t npack1 = (size_t)d->npack + (d->remain ? 1 : 0);
    int ok = fwrite("epiGPU", 1, 6, f) == 6 && fwrite(hdr, sizeof(int), 5, f) == 5 &&
             fwrite(d->dat, sizeof(ped), (size_t)d->nid, f) == (size_t)d->nid &&
             fwrite(d->genmap, sizeof(map), (size_t)d->nsnp, f) == (size_t)d->nsnp &&
             fwrite(d->chrstat, sizeof(chromosome), (size_t)d->nchr, f) == (size_t)d->nchr &&
             fwrite(d->gpack, sizeof(int32_t), npack1 * d->nsnp, f) == npack1 * (size_t)d->nsnp;
    return (fclose(f) == 0 && ok) ? 0 : 1;
}

/* src/main.c:191-222: nid values read with "%f"; prints the first and last three. */
int read_phenotype_file(const char *filename, int nid, ped *dat)
{
    FILE *f = fopen(filename, "rt");
    if (!f) return 1;
    printf("Reading in separate phenotype file\n");
    for (int i = 0; i < nid; i++) {
        float v;
        if (fscanf(f, "%f", &v) != 1) {
            fclose(f);
            return 1;
        }
        dat[i].phen = v;
        if (i == 0) printf("First 3 values: ");
        if (i < 3) printf("%f ", v);
        if (i == nid - 3) printf("\nLast 3 values: ");
        if (i >= nid - 3) printf("%f ", v);
    }
    fclose(f);
    printf("\nDone!\n\n");
    return 0;
}

/* src/readplink.c:118-147: a phenotype of only 1s and 2s is a binary trait */
int is_binary_phenotype(int nid, const ped *dat)
{
    for (int i = 0; i < nid; i++)
        if (dat[i].phen != 1.0f && dat[i].phen != 2.0f) return 0;
    return 1;
}
