/*
 * plink.c -- data mode: a PLINK text fileset (.ped + .map) to the packed .epigpu binary
 * (epiGPU -Dr) and back (epiGPU -De).
 *
 * Behaviour follows the reference's data mode:
 *   dims               src/readplink.c:8-60     rows = newlines; columns = runs of non-separator
 *                                               characters, separator = the file's first space
 *                                               or tab; ragged rows are an error; SNPs =
 *                                               (columns - 6) / 2
 *   readped            src/readplink.c:234-346  family, id, father, mother, sex, phenotype, then
 *                                               two allele characters per SNP; allele '0' =
 *                                               missing, a differing pair = heterozygote (1, and
 *                                               the pair becomes the SNP's allele names), a
 *                                               repeated allele = homozygote; per SNP the first
 *                                               homozygote met (in individual order) becomes 0
 *                                               and the first other homozygote after it 2
 *   readmap            src/readplink.c:351-414  chromosome, SNP name, genetic and physical
 *                                               distance; chromosomes numbered in order of
 *                                               first appearance, starts cumulative
 *   pack               src/readplink.c:1066-1102 16 codes per int32 word, first individual in
 *                                               the top bits, tail word right-aligned
 *   createpackedbinary src/readplink.c:1158-1181 (write_epigpu in epifile.c)
 *   extractfrombinary  src/readplink.c:150-223  the inverse, written as text
 * On space-delimited files (the PLINK layout) the output is byte-for-byte the reference's
 * record content. Deliberate differences: tabs also separate genotype columns (the
 * reference's skip set after each allele holds space, '/' and the letter 't', so it misreads
 * tab-delimited genotypes and drops lowercase 't' alleles); names longer than the 29
 * characters a record holds, and lines with too few genotype columns, are reported instead
 * of overrunning a buffer; a SNP with no homozygote keeps its heterozygote / missing codes
 * instead of the reference reading past the SNP.
 */
#include <ctype.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "epigpu_host.h"

#define MISS_CODE 3
#define NAME_MAX_CHARS 29

/* ---- text scanning ---------------------------------------------------------------- */

typedef struct scanner {
    FILE *f;
    long line;
} scanner;

/* next whitespace-delimited token (the "%s" rule), or 0 at end of file */
static int next_token(scanner *s, char *buf, size_t cap, int *too_long)
{
    int c;
    *too_long = 0;
    do {
        c = fgetc(s->f);
        if (c == '\n') s->line++;
    } while (c != EOF && isspace(c));
    if (c == EOF) return 0;
    size_t n = 0;
    while (c != EOF && !isspace(c)) {
        if (n + 1 < cap) buf[n++] = (char)c;
        else *too_long = 1;
        c = fgetc(s->f);
    }
    buf[n] = '\0';
    if (c != EOF) ungetc(c, s->f);
    return 1;
}

/* next allele character on the current line: separators are space, tab, '/' and '\r' */
static int next_allele(scanner *s)
{
    int c;
    do {
        c = fgetc(s->f);
    } while (c == ' ' || c == '\t' || c == '/' || c == '\r');
    if (c == '\n') {
        s->line++;
        return EOF;
    }
    return c;
}

static int copy_name(char *dst, const char *src, int too_long)
{
    if (too_long || strlen(src) > NAME_MAX_CHARS) return 1;
    strcpy(dst, src);
    return 0;
}

/* ---- dims -------------------------------------------------------------------------- */

static int plink_dims(const char *pedfile, int *nid, int *nsnp, char *err, size_t errlen)
{
    FILE *f = fopen(pedfile, "r");
    if (!f) {
        snprintf(err, errlen, "Cannot open %s", pedfile);
        return 1;
    }
    int c, sep = 0;
    while ((c = fgetc(f)) != EOF)
        if (c == ' ' || c == '\t') {
            sep = c;
            break;
        }
    if (!sep) {
        snprintf(err, errlen, "Problem with data, must be space or tab delimited");
        fclose(f);
        return 1;
    }
    rewind(f);
    printf("Getting %s dimensions...", pedfile);
    fflush(stdout);
    long rows = 0, cols = 0, first = -1;
    int in_field = 0, trailing = 0;
    while ((c = fgetc(f)) != EOF) {
        if (c == '\n') {
            rows++;
            if (first < 0) first = cols;
            else if (cols != first) {
                snprintf(err, errlen, "Ragged matrix: line %ld has %ld columns, line 1 has %ld", rows, cols, first);
                fclose(f);
                return 1;
            }
            cols = 0;
            in_field = 0;
            trailing = 0;
        } else if (c == sep) {
            in_field = 0;
        } else {
            if (!in_field) cols++;
            in_field = 1;
            trailing = 1;
        }
    }
    fclose(f);
    if (trailing) printf("\nwarning: the last line of %s has no newline and is not read\n", pedfile);
    if (rows < 1 || first < 8) {
        snprintf(err, errlen, "%s: no individual with genotype columns", pedfile);
        return 1;
    }
    *nid = (int)rows;
    *nsnp = (int)((first - 6) / 2);
    printf("done!\n%d SNPs, %d Individuals\n\n", *nsnp, *nid);
    fflush(stdout);
    return 0;
}

/* ---- .ped --------------------------------------------------------------------------- */

/* geno[s * nid + i]: 0/1/2/3, or (as in the reference) the allele character of a homozygote
 * that is neither of the SNP's first two homozygotes */
static int plink_read_ped(const char *pedfile, int nid, int nsnp, ped *dat, signed char *geno, map *genmap, char *err,
                          size_t errlen)
{
    FILE *f = fopen(pedfile, "r");
    if (!f) {
        snprintf(err, errlen, "Cannot open %s", pedfile);
        return 1;
    }
    scanner s = {f, 1};
    char tok[256];
    int too_long;
    printf("Reading in %s...", pedfile);
    fflush(stdout);
    for (int j = 0; j < nsnp; j++) genmap[j].allelename[0] = genmap[j].allelename[1] = 0;
    for (int i = 0; i < nid; i++) {
        char *names[4] = {dat[i].family, dat[i].id, dat[i].paternal, dat[i].maternal};
        for (int q = 0; q < 4; q++) {
            if (!next_token(&s, tok, sizeof(tok), &too_long)) {
                snprintf(err, errlen, "%s: individual %d is incomplete", pedfile, i + 1);
                fclose(f);
                return 1;
            }
            if (copy_name(names[q], tok, too_long)) {
                snprintf(err, errlen, "%s line %ld: name longer than %d characters", pedfile, s.line, NAME_MAX_CHARS);
                fclose(f);
                return 1;
            }
        }
        char *end;
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_line;
        dat[i].sex = (char)strtol(tok, &end, 10);
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_line;
        dat[i].phen = strtof(tok, &end);
        for (int j = 0; j < nsnp; j++) {
            const int a1 = next_allele(&s);
            const int a2 = a1 == EOF ? EOF : next_allele(&s);
            if (a1 == EOF || a2 == EOF) goto short_line;
            signed char g;
            if (a1 == '0') {
                g = MISS_CODE;
            } else if (a1 != a2) {
                genmap[j].allelename[0] = (char)a1;
                genmap[j].allelename[1] = (char)a2;
                g = 1;
            } else {
                g = (signed char)a1;
            }
            geno[(size_t)j * nid + i] = g;
        }
        continue;
    short_line:
        snprintf(err, errlen, "%s line %ld: fewer than %d genotype columns", pedfile, s.line, 2 * nsnp);
        fclose(f);
        return 1;
    }
    fclose(f);
    printf("done!\nConverting...");
    fflush(stdout);
    /* homozygote allele characters -> 0 / 2 per SNP */
    for (int j = 0; j < nsnp; j++) {
        signed char *g = geno + (size_t)j * nid;
        int first = 0;
        while (first < nid && (g[first] == 1 || g[first] == MISS_CODE)) first++;
        if (first == nid) continue;  /* no homozygote: nothing to convert */
        const signed char h1 = g[first];
        if (genmap[j].allelename[0] == 0) {
            genmap[j].allelename[0] = h1;
        } else if (h1 == genmap[j].allelename[1]) {
            genmap[j].allelename[1] = genmap[j].allelename[0];
            genmap[j].allelename[0] = h1;
        }
        int second = first + 1;
        while (second < nid && (g[second] == 1 || g[second] == h1 || g[second] == MISS_CODE)) second++;
        const int has2 = second < nid;
        const signed char h2 = has2 ? g[second] : 0;
        for (int i = first; i < nid; i++) {
            if (g[i] == h1) g[i] = 0;
            else if (has2 && g[i] == h2) g[i] = 2;
        }
    }
    printf("done!\n");
    return 0;
}

/* ---- .map --------------------------------------------------------------------------- */

static int plink_read_map(const char *mapfile, int nsnp, map *genmap, int *nchr, chromosome **chrstat, char *err,
                          size_t errlen)
{
    FILE *f = fopen(mapfile, "r");
    if (!f) {
        snprintf(err, errlen, "Cannot open %s", mapfile);
        return 1;
    }
    scanner s = {f, 1};
    char tok[256];
    int too_long, cap = 32;
    chromosome *cs = (chromosome *)calloc((size_t)cap, sizeof(chromosome));
    *nchr = 0;
    printf("Reading in %s...", mapfile);
    fflush(stdout);
    for (int i = 0; i < nsnp; i++) {
        char *end;
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_map;
        if (copy_name(genmap[i].chr, tok, too_long)) goto long_name;
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_map;
        if (copy_name(genmap[i].snpname, tok, too_long)) goto long_name;
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_map;
        genmap[i].gd = strtod(tok, &end);
        if (!next_token(&s, tok, sizeof(tok), &too_long)) goto short_map;
        genmap[i].pd = strtol(tok, &end, 0);  /* "%li": base from the prefix, as fscanf */
        int c = 0;
        while (c < *nchr && strcmp(genmap[i].chr, cs[c].chrname) != 0) c++;
        if (c == *nchr) {
            if (*nchr == cap) {
                cap *= 2;
                chromosome *grown = (chromosome *)realloc(cs, sizeof(chromosome) * (size_t)cap);
                if (!grown) {
                    snprintf(err, errlen, "Out of host memory reading %s", mapfile);
                    free(cs);
                    fclose(f);
                    return 1;
                }
                cs = grown;
                memset(cs + *nchr, 0, sizeof(chromosome) * (size_t)(cap - *nchr));
            }
            cs[c].chrid = c;
            strcpy(cs[c].chrname, genmap[i].chr);
            cs[c].chrsize = 0;
            (*nchr)++;
        }
        cs[c].chrsize++;
    }
    fclose(f);
    cs[0].chrstart = 0;
    for (int c = 1; c < *nchr; c++) cs[c].chrstart = cs[c - 1].chrstart + cs[c - 1].chrsize;
    printf("done!\n%d chromosomes\n", *nchr);
    for (int c = 0; c < *nchr; c++) printf("%s\t%d\t%d\n", cs[c].chrname, cs[c].chrsize, cs[c].chrstart);
    fflush(stdout);
    *chrstat = cs;
    return 0;
short_map:
    snprintf(err, errlen, "%s: fewer than %d SNP rows (4 columns each)", mapfile, nsnp);
    free(cs);
    fclose(f);
    return 1;
long_name:
    snprintf(err, errlen, "%s line %ld: name longer than %d characters", mapfile, s.line, NAME_MAX_CHARS);
    free(cs);
    fclose(f);
    return 1;
}

/* ---- packing ------------------------------------------------------------------------ */

/* 16 codes per word, first individual in bits 31:30; the tail word holds `remain` codes
 * right-aligned. Codes are OR-ed in as the reference does, so an out-of-range code (an
 * extra homozygote's character) lands in the same bits. */
static void pack_codes(int nid, int nsnp, const signed char *geno, int32_t *gpack)
{
    const int npack = nid / 16, remain = nid % 16, npack1 = npack + (remain ? 1 : 0);
    for (int s = 0; s < nsnp; s++) {
        const signed char *g = geno + (size_t)s * nid;
        int k = 0;
        for (int w = 0; w < npack1; w++) {
            const int n = w < npack ? 16 : remain;
            uint32_t p = (uint32_t)(int32_t)g[k++];
            for (int l = 1; l < n; l++) p = (p << 2) | (uint32_t)(int32_t)g[k++];
            gpack[(size_t)s * npack1 + w] = (int32_t)p;
        }
    }
}

int plink_to_epigpu(const char *pedfile, const char *mapfile, const char *binfile, char *err, size_t errlen)
{
    epigpu_data d;
    memset(&d, 0, sizeof(d));
    if (plink_dims(pedfile, &d.nid, &d.nsnp, err, errlen)) return 1;
    d.dat = (ped *)calloc((size_t)d.nid, sizeof(ped));
    d.genmap = (map *)calloc((size_t)d.nsnp, sizeof(map));
    signed char *geno = (signed char *)malloc((size_t)d.nid * d.nsnp);
    d.npack = d.nid / 16;
    d.remain = d.nid % 16;
    const size_t npack1 = (size_t)d.npack + (d.remain ? 1 : 0);
    d.gpack = (int32_t *)malloc(sizeof(int32_t) * npack1 * (size_t)d.nsnp);
    if (!d.dat || !d.genmap || !geno || !d.gpack) {
        snprintf(err, errlen, "Out of host memory for %d individuals x %d SNPs", d.nid, d.nsnp);
        free(geno);
        free_epigpu(&d);
        return 1;
    }
    int rc = plink_read_ped(pedfile, d.nid, d.nsnp, d.dat, geno, d.genmap, err, errlen);
    if (!rc) rc = plink_read_map(mapfile, d.nsnp, d.genmap, &d.nchr, &d.chrstat, err, errlen);
    if (!rc) {
        pack_codes(d.nid, d.nsnp, geno, d.gpack);
        printf("\nStoring\n- %d individuals\n- %d SNPs\n- %d chromosomes\nin epigpu binary format as file \"%s\"..",
               d.nid, d.nsnp, d.nchr, binfile);
        fflush(stdout);
        if (write_epigpu(binfile, &d)) {
            snprintf(err, errlen, "Cannot write %s", binfile);
            rc = 1;
        } else {
            printf("done!\n");
        }
    }
    free(geno);
    free_epigpu(&d);
    return rc;
}

/* ---- extraction --------------------------------------------------------------------- */

static int code_at(const epigpu_data *d, int s, int i)
{
    const int npack1 = d->npack + (d->remain ? 1 : 0);
    const uint32_t *row = (const uint32_t *)d->gpack + (size_t)s * npack1;
    if (i < 16 * d->npack) return (int)((row[i / 16] >> (30 - 2 * (i % 16))) & 3u);
    const int t = i - 16 * d->npack;
    return (int)((row[d->npack] >> (2 * (d->remain - 1 - t))) & 3u);
}

int epigpu_to_plink(const char *binfile, const char *pedfile, const char *mapfile, char *err, size_t errlen)
{
    epigpu_data d;
    if (read_epigpu(binfile, &d, err, errlen)) return 1;
    FILE *mf = fopen(mapfile, "w");
    FILE *pf = mf ? fopen(pedfile, "w") : NULL;
    if (!mf || !pf) {
        snprintf(err, errlen, "Cannot write %s / %s", pedfile, mapfile);
        if (mf) fclose(mf);
        free_epigpu(&d);
        return 1;
    }
    printf("Extracting data stored in \"%s\", and writing to \"%s\" and \"%s\"\n", binfile, pedfile, mapfile);
    for (int s = 0; s < d.nsnp; s++)
        fprintf(mf, "%s %s %f %ld\n", d.genmap[s].chr, d.genmap[s].snpname, d.genmap[s].gd, d.genmap[s].pd);
    const int binary = is_binary_phenotype(d.nid, d.dat);
    printf(binary ? "Writing to files (binary phenotype)..." : "Writing to files (continuous phenotype)...");
    for (int i = 0; i < d.nid; i++) {
        const ped *p = &d.dat[i];
        if (binary)
            fprintf(pf, "%s %s %s %s %d %d", p->family, p->id, p->paternal, p->maternal, (int)p->sex, (int)p->phen);
        else
            fprintf(pf, "%s %s %s %s %d %f", p->family, p->id, p->paternal, p->maternal, (int)p->sex, p->phen);
        for (int s = 0; s < d.nsnp; s++) {
            const char a = d.genmap[s].allelename[0], b = d.genmap[s].allelename[1];
            /* the characters are written as stored, a NUL name included, as the reference does */
            switch (code_at(&d, s, i)) {
            case 0: fputc(' ', pf); fputc(a, pf); fputc(' ', pf); fputc(a, pf); break;
            case 1: fputc(' ', pf); fputc(a, pf); fputc(' ', pf); fputc(b, pf); break;
            case 2: fputc(' ', pf); fputc(b, pf); fputc(' ', pf); fputc(b, pf); break;
            default: fputs(" 0 0", pf); break;
            }
        }
        fputc('\n', pf);
    }
    const int ok = fclose(pf) == 0 && fclose(mf) == 0;
    printf("done\n\n");
    free_epigpu(&d);
    if (!ok) snprintf(err, errlen, "Cannot write %s / %s", pedfile, mapfile);
    return ok ? 0 : 1;
}
