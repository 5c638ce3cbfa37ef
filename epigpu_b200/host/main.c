/*
 * main.c -- epiGPU's analysis-mode command line on the B200 scan.
 *
 *   epiGPU -A <epigpu file> <output file> [-p n] [-i n] [-d n] [-t f|i] [-F x] [-I x]
 *          [-s 0|1] [-P phenotype file] [-g a|p|t]
 *
 * Flags, defaults, validation and messages follow src/main.c:58-188 and :225-334
 * (defaults :244-249: no permutation, iteration size 128, device 0, test f, F 6.5,
 * I 10.5). -g (new) picks the GPU form: a = automatic, p = plain popcount form,
 * t = tensor-core form. Data mode (-D) is not part of this program.
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "epigpu_host.h"

int UPERM = 0;
int UDEVICE = 0;
int UCHUNKSIZE = 128;
int UTEST = 'f';
int USAFE = 0;
char plinkbin[100];
float UTHRESHOLD1 = 6.5f, UTHRESHOLD2 = 10.5f;
char UPHEN[1000];

static const char *usage_text =
    "\n\nepiGPU (B200) performs an exhaustive 2D scan for epistasis\n\n"
    "DATA MODE:\n\n"
    "<epigpu> -Dr [ .ped file ] [ .map file ] [ epigpu file ]\tread PLINK data into an epigpu file\n"
    "<epigpu> -De [ .ped file ] [ .map file ] [ epigpu file ]\textract an epigpu file to PLINK data\n\n"
    "ANALYSIS MODE:\n\n"
    "<epigpu> -A [ epigpu file] [ output file] [ Options ... ]\n\n"
    "Options:\n\n"
    "p [n]\tPermutation, default [n] = 0 (no permutation)\n"
    "i [n]\tIteration size, default [n] = 128 (sets the order of results within a block)\n"
    "d [n]\tDevice, default [n] = 0\n"
    "t [f/i]\tFull test or full test with interaction test, default = f\n"
    "F [n]\tF value threshold for full test, default [n] = 6.5\n"
    "I [n]\tF value threshold for interaction test, default [n] = 10.5\n"
    "s [0/1]\tNormal / Safe mode. Default = 0 (Normal mode)\n"
    "P [file]\tSeparate phenotype file, one value per individual\n"
    "g [a/p/t]\tGPU form: automatic, plain popcount, tensor core. Default = a\n"
    "N [n]\tPermutation threshold: also scan n permutations of the phenotype in the same launches\n"
    "\tand write each one's largest F and the family-wise thresholds to <output file>.perm\n"
    "R [0/1]\tResume exactly as the reference does (1 also skips, on later chromosomes, the blocks\n"
    "\tbefore the restart column). Default = 0\n\n"
    "Example:\n"
    "<epigpu> -A [ epigpu file ] [ output file ]\n"
    "<epigpu> -A [ epigpu file ] [ output file ] -i 512 -p 100 -F 7\n\n\n";

static int all_digits(const char *s)
{
    int bad = 0;
    for (; *s; ++s) bad += isdigit((unsigned char)*s) ? 0 : 1;
    return bad == 0;
}

/* basename of the data file (src/main.c:359-375) */
static void set_plinkbin(const char *path)
{
    const char *b = path;
    for (const char *p = path; *p; ++p)
        if (*p == '/' || *p == '\\') b = p + 1;
    snprintf(plinkbin, sizeof(plinkbin), "%s", b);
}

static void parse_analysis_args(int argc, char **argv, char **binfile, char **outfile)
{
    if (argc < 4 || (argc & 1) != 0) {
        printf("Incorrect arguments\n%s", usage_text);
        exit(1);
    }
    set_plinkbin(argv[2]);
    *binfile = argv[2];
    *outfile = argv[3];
    for (int i = 4; i < argc; i += 2) {
        if (argv[i][0] != '-') {
            printf("Incorrect optional arguments %c\n%s", argv[i][0], usage_text);
            exit(1);
        }
        const char *v = argv[i + 1];
        switch (argv[i][1]) {
        case 's':
            if (!all_digits(v) || (atoi(v) != 0 && atoi(v) != 1)) {
                printf("Safe mode option: Some graphics cards may not support all optimisation techniques. "
                       "To disable them set safe mode to 1.\nDefault = 0 (normal mode)\n\n");
                exit(1);
            }
            USAFE = atoi(v);
            break;
        case 'p':
            if (!all_digits(v)) {
                printf("Please enter a numeric value for permutations\nDefault = 0 (no permutation)\n\n");
                exit(1);
            }
            UPERM = atoi(v);
            break;
        case 'i': {
            if (!all_digits(v)) {
                printf("Please enter a numeric value for iteration size\nDefault = 128\n\n");
                exit(1);
            }
            const int k = atoi(v);
            if (k < 16 || k % 16 != 0) {
                printf("Iteration size must be a multiple of 16\nDefault = 128\n\n");
                exit(1);
            }
            UCHUNKSIZE = k;
            break;
        }
        case 'd':
            if (!all_digits(v)) {
                printf("Please enter a numeric value for device\nDefault = 0\nOnly change this if you have "
                       "multiple graphics cards\n\n");
                exit(1);
            }
            UDEVICE = atoi(v);
            break;
        case 't':
            if (v[0] != 'f' && v[0] != 'i') {
                printf("Test selection:\nf\tFull 8df test\ni\tFull 8df test + 4df interaction test\n\n");
                exit(1);
            }
            UTEST = v[0];
            break;
        case 'F':
            UTHRESHOLD1 = (float)atof(v);
            if (UTHRESHOLD1 == 0) {
                printf("Please enter a numeric F-test threshold value.\nRecommended values 5.5 - 10\n"
                       "Default = 6.5\n\n");
                exit(1);
            }
            break;
        case 'I':
            UTHRESHOLD2 = (float)atof(v);
            if (UTHRESHOLD2 == 0) {
                printf("Please enter a numeric F-test threshold value.\nRecommended values 5.5 - 10\n"
                       "Default = 10.5\n\n");
                exit(1);
            }
            if (UTEST == 'f')
                printf("\n\nWarning: Interaction test threshold has been set, but interaction test isn't "
                       "being performed\n\n\n");
            break;
        case 'P': {
            FILE *f = fopen(v, "rt");
            if (!f) {
                printf("Separate phenotype file does not exist\n");
                exit(1);
            }
            fclose(f);
            snprintf(UPHEN, sizeof(UPHEN), "%s", v);
            break;
        }
        case 'R':
            UREFRESUME = atoi(v) != 0;
            break;
        case 'N':
            UNPERM = atoi(v);
            if (UNPERM < 0 || UNPERM > 100000) {
                printf("Permutation threshold: the number of phenotype permutations scanned with the data, "
                       "0 to 100000\nDefault = 0 (none)\n\n");
                exit(1);
            }
            break;
        case 'g':
            if (v[0] == 'a') UFORM = EPI_FORM_AUTO;
            else if (v[0] == 'p') UFORM = EPI_FORM_POPC;
            else if (v[0] == 't') UFORM = EPI_FORM_TENSOR;
            else {
                printf("GPU form:\na\tautomatic\np\tplain popcount form\nt\ttensor-core form\n\n");
                exit(1);
            }
            break;
        default:
            printf("Incorrect optional arguments %c\n", argv[i][0]);
            exit(1);
        }
    }
}

/* src/main.c:336-357: shuffle whole ped records with glibc rand(), write perm<n>.txt */
static void permute_records(int nid, ped *dat)
{
    for (int i = nid; i > 1; i--) {
        const int r = rand() % i;
        const ped t = dat[r];
        dat[r] = dat[i - 1];
        dat[i - 1] = t;
    }
    char fn[64];
    snprintf(fn, sizeof(fn), "perm%d.txt", UPERM);
    FILE *out = fopen(fn, "w");
    if (out) {
        fprintf(out, "Family ID Phenotype\n");
        for (int i = 0; i < nid; i++) fprintf(out, "%s %s %f\n", dat[i].family, dat[i].id, dat[i].phen);
        fclose(out);
    }
}

/* Data mode (src/readplink.c:1296-1431): -Dr reads a PLINK .ped/.map fileset into a .epigpu
 * file, -De writes one back out as text. The reference's other data-mode letters (c clean,
 * m impute, n random phenotype, s/q simulate, g GenABEL, u unpacked) are data preparation
 * outside the scan and are refused with a message. */
static int data_mode(int argc, char **argv)
{
    const char *flags = argv[1] + 2;
    int read = 0, extract = 0;
    if (strlen(argv[1]) > 6) {
        printf("Wrong flags\n%s", usage_text);
        exit(1);
    }
    for (const char *c = flags; *c; ++c) {
        if (*c == 'r') read = 1;
        else if (*c == 'e') extract = 1;
        else {
            printf("Data mode letter '%c' (cleaning, imputation, simulation, GenABEL or unpacked output) is not part of "
                   "this program; it reads PLINK data (-Dr) and extracts it (-De).\n", *c);
            exit(1);
        }
    }
    if (read == extract || argc != 5) {
        printf("Wrong arguments\n%s", usage_text);
        exit(1);
    }
    char err[512];
    int rc;
    if (extract)
        rc = epigpu_to_plink(argv[4], argv[2], argv[3], err, sizeof(err));
    else
        rc = plink_to_epigpu(argv[2], argv[3], argv[4], err, sizeof(err));
    if (rc) {
        printf("\n%s\n", err);
        exit(1);
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        printf("%s", usage_text);
        exit(1);
    }
    if (argv[1][0] != '-') {
        printf("Incorrect arguments\n%s", usage_text);
        exit(1);
    }
    if (argv[1][1] == 'D') return data_mode(argc, argv);
    if (argv[1][1] != 'A') {
        printf("%s", usage_text);
        exit(1);
    }
    char *binfile, *outfile;
    parse_analysis_args(argc, argv, &binfile, &outfile);

    printf("\n\nepiGPU (B200)\n\n"
           "This programme will perform an exhaustive 2D scan for\n"
           "epistasis on the GPU\n\n"
           "To interupt the scan press ctrl + c, and you will be able\n"
           "to resume later by using the same output file.\n\n\n");

    epigpu_data d;
    char err[256];
    printf("\nReading in data...\n");
    if (read_epigpu(binfile, &d, err, sizeof(err)) != 0) {
        printf("%s\n", err);
        exit(1);
    }
    printf("%d SNPs, %d individuals, %d chromosomes\n\n", d.nsnp, d.nid, d.nchr);
    fflush(stdout);

    if (UPHEN[0]) {
        if (read_phenotype_file(UPHEN, d.nid, d.dat) != 0) {
            printf("Could not read %d values from the phenotype file\n", d.nid);
            exit(1);
        }
    }
    if (is_binary_phenotype(d.nid, d.dat)) {
        printf("Error: Binary phenotype!\nepiGPU can only use quantitative phenotypes for analysis.\n\n");
        exit(1);
    }
    if (UPERM > 0) {
        printf("Permutation %d\n", UPERM);
        srand((unsigned)UPERM);
        permute_records(d.nid, d.dat);
        for (int i = 0; i < 10 && i < d.nid; i++) printf("%f\n", d.dat[i].phen);
    }
    if (USAFE) printf("Safe mode\n");
    printf(UTEST == 'i' ? "Performing 8 d.f. + 4 d.f. tests\n" : "Performing 8 d.f. test\n");

    perform_scan((int *)d.gpack, d.chrstat, d.dat, d.genmap, d.nid, d.nsnp, d.npack, d.remain, d.nchr, outfile);
    free_epigpu(&d);
    return 0;
}
