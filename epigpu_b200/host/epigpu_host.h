/*
 * epigpu_host.h -- the C host program of the B200 scan: epiGPU's analysis-mode command
 * line (src/main.c), the .epigpu reader (src/readplink.c:1183-1273) and the scan driver
 * that writes the results file (src/EpiOpenCL.c:1312-1686), on top of libepigpu.so.
 */
#ifndef EPIGPU_HOST_H
#define EPIGPU_HOST_H

#include <stdint.h>
#include <stdio.h>

#include "epigpu.h"

/* Records of the .epigpu file. Their byte layout is the file format, so they keep the
 * member order and sizes of src/readplink.h:17-39 (128, 88 and 44 bytes on x86-64). */
typedef struct ped {
    char family[30];
    char id[30];
    char paternal[30];
    char maternal[30];
    char sex;
    float phen;
} ped;

typedef struct map {
    char chr[30];
    char snpname[30];
    double gd;
    long pd;
    char allelename[2];
} map;

typedef struct chromosome {
    int chrid;
    char chrname[30];
    int chrsize;
    int chrstart;
} chromosome;

/* Analysis settings, the globals of src/epiopencl.h:9-16, plus the GPU form (-g). */
extern int UPERM;
extern int UDEVICE;
extern int UCHUNKSIZE;
extern int UTEST;
extern int USAFE;
extern int UFORM;
extern int UREFRESUME; /* -R: resume with the reference's restart-column rule */
extern int UNPERM; /* -N: permutations scanned beside the phenotype (0 = none) */
extern char plinkbin[100];
extern float UTHRESHOLD1, UTHRESHOLD2;
extern char UPHEN[1000];

typedef struct epigpu_data {
    int nid, nsnp, npack, remain, nchr;
    ped *dat;
    map *genmap;
    chromosome *chrstat;
    int32_t *gpack;
} epigpu_data;

/* epifile.c */
int read_epigpu(const char *filename, epigpu_data *d, char *err, size_t errlen);
int write_epigpu(const char *filename, const epigpu_data *d);
void free_epigpu(epigpu_data *d);
int read_phenotype_file(const char *filename, int nid, ped *dat);
int is_binary_phenotype(int nid, const ped *dat);

/* plink.c: data mode */
int plink_to_epigpu(const char *pedfile, const char *mapfile, const char *binfile, char *err, size_t errlen);
int epigpu_to_plink(const char *binfile, const char *pedfile, const char *mapfile, char *err, size_t errlen);

/* scan_driver.c */
int perform_scan(int *geno, chromosome *chrstat, ped *dat, map *genmap, int nid, int nsnp, int npack, int remain,
                 int nchr, char *filename);
int resume_point(const char *filename, int *chr1, int *chr2, int *tothits, int nid, int nsnp);

/* timing.c */
double wall_seconds(void);
void format_duration(char *out, size_t outlen, double seconds);

#endif
