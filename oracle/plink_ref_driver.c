/*
 * plink_ref_driver.c -- TEST INFRASTRUCTURE: a command-line driver around the reference's
 * own data-mode functions (src/readplink.c, compiled unmodified beside this file by the
 * Makefile into oracle/_ref/plinkref). It is the oracle for epiGPU -Dr / -De:
 *
 *   plinkref write <ped> <map> <epigpu>   dims, readped, readmap, pack, createpackedbinary
 *                                         (src/readplink.c:8-60, :234-414, :1066-1181), the
 *                                         steps of the reference's "-Dr" (:1330-1431)
 *   plinkref extract <epigpu> <ped> <map> extractfrombinary (:150-223), the "-De" step
 *
 * Record buffers are zero-filled first so that the bytes the reference leaves unset are
 * deterministic. Nothing in the product links or runs this.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "readplink.h"

int main(int argc, char **argv)
{
    if (argc == 5 && strcmp(argv[1], "write") == 0) {
        int nid = 0, nsnp = 0, nchr = 0, npack = 0, remain = 0, *gpack = NULL;
        dims(&nid, &nsnp, argv[2]);
        ped *dat = (ped *)calloc((size_t)nid, sizeof(ped));
        map *genmap = (map *)calloc((size_t)nsnp, sizeof(map));
        char *geno = (char *)calloc((size_t)nid * nsnp, 1);
        chromosome *chrstat = (chromosome *)calloc(50, sizeof(chromosome));
        readped(nid, nsnp, argv[2], dat, geno, genmap);
        readmap(nsnp, genmap, &nchr, chrstat, argv[3]);
        pack(nid, nsnp, &npack, &remain, &gpack, geno);
        createpackedbinary(nid, nsnp, npack, remain, nchr, genmap, dat, gpack, chrstat, argv[4]);
        return 0;
    }
    if (argc == 5 && strcmp(argv[1], "extract") == 0) {
        extractfrombinary(argv[2], argv[3], argv[4]);
        return 0;
    }
    fprintf(stderr, "usage: plinkref write <ped> <map> <epigpu> | plinkref extract <epigpu> <ped> <map>\n");
    return 2;
}
