/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Host harness around the reference's own CPU fixup_utoprim (fixup.c:764-827),
 * the neighbour interpolation of zones whose inversion failed. fixup.c is
 * compiled where it lies, against a configured config.h whose radfix_dens is
 * left as written (its CPU fixup1zone uses it as a plain constant). The
 * harness owns the globals fixup.c reads (pflag, failimage: decs.h:51,87) and
 * index_3D (main.c:355), and converts between the product's planar layout
 * (plane k of ksize doubles) and the reference's host layout
 * pv[block][index_3D][NPR].
 */
#include "include.h"
#include "decs.h"
#include <stdlib.h>

int(*restrict pflag[NB_LOCAL]);
int(*restrict failimage[NB_LOCAL])[NFAIL];

int index_3D(int n, int i, int j, int z) {
    return ((i - N1_GPU_offset[n]) + N1G) * (BS_2 + 2 * N2G) * (BS_3 + 2 * N3G)
         + ((j - N2_GPU_offset[n]) + N2G) * (BS_3 + 2 * N3G) + ((z - N3_GPU_offset[n]) + N3G);
}

/* pv: NPR planes, pfl: 1 plane, fi: NFAIL planes, all ksize apart */
void ref_fixup_utoprim(double *pv, int *pfl, int *fi, long ksize) {
    static double (*pvb[NB_LOCAL])[NPR];
    const long n = (long)(BS_1 + 2 * N1G) * (BS_2 + 2 * N2G) * (BS_3 + 2 * N3G);
    double (*P)[NPR] = malloc(sizeof(*P) * n);
    int *F = malloc(sizeof(int) * n);
    int (*FI)[NFAIL] = malloc(sizeof(*FI) * n);
    for (long c = 0; c < n; c++) {
        for (int k = 0; k < NPR; k++) P[c][k] = pv[k * ksize + c];
        F[c] = pfl[c];
        for (int q = 0; q < NFAIL; q++) FI[c][q] = fi[q * ksize + c];
    }
    nl[0] = 0;
    N1_GPU_offset[0] = N2_GPU_offset[0] = N3_GPU_offset[0] = 0;
    pvb[0] = P;
    pflag[0] = F;
    failimage[0] = FI;
    fixup_utoprim(pvb, 0);
    for (long c = 0; c < n; c++) {
        for (int k = 0; k < NPR; k++) pv[k * ksize + c] = P[c][k];
        pfl[c] = F[c];
        for (int q = 0; q < NFAIL; q++) fi[q * ksize + c] = FI[c][q];
    }
    pflag[0] = 0;
    failimage[0] = 0;
    free(P);
    free(F);
    free(FI);
}
