/*
 * Test infrastructure (oracle) -- never product code.
 *
 * Runs the reference's own dump and restart writers (dump.c, restart.c,
 * compiled where they lie with a configured config.h) for one block on one
 * rank, to produce golden files for the library's dumpio.py:
 *   dump_params (dump.c:168-272)        -> the parameter header
 *   dump_block (dump.c:276-357)         -> the float dump of the active zones
 *   rdump_block_write (restart.c:54-76) -> the double restart of the block
 * The MPI file functions of ref_stub/mpi.h are implemented here over stdio
 * (one rank: a handle is an index into a table of FILE*). Globals the
 * writers read that the other host-built files do not define are defined
 * here with the reference's declarations (decs.h).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "include.h"
#include "decs_MPI.h"

/* ---- single-rank MPI-IO over stdio ---- */
static FILE *ho_files[64];

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh) {
    (void)comm; (void)amode; (void)info;
    for (int k = 1; k < 64; k++)
        if (!ho_files[k]) {
            ho_files[k] = fopen(name, "wb");
            if (!ho_files[k]) return 1;
            *fh = k;
            return 0;
        }
    return 1;
}
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence) {
    (void)whence;
    return fseek(ho_files[fh], offset, SEEK_SET);
}
int MPI_File_iwrite(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Request *req) {
    if (req) *req = 0;
    return fwrite(buf, (size_t)type, (size_t)count, ho_files[fh]) == (size_t)count ? 0 : 1;
}
int MPI_File_iwrite_all(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Request *req) {
    return MPI_File_iwrite(fh, buf, count, type, req);
}
int MPI_File_close(MPI_File *fh) {
    if (ho_files[*fh]) fclose(ho_files[*fh]);
    ho_files[*fh] = NULL;
    return 0;
}
int MPI_Wait(MPI_Request *req, MPI_Status *status) { (void)req; (void)status; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t)count * (size_t)type);
    return 0;
}

/* ---- globals of the writers (decs.h declarations) ---- */
int BS1_read, BS2_read, BS3_read;
double *Bufferp_1[NB_LOCAL], *Bufferps_1[NB_LOCAL], *Bufferpsh_1[NB_LOCAL];
double DTd, DTl;
int DTr;
MPI_Status Statbound[NB_LOCAL][600];
double accreted_mass, t_prev;
float *array[NB_LOCAL], *array_reduced[NB_LOCAL], *array_diag[NB_LOCAL];
double *array_rdump[NB_LOCAL], *array_gdump1[NB_LOCAL], *array_gdump2[NB_LOCAL], *array_gdump1_reduced[NB_LOCAL],
    *array_gdump2_reduced[NB_LOCAL];
int *array_gdumpgrid, *array_rdumpgrid;
int (*block_read)[10];
gpuStream_t commandQueueGPU[NB_LOCAL];
int dump_cnt, dump_cnt_reduced;
int (*restrict failimage[NB_LOCAL])[NFAIL];
MPI_File fdump[2000], fdump_reduced[2000], fdumpdiag[2000], rdump[NB_LOCAL], gdump[NB_LOCAL], gdump_reduced[NB_LOCAL],
    grid_dump[1], grid_restart[1];
int first_dump, first_dump_reduced, first_rdump, first_gdump, restart_number;
int fix_mem[NB_LOCAL];
FILE *fparam_dump, *fparam_dump_reduced, *fparam_restart;
double mass_density_scale_cpu, metric_scale_cpu, magnetic_density_scale_cpu, mdot_cpu, t_mdot;
MPI_Comm mpi_cartcomm, mpi_self;
int n_active, *n_active_node, n_active_total, n_max;
int (*n_ord_node)[NB_LOCAL];
int nstep;
int numtasks, rank, local_rank, rc;
double *p_1[NB_LOCAL], *ps_1[NB_LOCAL];
double (*restrict p[NB_LOCAL])[NPR];
double (*restrict ps[NB_LOCAL])[NDIM];
double (*restrict psh[NB_LOCAL])[NDIM];
int rdump_cnt;
int read_NS, read_M1, read_M1_2, read_2T, read_Pnum, read_Res, read_Ye, read_nuclear, read_neutrinos;
MPI_Request req_block[NB_LOCAL][1], req_block_reduced[NB_LOCAL][1], req_block_rdump[NB_LOCAL][1],
    req_blockdiag[NB_LOCAL][1], req_gdump1[NB_LOCAL][1], req_gdump2[NB_LOCAL][1], req_gdump1_reduced[NB_LOCAL][1],
    req_gdump2_reduced[NB_LOCAL][1], req_rdumpgrid[1];
double t, tf;

int index_3D(int n, int i, int j, int z) {
    return ((i - N1_GPU_offset[n] + N1G) * (BS_2 + 2 * N2G) + (j - N2_GPU_offset[n] + N2G)) * (BS_3 + 2 * N3G) +
           (z - N3_GPU_offset[n] + N3G);
}

/* Writes the three files of one block, state in the device layout
 * (primitives NPR planes, face field 3 planes, plane stride ks), metric tables
 * in the device layout (gcov/gcon planes s*5 + loc, gdet planes loc, stride
 * gs): the reference's host tables are filled from them (get_geometry reads
 * those), the run parameters dump_params writes are set from the arguments.
 * Returns 0 on success. */
int ref_dump_files(const double *pv, const double *psv, long ks, const double *gcov_t, const double *gcon_t,
                   const double *gdet_t, long gs, const double *prm_d, const int *prm_i, const char *param_path,
                   const char *dump_path, const char *rdump_path) {
    static const int SI[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
    static const int SJ[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
    const long G1 = BS_1 + 2 * N1G, G2 = BS_2 + 2 * N2G, G3 = BS_3 + 2 * N3G, ncell = G1 * G2 * G3;
    nl[0] = 0;
    n_ord[0] = 0;
    n_active = n_active_total = 1;
    n_max = 0;
    numtasks = 1;
    static int nan_node[1];
    static int ord_node[1][NB_LOCAL];
    nan_node[0] = 1;
    ord_node[0][0] = 0;
    n_active_node = nan_node;
    n_ord_node = ord_node;
    for (int k = 0; k < NV; k++) block[0][k] = 0;
    N1_GPU_offset[0] = N2_GPU_offset[0] = N3_GPU_offset[0] = 0;
    /* prm_d: t, dt, DTd, DTl, startx1-3, dx1-3, tf, a, gam, cour, Rin, Rout, R0;
     * prm_i: nstep, dump_cnt, rdump_cnt, failed, lim, dump_cnt_reduced */
    t = prm_d[0]; dt = prm_d[1]; DTd = prm_d[2]; DTl = prm_d[3]; DTr = 0;
    for (int d = 1; d < 4; d++) { startx[d] = prm_d[3 + d]; dx[0][d] = prm_d[6 + d]; }
    tf = prm_d[10]; a = prm_d[11]; gam = prm_d[12]; cour = prm_d[13];
    Rin = prm_d[14]; Rout = prm_d[15]; R0 = prm_d[16];
    nstep = prm_i[0]; dump_cnt = prm_i[1]; rdump_cnt = prm_i[2]; failed = prm_i[3]; lim = prm_i[4];
    dump_cnt_reduced = prm_i[5];
    gcov[0] = malloc(sizeof(*gcov[0]) * G1 * G2);
    gcon[0] = malloc(sizeof(*gcon[0]) * G1 * G2);
    gdet[0] = malloc(sizeof(*gdet[0]) * G1 * G2);
    for (long idx = 0; idx < G1 * G2; idx++)
        for (int loc = 0; loc < NPG; loc++) {
            for (int q = 0; q < 10; q++) {
                const double cv = gcov_t[(long)(q * 5 + loc) * gs + idx], cn = gcon_t[(long)(q * 5 + loc) * gs + idx];
                gcov[0][idx][loc][SI[q]][SJ[q]] = gcov[0][idx][loc][SJ[q]][SI[q]] = cv;
                gcon[0][idx][loc][SI[q]][SJ[q]] = gcon[0][idx][loc][SJ[q]][SI[q]] = cn;
            }
            gdet[0][idx][loc] = gdet_t[(long)loc * gs + idx];
        }
    p[0] = malloc(sizeof(*p[0]) * ncell);
    ps[0] = malloc(sizeof(*ps[0]) * ncell);
    array[0] = malloc(sizeof(float) * NPRDUMP * BS_1 * BS_2 * BS_3);
    array_rdump[0] = malloc(sizeof(double) * (NPR + NDIM) * ncell);
    for (long c = 0; c < ncell; c++) {
        for (int k = 0; k < NPR; k++) p[0][c][k] = pv[(long)k * ks + c];
        ps[0][c][0] = 0.;
        for (int k = 1; k < NDIM; k++) ps[0][c][k] = psv[(long)(k - 1) * ks + c];
    }
    int rcode = 0;
    FILE *fp = fopen(param_path, "wb");
    if (!fp) rcode = 1;
    else {
        dump_params(fp, 0);
        fclose(fp);
    }
    MPI_File fh;
    if (!rcode && MPI_File_open(0, dump_path, 0, 0, &fh) == 0) {
        dump_block(&fh, 0);
        MPI_File_close(&fh);
    } else rcode = rcode ? rcode : 2;
    if (!rcode && MPI_File_open(0, rdump_path, 0, 0, &fh) == 0) {
        rdump_block_write(&fh, 0);
        MPI_File_close(&fh);
    } else rcode = rcode ? rcode : 3;
    free(p[0]); free(ps[0]); free(array[0]); free(array_rdump[0]);
    free(gcov[0]); free(gcon[0]); free(gdet[0]);
    return rcode;
}
