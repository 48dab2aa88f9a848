/*
 * hamr_b200.h -- C ABI of the B200 (sm_100a) single-block GRMHD step.
 *
 * This is the drop-in boundary for H-AMR's per-block device step. In the
 * reference the step is driven by advance_GPU() (step_ch.c:997) and
 * GPU_step_ch() (step_ch.c:916), which launch the per-block launchers
 * GPU_fluxcalc2D / GPU_fix_flux / GPU_consttransport1-3 / GPU_fixup
 * (GPU_main.cu:560,1126,1365,1393,1535,1740) on global buffers allocated by
 * set_arrays_GPU (GPU_mem.h:41) and filled by GPU_write / GPU_write_metric
 * (GPU_main.cu:309,139). Here the same work sits behind an explicit context:
 * no globals, plain pointers and sizes, return code 0 or a negative HAMR_E_*.
 *
 * Memory layout (identical to the reference device layout, GPU_program1.cu:90-94):
 *   cell arrays  plane k holds variable k (RHO, UU, U1, U2, U3, B1, B2, B3, KTOT);
 *                cell (i, j, z) of the ghosted block sits at (i*G2 + j)*G3 + z with
 *                G1 = n1 + 2*ng, G2 = n2 + 2*ng, G3 = n3 + 2*ng (G3 = 1 when n3 == 1);
 *                planes are ksize doubles apart.
 *   face field   3 planes; plane d-1 holds B^d (no sqrt(-g)) on the lower d-face.
 *   metric       gcov/gcon: plane (s*5 + loc), s the symmetric component
 *                (00,01,02,03,11,12,13,22,23,33), loc in {FACE1, FACE2, CORN, CENT,
 *                FACE3}; gdet: plane loc; conn: plane (s*4 + l) holding
 *                Gamma^l_{s}; every plane indexed (i*G2 + j), gsize doubles apart
 *                (GPU_main.cu:139-300).
 * Every entry point is thread-safe per context; contexts are independent.
 */
#ifndef HAMR_B200_H
#define HAMR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HAMR_NPR 9

enum hamr_status {
    HAMR_OK = 0,
    HAMR_E_ARG = -1,       /* invalid argument or size */
    HAMR_E_CUDA = -2,      /* a CUDA runtime call failed (see hamr_last_error) */
    HAMR_E_NOMEM = -3,     /* device allocation failed */
    HAMR_E_STATE = -4,     /* call out of order (e.g. stepping before geometry) */
    HAMR_E_PHYSICS = -5    /* non-finite or non-positive CFL step */
};

enum hamr_bc {
    HAMR_BC_PERIODIC = 0,
    HAMR_BC_OUTFLOW = 1,    /* copy + no-inflow check (bounds.c:158, GPU_bounds.h:1368) */
    HAMR_BC_POLE_TRANS = 2, /* transmissive polar axis, 3-D (GPU_bounds.h:510) */
    HAMR_BC_POLE_REFL = 3   /* reflective polar axis, 2-D (GPU_bounds.h:305) */
};

enum hamr_precision {
    HAMR_FP64 = 0,          /* everything in double */
    HAMR_MIXED = 1          /* reconstruction, Riemann flux and EMF in float; metric,
                               source, compensated update and inversion in double */
};

enum hamr_inversion {
    HAMR_INV_2D = 0,        /* Noble 2D Newton (Utoprim_2d, the shipped default) */
    HAMR_INV_NM = 1         /* Newman-Hamlin (Utoprim_NM, GPU_fixup.h:323, NEWMAN builds) */
};                          /* either way failures fall back to 1dvsq2fix1 then 1dfix1 */

enum hamr_recon {
    HAMR_RECON_PPM = 0,     /* PPM para (GPU_interp.h:60-111, PPM builds; ng = 3) */
    HAMR_RECON_MC = 1       /* linear MC slope_lim, factor 2 (GPU_interp.h:2-38, PPM = 0
                               builds; ng = 2 as there, or 3) */
};

enum hamr_riemann {
    HAMR_RIEMANN_HLL = 0,   /* HLL (fluxcalc2D2, the shipped default, HLLC 0) */
    HAMR_RIEMANN_HLLC = 1,  /* HLLC in the orthonormal face frame with its HLL fallback
                               and hydrodynamic sub-case (fluxcalc2D_FT, GPU_hllc.h:3) */
    HAMR_RIEMANN_HLLD = 2   /* HLLD there (calc_HLLD, GPU_hllc.h:398-876; HLLD builds,
                               marked "Does not work yet", config.h:482), falling back to
                               HLLC, then HLL, where its wave fan fails a check; single
                               blocks only (batches refuse it) */
};

typedef struct hamr_params {
    int n1, n2, n3;         /* active cells per direction (n3 == 1: 2-D, x1-x2) */
    int ng;                 /* ghost layers: 3 (NG = 2 + PPM, config.h:1280); 2 allowed with MC */
    long ksize;             /* plane stride of cell arrays; 0: reference rule G + 64 - G%64 */
    long gsize;             /* plane stride of metric tables; 0: reference rule */
    double dx1, dx2, dx3;   /* coordinate spacing */
    double gam;             /* adiabatic index */
    double cour;            /* Courant factor (COUR, config.h:455) */
    int pole1, pole2;       /* lower/upper x2 edge is a polar axis (POLE_1/2, GPU_main.cu:566) */
    int bc1, bc2, bc3;      /* enum hamr_bc per direction */
    int ct_upwind;          /* 1: upwinded edge EMFs (GR default); 0: face-EMF average
                               (the reference's CARTESIAN build, GPU_const_trans.h:187) */
    int precision;          /* enum hamr_precision */
    void *stream;           /* cudaStream_t to run on; NULL: the context creates one */
    int inversion;          /* enum hamr_inversion (zero-initialised: Noble 2D) */
    int recon;              /* enum hamr_recon (zero-initialised: PPM) */
    int riemann;            /* enum hamr_riemann (zero-initialised: HLL) */
    int halo;               /* sides shared with a neighbouring block of a decomposed
                               domain: bit 0 the lower x1 side, bit 1 the upper, bit 2
                               the lower x2 side, bit 3 the upper (zero-initialised:
                               none). No physical ghost fill and no radial mass-flux
                               fix there; an x2 halo side is no pole (pole1/pole2 0
                               there) and bc2 is not periodic. Such a block steps
                               through hamr_stage, hamr_bound_dim and the hamr_halo_*
                               exchange (the reference's block exchange, boundcomP.c) */
    int floors;             /* 1: drift-frame floors on rho, u and the velocity after the
                               inversion, with the Lorentz factor capped at 80 (fixup_cell's
                               body, GPU_fixup.h:1025-1800, compiled out in the reference;
                               zero-initialised: off, as the reference ships). A zone
                               whose Lorentz factor cannot be formed gets pflag -333
                               and counter 3 (GPU_fixup.h:398-415) */
    int repair;             /* zones whose inversion failed (pflag != 0) after each sub-step:
                               0 left as the solvers left them (the reference's step);
                               1 reset to rho = u = 1e-20 with zero velocity, then floored
                               when floors is on (fixuputoprim, GPU_fixup.h:735-852);
                               2 replaced by the average of good neighbours, in (i, j, z)
                               order, flags cleared (fixup_utoprim, fixup.c:764-827);
                               no usable stencil: counter 4. Mode 2 is refused for halo
                               blocks and in batches, and allocates one int per active
                               zone. Batch members share floors and repair */
} hamr_params;

typedef struct hamr_ctx hamr_ctx;

/* Create a context on the current CUDA device and allocate its device state.
 * Replaces set_arrays_GPU (GPU_mem.h:41-). */
int hamr_ctx_create(const hamr_params *params, hamr_ctx **out);
int hamr_ctx_destroy(hamr_ctx *ctx);
/* Text of the last error recorded on ctx (never NULL). */
const char *hamr_last_error(const hamr_ctx *ctx);
/* Plane strides chosen at creation. */
int hamr_strides(const hamr_ctx *ctx, long *ksize, long *gsize);

/* Upload host metric tables (layout above). Replaces GPU_write_metric
 * (GPU_main.cu:139). */
int hamr_set_geometry(hamr_ctx *ctx, const double *gcov, const double *gcon,
                      const double *gdet, const double *conn);

/* Host -> device copy of primitives (NPR planes) and face field (3 planes),
 * ghost zones included. Replaces GPU_write (GPU_main.cu:309). */
int hamr_upload(hamr_ctx *ctx, const double *p, const double *ps);
/* Device -> host copy of the current primitives and face field. Replaces
 * GPU_read (GPU_main.cu:2646). */
int hamr_download(hamr_ctx *ctx, double *p, double *ps);
/* Device -> host copy of the inversion flags (1 int plane) and failure
 * counters (5 int planes, NFAIL of config.h:1307: 2D failed, 1dvsq2fix1
 * failed, 1dfix1 failed, floor gamma failure, neighbour repair without a
 * usable stencil; GPU_fixup.h:360-415, fixup.c:819). Either pointer may be
 * NULL. */
int hamr_download_flags(hamr_ctx *ctx, int *pflag, int *failimage);

/* Ghost fill of the current state (GPU_boundprim, GPU_main.cu:2113). */
int hamr_bound(hamr_ctx *ctx);

/* ---- decomposed domains (halo != 0) ---------------------------------------
 * Such a block's hamr_stage leaves the ghost fill to the caller, which runs,
 * for the state the sub-step wrote (full: p, ps; else ph, psh), along x1:
 *   hamr_bound_dim(1)  physical x1 sides
 *   hamr_halo_pack on both neighbours' facing sides, transfer, hamr_halo_unpack
 *   hamr_bound_dim(3), hamr_bound_dim(2)
 * and along x2:
 *   hamr_bound_dim(1), hamr_bound_dim(3), hamr_bound_dim(2)  (poles, physical sides)
 *   the x2 halo exchange (sides 2, 3)
 * the order in which a single block fills x1, x3, x2 ghosts, so that the
 * decomposed step reproduces the undivided block bit for bit. The step size is
 * the harmonic combination 1/(1/d1 + 1/d2 + 1/d3) of the per-direction CFL
 * minima over all blocks (hamr_cfl_dirs after each block's full sub-step).
 * hamr_step, hamr_advance and hamr_profile_step refuse halo blocks. */
int hamr_bound_dim(hamr_ctx *ctx, int full, int dim);
/* Doubles a halo message buffer needs: the larger of an x1 side's
 * (NPR + 3) x ng x G2 x G3, laid out [component][layer][j][z], and an x2
 * side's (NPR + 3) x ng x G1 x G3, laid out [component][layer][i][z]. */
long hamr_halo_count(const hamr_ctx *ctx);
/* side 0: the lower x1 side, 1: the upper, 2: the lower x2 side, 3: the
 * upper. pack copies the ng active layers next to that side into buf (device
 * memory, hamr_halo_count doubles); unpack writes buf into the ghost layers
 * beyond that side. Asynchronous on the context stream. */
int hamr_halo_pack(hamr_ctx *ctx, int full, int side, double *buf);
int hamr_halo_unpack(hamr_ctx *ctx, int full, int side, const double *buf);
/* Per-direction CFL minima (x1, x2, x3; 1e9 for an inactive direction) of
 * the last full sub-step run by hamr_stage; waits for the device. */
int hamr_cfl_dirs(hamr_ctx *ctx, double *dt3);

/* One RK2 sub-step on the device, asynchronous on the context stream:
 * full == 0 advances (p, ps) by Dt into (ph, psh) and caches U(p);
 * full == 1 advances the cached U by Dt with the fluxes of (ph, psh) into (p, ps).
 * dt is the step size (polar EMF averaging scales by it, GPU_boundcomE.cu:58).
 * The written state gets its ghost zones filled. Replaces one advance_GPU()
 * call plus GPU_boundprim(0) (step_ch.c:926-936). */
int hamr_stage(hamr_ctx *ctx, int full, double Dt, double dt);

/* Whole RK2 step of size dt (half then full sub-step). When dt_next is not
 * NULL the call waits for the device and returns the CFL step of the full
 * sub-step, 1/(1/dt1 + 1/dt2 + 1/dt3) (step_ch.c:1320-1331). */
int hamr_step(hamr_ctx *ctx, double dt, double *dt_next);

/* nsteps RK2 steps with the step size kept in device memory: every
 * `interval` steps it becomes min(CFL step, 1.3 * dt) (the SAFE growth limit,
 * step_ch.c:973-975; interval 16 mirrors AMR_MAXTIMELEVEL). The sequence is
 * captured once into a CUDA graph per (nsteps, interval) and replayed.
 * dt_inout: in, the first step size; out, the step size after the last step
 * (this waits for the device). */
int hamr_advance(hamr_ctx *ctx, int nsteps, int interval, double *dt_inout);

/* Per-kernel-group device times of `reps` RK2 steps of size dt (the state
 * advances), averaged per step, from CUDA events recorded between the groups
 * on the context stream: ms[0..10] = x3 flux, x2 flux, x1 flux, polar flux
 * fix, centre EMF, edge EMF, polar EMF average, face update, conserved
 * update, inversion, ghost fill. nslots must be >= 11. */
int hamr_profile_step(hamr_ctx *ctx, double dt, int reps, double *ms, int nslots);

/* Device pointers of the live state, for zero-copy access (e.g. DLPack or
 * torch.from_blob in a test harness). Any pointer argument may be NULL. */
int hamr_device_state(hamr_ctx *ctx, double **p, double **ps, double **ph, double **psh);

/* ---- allocation-free step --------------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that may
 * not allocate device memory at all -- code running inside someone else's
 * CUDA graph capture (an allocation would break the capture), or a host
 * framework that owns every byte of HBM through its own pool and forbids
 * stray cudaMalloc calls. hamr_ctx_create allocates the whole working set, so
 * those callers use this instead: one RK2 step (half and full sub-step, ghost
 * fills) of a block whose state and metric tables the caller already holds in
 * device memory (layout as above; p, ps advanced in place; gcov/gcon/gdet/conn
 * read only). Every intermediate array lives in static device arrays inside
 * this library, sized for at most HAMR_NOALLOC_MAX_CELLS zones per plane
 * (ksize, ghosts and padding included; about 17 MB held on every GPU that
 * loads the library, until the process exits). Larger blocks are rejected with
 * HAMR_E_ARG before any device work. Nothing is allocated: no cudaMalloc,
 * cudaFree, stream or event creation.
 *   - runs on prm->stream (NULL: the legacy default stream);
 *   - accepts PPM or MC reconstruction, HLL or HLLC, Noble 2D or
 *     Newman-Hamlin inversion, every boundary kind; refuses with HAMR_E_ARG
 *     precision other than HAMR_FP64, riemann == HAMR_RIEMANN_HLLD,
 *     floors != 0, repair != 0 and halo != 0 (those need arrays or passes
 *     this step does not carry);
 *   - the first call on a device looks up the device addresses of the static
 *     arrays (cudaGetSymbolAddress); make that first call outside any stream
 *     capture;
 *   - all calls share the same arrays, which keep the previous call's
 *     contents (the ones read before written are cleared each call): calls
 *     that overlap on the GPU, from any thread or stream, race;
 *   - dt_next: when not NULL, the call waits for the device and returns the
 *     CFL step of the full sub-step, as hamr_step does. */
#define HAMR_NOALLOC_MAX_CELLS 32768
int hamr_step_noalloc(const hamr_params *prm, const double *gcov, const double *gcon,
                      const double *gdet, const double *conn, double *p, double *ps,
                      double dt, double *dt_next);

/* max over active cells of |div B| of the current face field, definition of
 * divb_calc (diag.c:153-199); waits for the device. */
int hamr_divb_max(hamr_ctx *ctx, double *out);

/* ---- host geometry builder (no device needed) ----------------------------
 * Fills metric tables for a block of n1 x n2 x n3 active cells in the layout
 * above, following set_grid (main.c:380-455):
 *   coords == 0: Kerr-Schild metric of spin `spin` in the reference's code
 *                coordinates (X1 = log r, uniform theta map, X3 = phi;
 *                vofx_matthewcoords, coord.c:147) with the Jacobian and the
 *                connection by central differences (metric.c:427-519);
 *   coords == 1: Minkowski in Cartesian code coordinates (CARTESIAN build).
 * startx/dx are 4-vectors (index 0 unused). gsize 0: reference rule. */
int hamr_build_geometry(int coords, double spin, int n1, int n2, int n3, int ng, long gsize,
                        const double *startx, const double *dx,
                        double *gcov, double *gcon, double *gdet, double *conn);
/* Boyer-Lindquist (r, theta, phi) of a code-coordinate point (bl_coord, coord.c:111). */
int hamr_bl_coord(int coords, double spin, const double *X, double *rthph);

/* ---- batched ensembles -----------------------------------------------------
 * A batch advances many independent blocks -- uneven sizes, spins, grids --
 * together: each phase of a sub-step (three face-flux directions, polar flux
 * fix, centre and edge EMFs, polar EMF average, face update, conserved update,
 * inversion, three ghost fills) is ONE launch for the whole ensemble, whose
 * CTAs walk a tile space covering every block. The reference steps blocks one
 * after another, a launch sequence per block (GPU_step_ch, step_ch.c:916-990,
 * looping over n_active blocks); independent problems there are separate
 * runs. Each block keeps its own step size: arrays of n doubles below are
 * indexed like `blocks`.
 *
 * Members are existing contexts with geometry set; they must share precision,
 * reconstruction and inversion. The batch runs on its own stream (`stream`, or
 * one it creates when NULL) and uses the members' device arrays: do not step a
 * member through its context while the batch is in use. */
typedef struct hamr_batch hamr_batch;

#define HAMR_BATCH_PHASES 13

int hamr_batch_create(hamr_ctx *const *blocks, int n, void *stream, hamr_batch **out);
int hamr_batch_destroy(hamr_batch *b);
const char *hamr_batch_last_error(hamr_batch *b);

/* One RK2 step of every block with its own dt[k]; dt_next[k] (may be NULL)
 * receives each block's CFL step, as hamr_step. */
int hamr_batch_step(hamr_batch *b, const double *dt, double *dt_next);

/* nsteps RK2 steps of every block with the per-block step-size refresh of
 * hamr_advance, replayed from one captured CUDA graph per (nsteps, interval).
 * dt_inout[k]: in, block k's first step size; out, its step size after the
 * last step (waits for the device). */
int hamr_batch_advance(hamr_batch *b, int nsteps, int interval, double *dt_inout);

/* Autotuner: times each phase over candidate launch shapes (items per tile,
 * persistent grid size or one tile per CTA, schedule order as given or
 * largest block first) on this batch, probe step sizes dt[k], `reps` timed
 * launches per candidate, and keeps the fastest. Leaves p and ps untouched. */
int hamr_batch_autotune(hamr_batch *b, const double *dt, int reps);

/* One persistent cooperative launch per sub-step (on != 0) instead of one
 * launch per phase: every CTA the device holds at once runs all phases of the
 * sub-step, with a grid-wide barrier (bounded waits; a wait that gives up is
 * reported as HAMR_E_CUDA) wherever a phase reads what the previous wrote.
 * For PPM, HLL, Noble 2D, no floors or repair (else HAMR_E_ARG); the phases
 * keep their tile maps. Replaces the role of GPU_step_ch's per-kernel
 * launches (step_ch.c:916-1335) for a whole ensemble; no reference
 * counterpart. */
int hamr_batch_set_persistent(hamr_batch *b, int on);

/* The launch shape chosen for each of the HAMR_BATCH_PHASES phases (order:
 * flux x3, x2, x1, polar flux fix, centre EMF, edge EMF, polar EMF average,
 * face update, conserved update, inversion, ghost fill x1, x3, x2) and its
 * tuned time in ms. tile 0 for the conserved update: one CTA per row of a
 * block with its fluxes staged by bulk copies (every block 3-D with n3 >= 32;
 * the default with float fluxes, and an autotuner candidate); tile 0 for the
 * x3 fluxes and the centre EMFs: the zone-slot kernel, which computes both
 * (every block 3-D). Any output pointer may be NULL. */
int hamr_batch_tuning(hamr_batch *b, int *tile, int *grid, int *order, float *ms, int nphases);

/* ---- adjoint ---------------------------------------------------------------
 * Reverse mode of the FP64 RK2 step (no counterpart in the reference, which
 * has no derivatives), for axisymmetric blocks: n3 == 1, PPM, Noble 2D
 * inversion, outflow x1, reflective polar axis, upwinded CT -- the 2-D torus
 * configuration. Step sizes are held fixed (no derivative through the CFL
 * choice). The objective is J = sum_n w_n Mdot_n with the accretion rate
 * through x1 face column `mdot_face` of the full sub-step,
 * Mdot = -sum_j F1[RHO](mdot_face, j) dx2 dx3 (F1 includes gdet; calc_Mdot,
 * restart.c:864-903, measures the same flux through a sphere).
 * The adjoint holds its cotangent arrays on the device, in the context's
 * layout: ap (9 planes), aps (3 planes), and the accumulated d/d gamma. */
typedef struct hamr_adjoint hamr_adjoint;

int hamr_adjoint_create(hamr_ctx *ctx, int mdot_face, hamr_adjoint **out);
int hamr_adjoint_destroy(hamr_adjoint *a);
const char *hamr_adjoint_last_error(hamr_adjoint *a);
/* device pointers of the state cotangents (any may be NULL) */
int hamr_adjoint_cotangent(hamr_adjoint *a, double **ap, double **aps, double **agam);
int hamr_adjoint_zero(hamr_adjoint *a);

/* C-ABI backward of one RK2 step of size dt. On entry the context holds the
 * step's input state (with ghosts) and ap/aps the cotangent of its output;
 * on return ap/aps hold the cotangent of the input (ghost entries included:
 * they belong to the previous ghost fill), d/d gamma is accumulated, and
 * mdot_weight * Mdot of this step is part of the objective. The context's
 * state is unchanged; its intermediate arrays are overwritten. */
int hamr_step_backward(hamr_adjoint *a, double dt, double mdot_weight);

/* Forward sweep for the objective: ghost fill, then nsteps steps of sizes
 * dt[n] (weights w_n = dt[n]); J receives the objective; the state advances. */
int hamr_mdot_forward(hamr_adjoint *a, int nsteps, const double *dt, double *J);

/* Objective and its gradient w.r.t. the initial state (host arrays in the
 * context's layout, NULL to skip) and gamma, with checkpoints every `every`
 * steps and recompute; the state is left at its initial value. */
int hamr_adjoint_run(hamr_adjoint *a, int nsteps, const double *dt, int every, double *J, double *grad_p,
                     double *grad_ps, double *grad_gam);

#ifdef __cplusplus
}
#endif
#endif /* HAMR_B200_H */
