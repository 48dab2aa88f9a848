// Batched ensembles: many independent blocks (different sizes, spins, grids)
// advanced together, one launch per phase of the sub-step for the whole
// ensemble. Included at the end of hamr_kernels.cu (same translation unit):
// the per-item bodies (flux_face, k_cons_at, ...) are the ones the
// single-block kernels run, so a block advances identically alone or in a
// batch.
//
// Work layout. Each phase has, per block, a count of work items (faces,
// zones, edges or ghost columns). Items are cut into tiles of `tile` items;
// the tiles of all blocks form one index space, blocks concatenated in a
// schedule order. A launch runs `grid` CTAs of BLK threads; CTA b takes tiles
// b, b + grid, ... (grid == number of tiles: one tile per CTA; smaller grids:
// persistent CTAs). A tile never straddles two blocks, so the CFL minimum of
// a tile goes to its own block's slot. Tile size, grid and schedule order are
// chosen per phase by the autotuner (hamr_batch_autotune) or default to one
// BLK-item tile per CTA in the caller's order.

namespace {

// everything one block's kernels touch; the step-size slots point into the
// batch's own contiguous arrays
struct BEntry {
    Dims d;
    Geom m;
    double *p, *ph, *ps, *psh, *U, *F1, *F2, *F3, *Ec, *emf, *W;
    int *pflag, *failimage;
    int *nfail, *kerr;           // the block's failed-zone count; the batch's error word
    unsigned long long *dtbits;  // 4 per block
    double *ndt, *dt_state;      // 1 per block
    int *counter;                // 1 per block
};

struct StageArg {
    int full;      // 0: half sub-step (writes ph, psh), 1: full (writes p, ps)
    int calc_dt;   // collect the CFL minimum (full sub-step)
    double frac;   // Dt = frac * dt of each block
};

__device__ __forceinline__ StepSize entry_step(const BEntry &e, const StageArg &a) {
    return StepSize{e.dt_state, a.frac, 0., 0.};
}

// ---- phases: item count per block and the item body ----------------------
enum { PH_FLUX3, PH_FLUX2, PH_FLUX1, PH_FIXFLUX, PH_EMFC, PH_EMFE, PH_POLE, PH_FACE, PH_CONS, PH_INV,
       PH_BX1, PH_BX3, PH_BX2, PH_N };

__host__ __device__ inline long phase_items(int ph, const Dims &d) {
    switch (ph) {
    case PH_FLUX3: return d.d3 ? n_faces<3>(d) : 0;
    case PH_FLUX2: return n_faces<2>(d);
    case PH_FLUX1: return n_faces<1>(d);
    case PH_FIXFLUX: return d.bc2 == HAMR_BC_POLE_REFL ? n_fix_flux(d) : 0;
    case PH_EMFC: return (long)(d.n1 + 2 * d.d1) * (d.n2 + 2 * d.d2) * (d.n3 + 2 * d.d3);
    case PH_EMFE:
    case PH_FACE: return (long)(d.n1 + d.d1) * (d.n2 + d.d2) * (d.n3 + d.d3);
    case PH_POLE: return d.bc2 == HAMR_BC_POLE_TRANS ? 2L * (d.n1 + d.ng1) : 0;
    case PH_CONS:
    case PH_INV: return (long)d.n1 * d.n2 * d.n3;
    case PH_BX1: return d.d1 ? (long)d.ng1 * d.G2 * d.G3 : 0;
    case PH_BX3: return d.d3 ? n_bound_x3(d) : 0;
    case PH_BX2: return d.d2 ? n_bound_x2(d) : 0;
    }
    return 0;
}

template <int DIR, typename T, int REC>
struct OpFlux {
    static constexpr int PH = DIR == 3 ? PH_FLUX3 : (DIR == 2 ? PH_FLUX2 : PH_FLUX1);
    static constexpr int MINB = sizeof(T) == 8 ? HAMR_FLUX_MINB : HAMR_FLUX_MINB_F;
    static constexpr bool REDUCE = true;
    static constexpr int SLOT = DIR;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        T *F = reinterpret_cast<T *>(DIR == 1 ? e.F1 : (DIR == 2 ? e.F2 : e.F3));
        return dt_of_ctop(e.d, DIR, flux_face<DIR, T, REC>(e.d, e.m, a.full ? e.ph : e.p, a.full ? e.psh : e.ps, F, t));
    }
};

template <typename T>
struct OpFixFlux {
    static constexpr int PH = PH_FIXFLUX, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &, long t) {
        fix_flux_at(e.d, reinterpret_cast<T *>(e.F1), reinterpret_cast<T *>(e.F2), reinterpret_cast<T *>(e.F3), t);
        return 1.e9;
    }
};

template <typename T>
struct OpEmfCentre {
    static constexpr int PH = PH_EMFC, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_emf_centre_at(e.d, e.m, a.full ? e.ph : e.p, reinterpret_cast<T *>(e.Ec), t);
        return 1.e9;
    }
};

template <typename T>
struct OpEmfEdge {
    static constexpr int PH = PH_EMFE, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &, long t) {
        k_emf_edge_at(e.d, reinterpret_cast<const T *>(e.Ec), reinterpret_cast<const T *>(e.F1),
                      reinterpret_cast<const T *>(e.F2), reinterpret_cast<const T *>(e.F3),
                      reinterpret_cast<T *>(e.emf), t);
        return 1.e9;
    }
};

template <typename T>
struct OpPole {
    static constexpr int PH = PH_POLE, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_pole_average_at(e.d, reinterpret_cast<T *>(e.emf), entry_step(e, a), t);
        return 1.e9;
    }
};

template <typename T>
struct OpFace {
    static constexpr int PH = PH_FACE, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_face_update_at(e.d, e.m, e.ps, a.full ? e.ps : e.psh, reinterpret_cast<const T *>(e.emf),
                         entry_step(e, a), t);
        return 1.e9;
    }
};

template <typename T>
struct OpCons {
    static constexpr int PH = PH_CONS, MINB = HAMR_CONS_MINB, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_cons_at(e.d, e.m, e.p, a.full ? e.ph : e.p, e.U, reinterpret_cast<const T *>(e.F1),
                  reinterpret_cast<const T *>(e.F2), reinterpret_cast<const T *>(e.F3), e.W, a.full,
                  entry_step(e, a), t);
        return 1.e9;
    }
};

template <int INV, int FIX>
// (the batched inversion keeps 5 blocks per SM: its tiles measured slower at
// the single-block kernel's 6)
struct OpInvert {
    static constexpr int PH = PH_INV, MINB = 5, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_invert_at<INV, FIX>(e.d, e.m, a.full ? e.ph : e.p, e.W, a.full ? e.ps : e.psh, a.full ? e.p : e.ph,
                              e.pflag, e.failimage, t);
        return 1.e9;
    }
};

// The conserved update phase with the single-block kernel's bulk-copy
// staging (cons_tma_row): one CTA per row piece of a block, rstart[k] the
// first CTA of block k (every block 3-D with n3 >= 32 and aligned flux
// planes). Same values as OpCons. (The primary inversion inside, as the
// single-block kernel runs it, measured slower here: rows of 32-96 zones.)
// resident CTAs (of up to 256 threads) per SM, FP64 / float fluxes; on the
// 64-torus ensemble (rows of 32-96 zones) the float update took 2.37 ms per
// sub-step at 3 (80 registers), 2.61 at 4 (64), and at 5 (48 registers,
// 0.7 KB of spills) lost to the tiled update
#ifndef HAMR_BATCH_CONS_TMA_MINB
#define HAMR_BATCH_CONS_TMA_MINB HAMR_CONS_TMA_MINB
#endif
#ifndef HAMR_BATCH_CONS_TMA_MINB_F
#define HAMR_BATCH_CONS_TMA_MINB_F HAMR_CONS_TMA_MINB_F
#endif
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? HAMR_BATCH_CONS_TMA_MINB : HAMR_BATCH_CONS_TMA_MINB_F)
    k_batch_cons_tma(const BEntry *__restrict__ E, const long *__restrict__ rstart, int n, const StageArg a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ BEntry e;
    int lo = 0, hi = n;   // rstart[lo] <= blockIdx.x < rstart[lo + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (rstart[mid] <= (long)blockIdx.x) lo = mid;
        else hi = mid;
    }
    {
        const int *src = reinterpret_cast<const int *>(&E[lo]);
        int *dst = reinterpret_cast<int *>(&e);
        for (int k = threadIdx.x; k < (int)(sizeof(BEntry) / 4); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int npiece = (e.d.n3 + 255) / 256, lpiece = (e.d.n3 + npiece - 1) / npiece;
    cons_tma_row<T, 0>(e.d, e.m, e.p, a.full ? e.ph : e.p, e.U, reinterpret_cast<const T *>(e.F1),
                       reinterpret_cast<const T *>(e.F2), reinterpret_cast<const T *>(e.F3), e.W, a.full,
                       entry_step(e, a), e.nfail, e.kerr, npiece, lpiece, (int)(blockIdx.x - rstart[lo]), smem,
                       nullptr, nullptr, nullptr, nullptr, nullptr);
}

// The x3 fluxes of the batch by zone slots, with the centre EMFs: the
// single-block slot kernel's body (flux_x3_slots), each zone reconstructed
// once. The blocks' CTA ranges are concatenated, xstart[k] the first CTA of
// block k (every block 3-D). Same values as OpFlux<3> and OpEmfCentre.
template <typename T, int REC>
__global__ void __launch_bounds__(BLK, sizeof(T) == 8 ? ((REC & 2) != 0 ? HAMR_FLUX_FT_X3_MINB : HAMR_FLUX_X3_MINB)
                                                         : ((REC & 2) != 0 ? HAMR_FLUX_FT_X3_MINB_F : HAMR_FLUX_X3_MINB_F))
    k_batch_flux_x3(const BEntry *__restrict__ E, const long *__restrict__ xstart, int n, const StageArg a) {
    __shared__ BEntry e;
    int lo = 0, hi = n;   // xstart[lo] <= blockIdx.x < xstart[lo + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xstart[mid] <= (long)blockIdx.x) lo = mid;
        else hi = mid;
    }
    {
        const int *src = reinterpret_cast<const int *>(&E[lo]);
        int *dst = reinterpret_cast<int *>(&e);
        for (int k = threadIdx.x; k < (int)(sizeof(BEntry) / 4); k += BLK) dst[k] = src[k];
    }
    __syncthreads();
    const double cmx = flux_x3_slots<T, REC>(e.d, e.m, a.full ? e.ph : e.p, a.full ? e.psh : e.ps,
                                             reinterpret_cast<T *>(e.F3), reinterpret_cast<T *>(e.Ec),
                                             (long)blockIdx.x - xstart[lo]);
    if (a.calc_dt) cta_max_ctop(e.d, 3, cmx, &e.dtbits[3]);
}

struct OpBoundX1 {
    static constexpr int PH = PH_BX1, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_bound_x1_at(e.d, e.m, a.full ? e.p : e.ph, a.full ? e.ps : e.psh, t);
        return 1.e9;
    }
};

struct OpBoundX3 {
    static constexpr int PH = PH_BX3, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_bound_x3_at(e.d, a.full ? e.p : e.ph, a.full ? e.ps : e.psh, t);
        return 1.e9;
    }
};

struct OpBoundX2 {
    static constexpr int PH = PH_BX2, MINB = 1, SLOT = 0;
    static constexpr bool REDUCE = false;
    __device__ static double run(const BEntry &e, const StageArg &a, long t) {
        k_bound_x2_at(e.d, a.full ? e.p : e.ph, a.full ? e.ps : e.psh, t);
        return 1.e9;
    }
};

}  // namespace

namespace {

// tile space of one phase: start[k] = first tile of the k-th block in the
// schedule, order[k] = that block's index in the batch
struct TileMap {
    const long *start;   // n + 1 entries
    const int *order;    // n entries
    int n;
    int tile;            // items per tile
};

template <class Op>
__global__ void __launch_bounds__(BLK, Op::MINB) k_batch(const BEntry *__restrict__ E, const TileMap tm,
                                                          const StageArg a) {
    // the tile's block description, staged in shared memory: the bodies read
    // sizes, strides and pointers from there instead of holding them in registers
    __shared__ BEntry e;
    const long ntiles = tm.start[tm.n];
    for (long w = blockIdx.x; w < ntiles; w += gridDim.x) {
        int lo = 0, hi = tm.n;   // start[lo] <= w < start[lo + 1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tm.start[mid] <= w) lo = mid;
            else hi = mid;
        }
        __syncthreads();   // the previous tile is done with e
        {
            static_assert(sizeof(BEntry) % 4 == 0, "BEntry copied as words");
            const int *src = reinterpret_cast<const int *>(&E[tm.order[lo]]);
            int *dst = reinterpret_cast<int *>(&e);
            for (int k = threadIdx.x; k < (int)(sizeof(BEntry) / 4); k += BLK) dst[k] = src[k];
        }
        __syncthreads();
        const long first = (w - tm.start[lo]) * tm.tile;
        const long cnt = phase_items(Op::PH, e.d);
        const long last = first + tm.tile < cnt ? first + tm.tile : cnt;
        double dtf = 1.e9;
        for (long t = first + threadIdx.x; t < last; t += BLK) dtf = d_min(dtf, Op::run(e, a, t));
        if (Op::REDUCE && a.calc_dt) cta_min_dt(dtf, &e.dtbits[Op::SLOT]);
    }
}

// one thread per block of the batch
__global__ void k_batch_dt_reset(const BEntry *__restrict__ E, int n) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    for (int k = 0; k < 4; k++) E[b].dtbits[k] = BITS_1E9;
}

// per block: the CFL step of the full sub-step, and (advance mode) the
// step-size update min(ndt, 1.3 dt) every `interval` steps, as k_dt_finalize
__global__ void k_batch_dt_finalize(const BEntry *__restrict__ E, int n, int update, int interval) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const BEntry &e = E[b];
    const double d1 = __longlong_as_double((long long)e.dtbits[1]);
    const double d2 = __longlong_as_double((long long)e.dtbits[2]);
    const double d3 = __longlong_as_double((long long)e.dtbits[3]);
    const double ndt = 1. / (1. / d1 + 1. / d2 + 1. / d3);
    *e.ndt = ndt;
    if (update) {
        const int c = ++(*e.counter);
        if (interval <= 1 || c % interval == 0) {
            const double dt = *e.dt_state;
            *e.dt_state = ndt > 1.3 * dt ? 1.3 * dt : ndt;
        }
    }
    for (int k = 0; k < 4; k++) e.dtbits[k] = BITS_1E9;
}

// ---- one persistent launch per sub-step ------------------------------------
// The alternative to one launch per phase: a cooperative launch of as many
// CTAs as fit on the device at once runs every phase of a sub-step, phase
// after phase, each CTA taking tiles b, b + grid, ... of the phase's tile
// map, with a grid-wide barrier wherever the next phase reads what the
// previous wrote (x3/x2/x1 fluxes and centre EMFs | polar flux fix | edge
// EMFs and conserved update | polar EMF average | face update | inversion |
// ghost fills x1 | x3 | x2). The cost is one register budget for all phases
// (the FP64 flux's), instead of each phase's own.

struct PhaseMaps {
    TileMap tm[PH_N];
};

// the tile loop of k_batch for one phase, inside the persistent kernel
template <class Op>
__device__ __forceinline__ void run_phase(const BEntry *__restrict__ E, const TileMap &tm, const StageArg &a,
                                          BEntry &e) {
    if (tm.start == nullptr) return;   // no items in this phase
    const long ntiles = tm.start[tm.n];
    for (long w = blockIdx.x; w < ntiles; w += gridDim.x) {
        int lo = 0, hi = tm.n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tm.start[mid] <= w) lo = mid;
            else hi = mid;
        }
        __syncthreads();
        {
            const int *src = reinterpret_cast<const int *>(&E[tm.order[lo]]);
            int *dst = reinterpret_cast<int *>(&e);
            for (int k = threadIdx.x; k < (int)(sizeof(BEntry) / 4); k += BLK) dst[k] = src[k];
        }
        __syncthreads();
        const long first = (w - tm.start[lo]) * tm.tile;
        const long cnt = phase_items(Op::PH, e.d);
        const long last = first + tm.tile < cnt ? first + tm.tile : cnt;
        double dtf = 1.e9;
        for (long t = first + threadIdx.x; t < last; t += BLK) dtf = d_min(dtf, Op::run(e, a, t));
        if (Op::REDUCE && a.calc_dt) cta_min_dt(dtf, &e.dtbits[Op::SLOT]);
    }
}

// Grid-wide barrier of a cooperative launch (all CTAs resident): bar[0]
// counts arrivals, bar[1] is the generation. Thread 0 publishes the CTA's
// writes (fence), arrives, and waits for the generation to move, at most
// 2^24 polls of 64 ns; a wait that gives up sets *kerr = 2 and goes on (the
// sub-step's results are then invalid and the host reports the error).
__device__ __forceinline__ void grid_barrier(unsigned *bar, int *kerr) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1 == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            for (int it = 0; *gen == g; it++) {
                if (it >= (1 << 24)) {
                    atomicExch(kerr, 2);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

constexpr int PERSIST_MINB = HAMR_FLUX_MINB;   // the FP64 flux phases' budget

template <typename T>
__global__ void __launch_bounds__(BLK, PERSIST_MINB)
    k_batch_stage(const BEntry *__restrict__ E, const PhaseMaps pm, const StageArg a, unsigned *bar, int *kerr) {
    __shared__ BEntry e;
    auto has = [&](int ph) { return pm.tm[ph].start != nullptr && pm.tm[ph].n > 0; };
    run_phase<OpFlux<3, T, 0>>(E, pm.tm[PH_FLUX3], a, e);
    run_phase<OpFlux<2, T, 0>>(E, pm.tm[PH_FLUX2], a, e);
    run_phase<OpFlux<1, T, 0>>(E, pm.tm[PH_FLUX1], a, e);
    run_phase<OpEmfCentre<T>>(E, pm.tm[PH_EMFC], a, e);
    grid_barrier(bar, kerr);
    if (has(PH_FIXFLUX)) {
        run_phase<OpFixFlux<T>>(E, pm.tm[PH_FIXFLUX], a, e);
        grid_barrier(bar, kerr);
    }
    run_phase<OpEmfEdge<T>>(E, pm.tm[PH_EMFE], a, e);
    run_phase<OpCons<T>>(E, pm.tm[PH_CONS], a, e);
    grid_barrier(bar, kerr);
    if (has(PH_POLE)) {
        run_phase<OpPole<T>>(E, pm.tm[PH_POLE], a, e);
        grid_barrier(bar, kerr);
    }
    run_phase<OpFace<T>>(E, pm.tm[PH_FACE], a, e);
    grid_barrier(bar, kerr);
    run_phase<OpInvert<HAMR_INV_2D, 0>>(E, pm.tm[PH_INV], a, e);
    grid_barrier(bar, kerr);
    run_phase<OpBoundX1>(E, pm.tm[PH_BX1], a, e);
    grid_barrier(bar, kerr);
    run_phase<OpBoundX3>(E, pm.tm[PH_BX3], a, e);
    grid_barrier(bar, kerr);
    run_phase<OpBoundX2>(E, pm.tm[PH_BX2], a, e);
}

}  // namespace

// ===========================================================================
struct hamr_batch {
    int n = 0;
    int precision = 0, recon = 0, inversion = 0, riemann = 0;
    int fix = 0;   // FIX_* bits of the inversion phase (opt-in floors, reset of failed zones)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nsm = 148;
    std::string err;
    std::vector<hamr_ctx *> ctx;
    BEntry *E = nullptr;                    // device, n entries
    unsigned long long *dtbits = nullptr;   // device, 4n
    double *dts = nullptr, *ndts = nullptr; // device, n each
    int *counters = nullptr;                // device, n
    std::vector<long> items[PH_N];          // host: work items per block and phase
    long ntiles[PH_N] = {};
    long *dstart[PH_N] = {};                // device tile maps
    int *dorder[PH_N] = {};
    int tile[PH_N], grid[PH_N], order_mode[PH_N];
    float tuned_ms[PH_N] = {};
    cudaGraphExec_t graph = nullptr;
    int graph_steps = -1, graph_interval = -1;
    // one persistent launch per sub-step (hamr_batch_set_persistent)
    // conserved update phase with bulk-copy staging (k_batch_cons_tma): every
    // block allows it (cons_tma_ok) and it is in use (cons_tma: by default in
    // the mixed step; the autotuner times it against the tiled update)
    bool cons_tma_ok = false, cons_tma = false;
    // x3 fluxes and centre EMFs by zone slots (k_batch_flux_x3): every block
    // 3-D; off with HAMR_BATCH_FLUX_X3=0
    bool flux3_slots = false;
    long *xstart = nullptr;      // device, n + 1: first CTA of each block
    long nx3_ctas = 0;
    long *rstart = nullptr;      // device, n + 1: first CTA of each block
    long ncons_ctas = 0;
    int cons_block = 0;          // threads per CTA: the longest row piece, in warps
    size_t cons_smem = 0;        // dynamic shared memory: the longest piece's layout
    bool persistent = false;
    int persist_grid = 0;        // CTAs of the cooperative launch
    unsigned *bar = nullptr;     // grid barrier: arrivals, generation
    int *kerr = nullptr;         // set when a barrier wait gave up
};

namespace {

int bfail(hamr_batch *b, cudaError_t e, const char *what) {
    b->err = std::string(what) + ": " + cudaGetErrorString(e);
    return HAMR_E_CUDA;
}

#define BCK(call)                                               \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return bfail(b, e_, #call);      \
    } while (0)

// tile map of one phase from its tuning: schedule order (0: as given, 1:
// largest block first), tiles of `tile` items, prefix over the schedule
int build_tiles(hamr_batch *b, int ph) {
    const int n = b->n;
    std::vector<int> order(n);
    for (int k = 0; k < n; k++) order[k] = k;
    if (b->order_mode[ph] == 1)
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return b->items[ph][x] > b->items[ph][y]; });
    std::vector<long> start(n + 1, 0);
    const long tl = b->tile[ph];
    for (int k = 0; k < n; k++) start[k + 1] = start[k] + (b->items[ph][order[k]] + tl - 1) / tl;
    b->ntiles[ph] = start[n];
    BCK(cudaMemcpyAsync(b->dstart[ph], start.data(), sizeof(long) * (n + 1), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->dorder[ph], order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, b->stream));
    // the host vectors go out of scope: finish the copies first
    BCK(cudaStreamSynchronize(b->stream));
    return HAMR_OK;
}

template <class Op>
void launch_phase(hamr_batch *b, const StageArg &a) {
    const int ph = Op::PH;
    const long nt = b->ntiles[ph];
    if (nt == 0) return;
    const long g = b->grid[ph] > 0 && b->grid[ph] < nt ? b->grid[ph] : nt;
    k_batch<Op><<<(unsigned)g, BLK, 0, b->stream>>>(b->E, TileMap{b->dstart[ph], b->dorder[ph], b->n, b->tile[ph]}, a);
}

unsigned nblk_b(int n) { return (unsigned)((n + 127) / 128); }

// launches phase `only` (or every phase when only < 0) of one sub-step
template <typename T, int REC, int INV>
void batch_stage_t(hamr_batch *b, int full, bool calc_dt, int only) {
    const StageArg a{full, calc_dt ? 1 : 0, full ? 1.0 : 0.5};
    auto want = [&](int ph) { return only < 0 || only == ph; };
    if (want(PH_FLUX3)) {
        if (b->flux3_slots)
            k_batch_flux_x3<T, REC><<<(unsigned)b->nx3_ctas, BLK, 0, b->stream>>>(b->E, b->xstart, b->n, a);
        else
            launch_phase<OpFlux<3, T, REC>>(b, a);
    }
    if (want(PH_FLUX2)) launch_phase<OpFlux<2, T, REC>>(b, a);
    if (want(PH_FLUX1)) launch_phase<OpFlux<1, T, REC>>(b, a);
    if (want(PH_FIXFLUX)) launch_phase<OpFixFlux<T>>(b, a);
    if (want(PH_EMFC) && !b->flux3_slots) launch_phase<OpEmfCentre<T>>(b, a);   // else done by the x3 slots
    if (want(PH_EMFE)) launch_phase<OpEmfEdge<T>>(b, a);
    if (want(PH_POLE)) launch_phase<OpPole<T>>(b, a);
    if (want(PH_FACE)) launch_phase<OpFace<T>>(b, a);
    if (want(PH_CONS)) {
        if (b->cons_tma)
            k_batch_cons_tma<T><<<(unsigned)b->ncons_ctas, b->cons_block, b->cons_smem, b->stream>>>(b->E, b->rstart,
                                                                                                 b->n, a);
        else
            launch_phase<OpCons<T>>(b, a);
    }
    if (want(PH_INV)) {
        switch (b->fix) {
            case FIX_FLOORS: launch_phase<OpInvert<INV, FIX_FLOORS>>(b, a); break;
            case FIX_RESET: launch_phase<OpInvert<INV, FIX_RESET>>(b, a); break;
            case FIX_FLOORS | FIX_RESET: launch_phase<OpInvert<INV, FIX_FLOORS | FIX_RESET>>(b, a); break;
            default: launch_phase<OpInvert<INV, 0>>(b, a);
        }
    }
    if (want(PH_BX1)) launch_phase<OpBoundX1>(b, a);
    if (want(PH_BX3)) launch_phase<OpBoundX3>(b, a);
    if (want(PH_BX2)) launch_phase<OpBoundX2>(b, a);
}

template <typename T, int REC>
void batch_stage_r(hamr_batch *b, int full, bool calc_dt, int only) {
    if (b->inversion == HAMR_INV_NM) batch_stage_t<T, REC, HAMR_INV_NM>(b, full, calc_dt, only);
    else batch_stage_t<T, REC, HAMR_INV_2D>(b, full, calc_dt, only);
}

template <typename T>
void batch_stage_p(hamr_batch *b, int full, bool calc_dt, int only) {
    switch (b->recon | (b->riemann << 1)) {
    case 1: batch_stage_r<T, 1>(b, full, calc_dt, only); break;
    case 2: batch_stage_r<T, 2>(b, full, calc_dt, only); break;
    case 3: batch_stage_r<T, 3>(b, full, calc_dt, only); break;
    default: batch_stage_r<T, 0>(b, full, calc_dt, only); break;
    }
}

void batch_stage(hamr_batch *b, int full, bool calc_dt, int only = -1) {
    if (b->precision == HAMR_MIXED) batch_stage_p<float>(b, full, calc_dt, only);
    else batch_stage_p<double>(b, full, calc_dt, only);
}


// one sub-step of every block in one cooperative launch (k_batch_stage)
int batch_stage_persistent(hamr_batch *b, int full, bool calc_dt) {
    PhaseMaps pm;
    for (int ph = 0; ph < PH_N; ph++)
        pm.tm[ph] = b->ntiles[ph] ? TileMap{b->dstart[ph], b->dorder[ph], b->n, b->tile[ph]}
                                  : TileMap{nullptr, nullptr, 0, BLK};
    StageArg a{full, calc_dt ? 1 : 0, full ? 1.0 : 0.5};
    const BEntry *E = b->E;
    void *args[] = {(void *)&E, (void *)&pm, (void *)&a, (void *)&b->bar, (void *)&b->kerr};
    const void *fn = b->precision == HAMR_MIXED ? (const void *)k_batch_stage<float>
                                                : (const void *)k_batch_stage<double>;
    BCK(cudaMemsetAsync(b->bar, 0, 2 * sizeof(unsigned), b->stream));
    BCK(cudaLaunchCooperativeKernel(fn, dim3(b->persist_grid), dim3(BLK), args, 0, b->stream));
    return HAMR_OK;
}

// the batch's error word, read after the caller's synchronisation and
// cleared: 2 from a grid barrier of the persistent kernel that gave up, 1 from
// a bulk-copy wait of k_batch_cons_tma that gave up
int batch_check_kerr(hamr_batch *b) {
    if (!b->kerr) return HAMR_OK;
    int v = 0;
    BCK(cudaMemcpyAsync(&v, b->kerr, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (!v) return HAMR_OK;
    BCK(cudaMemsetAsync(b->kerr, 0, sizeof(int), b->stream));
    b->err = v == 2 ? "a grid barrier of the persistent sub-step timed out (the step's results are invalid)"
                    : "a bulk-copy wait of the conserved update gave up (the step's results are invalid)";
    return HAMR_E_CUDA;
}

// one RK2 step of every block: step sizes from b->dts (frac 1/2, then 1)
int batch_step_launch(hamr_batch *b, int update, int interval) {
    if (b->persistent) {
        int rc = batch_stage_persistent(b, 0, false);
        if (!rc) rc = batch_stage_persistent(b, 1, true);
        if (rc) return rc;
        k_batch_dt_finalize<<<nblk_b(b->n), 128, 0, b->stream>>>(b->E, b->n, update, interval);
        BCK(cudaGetLastError());
        return HAMR_OK;
    }
    batch_stage(b, 0, false);
    batch_stage(b, 1, true);
    k_batch_dt_finalize<<<nblk_b(b->n), 128, 0, b->stream>>>(b->E, b->n, update, interval);
    BCK(cudaGetLastError());
    return HAMR_OK;
}

// The x3 slot kernel (k_batch_flux_x3) when every block is 3-D: CTAs per
// block as the single-block launch.
int batch_setup_flux3_slots(hamr_batch *b) {
    b->flux3_slots = false;
    if (const char *e = getenv("HAMR_BATCH_FLUX_X3"))
        if (atoi(e) == 0) return HAMR_OK;
    std::vector<long> xs(b->n + 1, 0);
    for (int k = 0; k < b->n; k++) {
        const Dims &d = b->ctx[k]->d;
        if (!d.d3) return HAMR_OK;
        xs[k + 1] = xs[k] + n_x3_slot_ctas(d);
    }
    if (xs[b->n] > 0x7fffffffL) return HAMR_OK;
    BCK(cudaMemcpyAsync(b->xstart, xs.data(), sizeof(long) * (b->n + 1), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));   // xs goes out of scope
    b->nx3_ctas = xs[b->n];
    b->flux3_slots = true;
    return HAMR_OK;
}

// The bulk-copy update phase (k_batch_cons_tma) when every block allows it,
// as a single block decides for itself: 3-D, n3 >= 32, flux planes 16-byte
// aligned, the block's own switch on (HAMR_CONS_TMA). CTAs per block: its
// row pieces; block size and shared memory: the longest piece's.
template <typename T>
int batch_setup_cons_tma(hamr_batch *b) {
    b->cons_tma_ok = b->cons_tma = false;
    std::vector<long> rs(b->n + 1, 0);
    int block = 0;
    int sm = 0;
    for (int k = 0; k < b->n; k++) {
        hamr_ctx *c = b->ctx[k];
        const Dims &d = c->d;
        if (!(c->cons_tma && d.d3 && d.n3 >= 32 &&
              cons_tma_aligned<T>(c, d, reinterpret_cast<const T *>(c->F1), reinterpret_cast<const T *>(c->F2),
                                  reinterpret_cast<const T *>(c->F3))))
            return HAMR_OK;
        const int npiece = (d.n3 + 255) / 256, lpiece = (d.n3 + npiece - 1) / npiece;
        rs[k + 1] = rs[k] + (long)d.n1 * d.n2 * npiece;
        block = std::max(block, (lpiece + 31) / 32 * 32);
        sm = std::max(sm, cons_tma_layout<T>(lpiece).total);
    }
    if (rs[b->n] > 0x7fffffffL) return HAMR_OK;   // more CTAs than one launch's grid holds
    BCK(cudaFuncSetAttribute(k_batch_cons_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    BCK(cudaMemcpyAsync(b->rstart, rs.data(), sizeof(long) * (b->n + 1), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));   // rs goes out of scope
    b->ncons_ctas = rs[b->n];
    b->cons_block = block;
    b->cons_smem = (size_t)sm;
    b->cons_tma_ok = true;
    // measured on the 64-torus ensemble (rows of 32-96 zones), per sub-step:
    // float fluxes 2.37 ms against 2.69 for the tiled update; FP64 3.20
    // against 2.59 (the FP64 staging holds 6 CTAs of at most 96 threads per SM)
    b->cons_tma = sizeof(T) == 4;
    if (const char *e = getenv("HAMR_BATCH_CONS_TMA")) b->cons_tma = atoi(e) != 0;   // 1: also FP64; 0: off
    return HAMR_OK;
}

}  // namespace

extern "C" {

int hamr_batch_create(hamr_ctx *const *blocks, int n, void *stream, hamr_batch **out) {
    if (!blocks || !out || n < 1) return HAMR_E_ARG;
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        if (!blocks[k]) return HAMR_E_ARG;
        if (!blocks[k]->have_geom) return HAMR_E_STATE;
        const hamr_params &p0 = blocks[0]->prm, &pk = blocks[k]->prm;
        // one instantiation of every phase kernel serves the whole batch
        if (pk.precision != p0.precision || pk.recon != p0.recon || pk.inversion != p0.inversion ||
            pk.riemann != p0.riemann)
            return HAMR_E_ARG;
        if (pk.halo) return HAMR_E_ARG;   // members are whole problems: no neighbours to exchange with
        if (pk.riemann == HAMR_RIEMANN_HLLD) return HAMR_E_ARG;   // HLLD steps one block at a time
        // one inversion instantiation for all members; the neighbour repair
        // (its scan and one-CTA chain per block) steps one block at a time
        if (pk.floors != p0.floors || pk.repair != p0.repair || pk.repair == 2) return HAMR_E_ARG;
        for (int j = 0; j < k; j++)
            if (blocks[j] == blocks[k]) return HAMR_E_ARG;
    }
    hamr_batch *b = new hamr_batch();
    b->n = n;
    b->precision = blocks[0]->prm.precision;
    b->recon = blocks[0]->prm.recon;
    b->inversion = blocks[0]->prm.inversion;
    b->fix = (blocks[0]->prm.floors ? FIX_FLOORS : 0) | (blocks[0]->prm.repair == 1 ? FIX_RESET : 0);
    b->riemann = blocks[0]->prm.riemann;
    b->ctx.assign(blocks, blocks + n);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { delete b; return HAMR_E_CUDA; }
        b->own_stream = true;
    }
    bool ok = cudaMalloc(&b->E, sizeof(BEntry) * n) == cudaSuccess &&
              cudaMalloc(&b->dtbits, sizeof(unsigned long long) * 4 * n) == cudaSuccess &&
              cudaMalloc(&b->dts, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&b->ndts, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&b->counters, sizeof(int) * n) == cudaSuccess &&
              cudaMalloc(&b->kerr, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&b->rstart, sizeof(long) * (n + 1)) == cudaSuccess &&
              cudaMalloc(&b->xstart, sizeof(long) * (n + 1)) == cudaSuccess;
    for (int ph = 0; ph < PH_N && ok; ph++)
        ok = cudaMalloc(&b->dstart[ph], sizeof(long) * (n + 1)) == cudaSuccess &&
             cudaMalloc(&b->dorder[ph], sizeof(int) * n) == cudaSuccess;
    if (!ok) {
        hamr_batch_destroy(b);
        return HAMR_E_NOMEM;
    }
    std::vector<BEntry> host(n);
    for (int k = 0; k < n; k++) {
        hamr_ctx *c = blocks[k];
        BEntry &e = host[k];
        e.d = c->d;
        e.m = geom_of(c);
        e.p = c->p; e.ph = c->ph; e.ps = c->ps; e.psh = c->psh; e.U = c->U;
        e.F1 = c->F1; e.F2 = c->F2; e.F3 = c->F3; e.Ec = c->Ec; e.emf = c->emf; e.W = c->W;
        e.pflag = c->pflag; e.failimage = c->failimage;
        e.dtbits = b->dtbits + 4 * k;
        e.ndt = b->ndts + k;
        e.dt_state = b->dts + k;
        e.counter = b->counters + k;
        e.nfail = c->nfail;
        e.kerr = b->kerr;
        for (int ph = 0; ph < PH_N; ph++) b->items[ph].push_back(phase_items(ph, c->d));
    }
    int rc = HAMR_OK;
    // the members' own streams may still be filling their state
    for (hamr_ctx *c : b->ctx)
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = HAMR_E_CUDA;
    if (rc == HAMR_OK &&
        cudaMemcpyAsync(b->E, host.data(), sizeof(BEntry) * n, cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
        rc = HAMR_E_CUDA;
    for (int ph = 0; ph < PH_N && rc == HAMR_OK; ph++) {
        b->tile[ph] = BLK;      // default: one BLK-item tile per CTA, caller's order
        b->grid[ph] = 0;
        b->order_mode[ph] = 0;
        rc = build_tiles(b, ph);
    }
    if (rc == HAMR_OK && cudaMemsetAsync(b->kerr, 0, sizeof(int), b->stream) != cudaSuccess) rc = HAMR_E_CUDA;
    if (rc == HAMR_OK)
        rc = b->precision == HAMR_MIXED ? batch_setup_cons_tma<float>(b) : batch_setup_cons_tma<double>(b);
    if (rc == HAMR_OK) rc = batch_setup_flux3_slots(b);
    if (rc == HAMR_OK) {
        k_batch_dt_reset<<<nblk_b(n), 128, 0, b->stream>>>(b->E, n);
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) rc = HAMR_E_CUDA;
    }
    if (rc) {
        hamr_batch_destroy(b);
        return rc;
    }
    *out = b;
    return HAMR_OK;
}

int hamr_batch_destroy(hamr_batch *b) {
    if (!b) return HAMR_E_ARG;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->E);
    cudaFree(b->dtbits);
    cudaFree(b->dts);
    cudaFree(b->ndts);
    cudaFree(b->counters);
    cudaFree(b->bar);
    cudaFree(b->kerr);
    cudaFree(b->rstart);
    cudaFree(b->xstart);
    for (int ph = 0; ph < PH_N; ph++) {
        cudaFree(b->dstart[ph]);
        cudaFree(b->dorder[ph]);
    }
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HAMR_OK;
}

const char *hamr_batch_last_error(hamr_batch *b) { return b ? b->err.c_str() : "null batch"; }

int hamr_batch_step(hamr_batch *b, const double *dt, double *dt_next) {
    if (!b || !dt) return HAMR_E_ARG;
    for (int k = 0; k < b->n; k++)
        if (!(dt[k] > 0)) return HAMR_E_ARG;
    BCK(cudaMemcpyAsync(b->dts, dt, sizeof(double) * b->n, cudaMemcpyHostToDevice, b->stream));
    k_batch_dt_reset<<<nblk_b(b->n), 128, 0, b->stream>>>(b->E, b->n);
    int rc = batch_step_launch(b, 0, 0);
    if (rc) return rc;
    if ((b->persistent || b->cons_tma_ok) && (rc = batch_check_kerr(b))) return rc;
    if (dt_next) {
        BCK(cudaMemcpyAsync(dt_next, b->ndts, sizeof(double) * b->n, cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        for (int k = 0; k < b->n; k++)
            if (!(dt_next[k] > 0) || !isfinite(dt_next[k])) {
                b->err = "non-finite or non-positive CFL step in block " + std::to_string(k);
                return HAMR_E_PHYSICS;
            }
    }
    return HAMR_OK;
}

int hamr_batch_advance(hamr_batch *b, int nsteps, int interval, double *dt_inout) {
    if (!b || !dt_inout || nsteps < 1 || interval < 1) return HAMR_E_ARG;
    for (int k = 0; k < b->n; k++)
        if (!(dt_inout[k] > 0)) return HAMR_E_ARG;
    BCK(cudaMemcpyAsync(b->dts, dt_inout, sizeof(double) * b->n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemsetAsync(b->counters, 0, sizeof(int) * b->n, b->stream));
    k_batch_dt_reset<<<nblk_b(b->n), 128, 0, b->stream>>>(b->E, b->n);
    if (!b->graph || b->graph_steps != nsteps || b->graph_interval != interval) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaGraph_t g;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = HAMR_OK;
        for (int s = 0; s < nsteps && rc == HAMR_OK; s++) rc = batch_step_launch(b, 1, interval);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return bfail(b, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, e, "cudaGraphInstantiate");
        b->graph_steps = nsteps;
        b->graph_interval = interval;
    }
    BCK(cudaGraphLaunch(b->graph, b->stream));
    BCK(cudaMemcpyAsync(dt_inout, b->dts, sizeof(double) * b->n, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return b->persistent || b->cons_tma_ok ? batch_check_kerr(b) : HAMR_OK;
}

// One persistent cooperative launch per sub-step instead of one launch per
// phase (PPM, HLL, Noble 2D, no floors or repair; the tile maps stay those
// of the autotuner or the default). The grid is every CTA the device can
// hold at once at the kernel's register budget.
int hamr_batch_set_persistent(hamr_batch *b, int on) {
    if (!b) return HAMR_E_ARG;
    if (!on) {
        b->persistent = false;
    } else {
        if (b->recon != HAMR_RECON_PPM || b->riemann != HAMR_RIEMANN_HLL || b->inversion != HAMR_INV_2D || b->fix)
            return HAMR_E_ARG;
        int dev = 0, coop = 0, per_sm = 0;
        BCK(cudaGetDevice(&dev));
        BCK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        if (!coop) {
            b->err = "the device does not support cooperative launches";
            return HAMR_E_CUDA;
        }
        const void *fn = b->precision == HAMR_MIXED ? (const void *)k_batch_stage<float>
                                                    : (const void *)k_batch_stage<double>;
        BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, BLK, 0));
        if (per_sm < 1) {
            b->err = "the persistent sub-step kernel does not fit on a multiprocessor";
            return HAMR_E_CUDA;
        }
        if (!b->bar) BCK(cudaMalloc(&b->bar, 2 * sizeof(unsigned)));
        if (!b->kerr) BCK(cudaMalloc(&b->kerr, sizeof(int)));
        BCK(cudaMemsetAsync(b->bar, 0, 2 * sizeof(unsigned), b->stream));
        BCK(cudaMemsetAsync(b->kerr, 0, sizeof(int), b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        b->persist_grid = per_sm * b->nsm;
        b->persistent = true;
    }
    if (b->graph) {   // the captured advance holds the other launch form
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_steps = b->graph_interval = -1;
    }
    return HAMR_OK;
}

// Picks, phase by phase in stage order, the tile size, grid and schedule
// order with the shortest device time for this batch: every candidate runs
// the phase of a half sub-step `reps` times after one warm-up launch, timed
// with CUDA events on the batch stream. Half sub-steps only write the
// intermediate arrays (ph, psh, fluxes, EMFs, U cache, scratch), so p and ps
// are untouched; the inversion failure counters are cleared afterwards.
int hamr_batch_autotune(hamr_batch *b, const double *dt, int reps) {
    if (!b || !dt || reps < 1) return HAMR_E_ARG;
    for (int k = 0; k < b->n; k++)
        if (!(dt[k] > 0)) return HAMR_E_ARG;
    BCK(cudaMemcpyAsync(b->dts, dt, sizeof(double) * b->n, cudaMemcpyHostToDevice, b->stream));
    const int tiles[] = {BLK, 4 * BLK, 16 * BLK, 64 * BLK};
    const int grids[] = {0, 2 * b->nsm, 4 * b->nsm, 8 * b->nsm, 16 * b->nsm};
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    int rc = HAMR_OK;
    for (int ph = 0; ph < PH_N && rc == HAMR_OK; ph++) {
        long work = 0;
        for (long x : b->items[ph]) work += x;
        if (work == 0 || (ph == PH_EMFC && b->flux3_slots)) continue;   // nothing launched
        // the x3 slot kernel has one launch shape: timed once
        const bool fixed = ph == PH_FLUX3 && b->flux3_slots;
        bool timed = false;
        float best = 1e30f;
        int bt = b->tile[ph], bg = b->grid[ph], bo = b->order_mode[ph];
        // device ms of the phase's current launch form, < 0 on a CUDA error
        auto time_phase = [&]() -> float {
            batch_stage(b, 0, false, ph);   // warm-up
            cudaEventRecord(e0, b->stream);
            for (int r = 0; r < reps; r++) batch_stage(b, 0, false, ph);
            cudaEventRecord(e1, b->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            return ms / reps;
        };
        // the conserved update's bulk-copy kernel is one more candidate (its
        // launch shape is fixed)
        bool tma_best = false;
        if (ph == PH_CONS && b->cons_tma_ok) {
            b->cons_tma = true;
            const float ms = time_phase();
            if (ms < 0) rc = bfail(b, cudaGetLastError(), "autotune");
            else { best = ms; tma_best = true; }
            b->cons_tma = false;
        }
        for (int om = 0; om < 2 && rc == HAMR_OK; om++)
            for (int tl : tiles)
                for (int gr : grids) {
                    b->tile[ph] = tl;
                    b->grid[ph] = gr;
                    b->order_mode[ph] = om;
                    if ((rc = build_tiles(b, ph))) break;
                    if (gr > 0 && gr >= b->ntiles[ph]) continue;   // same launch as one tile per CTA
                    if (fixed && timed) continue;
                    timed = true;
                    const float ms = time_phase();
                    if (ms < 0) { rc = bfail(b, cudaGetLastError(), "autotune"); break; }
                    if (ms < best) { best = ms; bt = tl; bg = gr; bo = om; tma_best = false; }
                }
        if (ph == PH_CONS) b->cons_tma = tma_best;
        b->tile[ph] = bt;
        b->grid[ph] = bg;
        b->order_mode[ph] = bo;
        b->tuned_ms[ph] = best;
        if (rc == HAMR_OK) rc = build_tiles(b, ph);
        if (rc == HAMR_OK) batch_stage(b, 0, false, ph);   // leave this phase's outputs for the next phase
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (hamr_ctx *c : b->ctx) BCK(cudaMemsetAsync(c->failimage, 0, 4 * sizeof(int) * c->d.ks, b->stream));
    k_batch_dt_reset<<<nblk_b(b->n), 128, 0, b->stream>>>(b->E, b->n);
    BCK(cudaStreamSynchronize(b->stream));
    if (b->graph) {   // launch shapes changed
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return HAMR_OK;
}

// Chosen launch shape of each phase (HAMR_BATCH_PHASES entries each): items
// per tile, grid (0: one tile per CTA), schedule order (0: as given, 1:
// largest block first), and the tuned device time of the phase in ms (0 when
// not tuned). Any output pointer may be NULL.
int hamr_batch_tuning(hamr_batch *b, int *tile, int *grid, int *order, float *ms, int nphases) {
    if (!b || nphases < PH_N) return HAMR_E_ARG;
    for (int ph = 0; ph < PH_N; ph++) {
        if (tile)
            tile[ph] = (ph == PH_CONS && b->cons_tma) || ((ph == PH_FLUX3 || ph == PH_EMFC) && b->flux3_slots)
                           ? 0 : b->tile[ph];
        if (grid) grid[ph] = b->grid[ph];
        if (order) order[ph] = b->order_mode[ph];
        if (ms) ms[ph] = b->tuned_ms[ph];
    }
    return HAMR_OK;
}

}  // extern "C"
