/*
 * fcc.h — C ABI of the B200-native Fourier contour cell time step.
 *
 * This is the drop-in boundary for the hot path of FourierContourCells.jl: the
 * Julia API `Simulation`, `step!`, `run!`, `compute_gradients!`, `shape_index`
 * (src/FourierContourCells.jl:55-76) becomes a handle plus plain-pointer calls
 * that a Julia `ccall` shim (or Python ctypes) binds.  No C++ or torch types
 * cross this boundary.
 *
 * Conventions that follow the reference so that its callers need no changes:
 *   - body, type and parent ids are 1-based, as in `Bodies` (src/bodies.jl:62-86);
 *   - per-body matrices are column-major with one column per body, e.g. `coef`
 *     is ncoef x N with column i = [a0; a2..aM; b2..bM] of body i
 *     (src/basis.jl:10-14, src/bodies.jl:56), contour arrays are ntheta x N;
 *   - every floating-point value crosses the ABI as double and is converted to
 *     the simulation precision on the way in, as `convert_precision` and
 *     `_convert_eltype` do (src/energies/interface.jl:220-257,
 *     src/simulation.jl:312);
 *   - errors are status codes; FCC_ERR_ARGUMENT and FCC_ERR_DIMENSION are
 *     raised exactly where the reference throws ArgumentError and
 *     DimensionMismatch, and fcc_last_error() returns the message.
 *
 * Ownership: the library copies host arrays in and owns every device buffer;
 * getters copy out into caller buffers.  Each handle owns one CUDA stream.
 * Handles are independent: concurrent handles on separate host threads give
 * the same results as sequential runs (test/test_cuda.jl:187-196).
 */
#ifndef FCC_H
#define FCC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FCC_MAX_TYPES 8   /* body types per simulation (BodyType table) */
#define FCC_MAX_TERMS 16  /* energy terms per simulation */
#define FCC_MAX_MODES 9   /* shape modes n = 2..10, i.e. maxmode <= 10 */

typedef int32_t fcc_status;
enum {
    FCC_OK = 0,
    FCC_ERR_ARGUMENT = 1,    /* reference: ArgumentError */
    FCC_ERR_DIMENSION = 2,   /* reference: DimensionMismatch */
    FCC_ERR_CUDA = 3,        /* CUDA runtime error (message has the CUDA text) */
    FCC_ERR_UNSUPPORTED = 4, /* valid model outside these kernels */
    FCC_ERR_DEVICE = 5,      /* device-side error status (e.g. non-finite state) */
    FCC_ERR_NOMEM = 6,       /* device allocation failed */
    FCC_ERR_FULL = 7         /* pool: no room for this simulation until others leave */
};

/* Energy term kinds (src/energies/body_terms.jl, contact.jl, bonds.jl). */
enum {
    FCC_TENSION = 1,               /* Tension(eta):           a = eta            */
    FCC_PERIMETER_ELASTICITY = 2,  /* PerimeterElasticity(l, p0): a = l, b = p0 */
    FCC_OVERLAP = 3,               /* Overlap(J; related):    J, Jrel tables     */
    FCC_LINEAR_REPULSION = 4,      /* LinearRepulsion(k):     a = k              */
    FCC_HARMONIC_BOND = 5,         /* HarmonicBond(k; r0):    a = k, b = r0      */
    /* user terms compiled into the library (include/fcc_user_terms.h):
     * fcc_term.user is the index in that kind's table, a and b its parameters */
    FCC_USER_BODY = 6,             /* a BodyTerm: integrands q_j(R, R', R''), energy F(Q) */
    FCC_USER_CONTACT = 7,          /* a ContactTerm: pressure g(d), interaction range    */
    FCC_USER_BOND = 8              /* a BondTerm: bond energy gradient                   */
};

/* One energy term.  `ntypes_on > 0` wraps the term in OnTypes(term, types_on...)
 * (src/energies/interface.jl:278-298).  Overlap couplings are nJ x nJ tables,
 * column-major, indexed (type_i, type_j) like the reference's SMatrix
 * (src/energies/contact.jl:12-28); a scalar coupling is nJ = 1.  `user`
 * selects the compiled user term of an FCC_USER_* kind (the reference's
 * user-defined BodyTerm / ContactTerm / BondTerm, src/energies/interface.jl:27-106);
 * at most FCC_MAX_USER_TERMS of each user kind per simulation. */
#define FCC_MAX_USER_TERMS 4
typedef struct {
    int32_t kind;
    int32_t ntypes_on;
    int32_t types_on[FCC_MAX_TYPES];
    double a, b;
    int32_t nJ;
    double J[FCC_MAX_TYPES * FCC_MAX_TYPES];
    double Jrel[FCC_MAX_TYPES * FCC_MAX_TYPES];
    int32_t user;
} fcc_term;

/* BodyType(; v0, Dr, Dt, mu_r, mu_theta, mu_ab, drag) (src/bodies.jl:30-45);
 * parent_drag = 1 is drag = :parent.  maxmode limits the shape modes of this
 * type's bodies to n = 2..maxmode (0: every mode of the simulation; 1: none,
 * rigid circles): modes above it are zero on entry and stay zero.  No
 * counterpart in the reference, where every type shares the simulation's
 * ncoef (docs/nucleus.md:121-122); maxmode = 0 is the reference's behaviour. */
typedef struct {
    double v0, Dr, Dt, mu_r, mu_theta, mu_ab;
    int32_t parent_drag;
    int32_t maxmode;
} fcc_body_type;

/* Keyword arguments of Simulation(bodies, box; ...) (src/simulation.jl:66-68). */
typedef struct {
    double Lx, Ly;            /* PeriodicBox(Lx, Ly) */
    double dt;                /* time step (default 0.005) */
    int32_t ntheta;           /* contour nodes nθ (default 40) */
    int32_t precision;        /* 64: Float64; 32: Float32 bulk, FP64 a0/projection/observables */
    uint64_t seed;            /* Philox key (src/random.jl:103) */
    double skin;              /* Verlet skin (default 0.3) */
    int32_t ntypes;
    const fcc_body_type* types;
    int32_t nterms;
    const fcc_term* terms;
    int64_t nbonds;           /* bonds = [(i, j), ...]; 2*nbonds 1-based ids */
    const int32_t* bonds;
    int32_t nl_capacity;      /* initial neighbour-list capacity (0: 32, as NeighborList) */
} fcc_params;

/* Host body state, the fields of Bodies (src/bodies.jl:62-72). */
typedef struct {
    int64_t n;
    int32_t ncoef;            /* 2K + 1, K = maxmode - 1 */
    double* x;
    double* y;
    double* theta;
    int32_t* imgx;
    int32_t* imgy;
    double* coef;             /* ncoef x n, column-major */
    double* R0;
    int32_t* type;            /* 1-based */
    int32_t* parent;          /* 1-based */
} fcc_bodies_host;

/* Gradient buffers of Gradients (src/gradients.jl:15-38).  Any pointer may be
 * NULL to skip that field. */
typedef struct {
    double* GR;      /* ntheta x n, dE/dR */
    double* GD;      /* ntheta x n, dE/dR' */
    double* GDD;     /* ntheta x n, dE/dR'' */
    double* P;       /* ntheta x n, contact energy density */
    double* gx;      /* n */
    double* gy;      /* n */
    double* gtheta;  /* n */
    double* glab;    /* ncoef x n, dE/dlab / R0 */
    double* gcoef;   /* ncoef x n, body-frame gradient, row 1 = raw dE/da0 */
    double* Ebody;   /* n */
} fcc_gradients_host;

/* Derived geometry of Geometry (src/geometry.jl:13-32); NULL skips a field. */
typedef struct {
    double* lab;     /* ncoef x n */
    double* labR0;   /* ncoef x n */
    double* R;       /* ntheta x n */
    double* dR;      /* ntheta x n */
    double* ddR;     /* ntheta x n */
    double* rmax;    /* n */
} fcc_geometry_host;

/* Cell list and neighbour list (src/neighbors.jl:16-33, 110-127), 1-based as
 * in the reference.  Arrays are sized by the caller from fcc_neighbor_dims. */
typedef struct {
    int32_t* cellid;  /* n, cx + ncx*cy + 1 */
    int32_t* perm;    /* n, bodies sorted stably by cellid */
    int32_t* start;   /* ncx*ncy, empty cells: start = 1, stop = 0 */
    int32_t* stop;    /* ncx*ncy */
    int32_t* idx;     /* cap x n, neighbours of body i in column i */
    int32_t* count;   /* n */
} fcc_neighbors_host;

typedef struct fcc_sim fcc_sim;

/* Callback of fcc_run, called every `every` steps (src/simulation.jl:220-235). */
typedef void (*fcc_callback)(fcc_sim* sim, void* user);

/* Simulation(bodies, box; ...): src/simulation.jl:66-105.  Copies `bodies`
 * to the device, enforces the shape constraints and builds the geometry. */
fcc_status fcc_create(const fcc_params* params, const fcc_bodies_host* bodies, fcc_sim** out);
fcc_status fcc_destroy(fcc_sim* sim);

/* step!(sim, n): src/simulation.jl:165-173 (eager launches, one host sync at the end). */
fcc_status fcc_step(fcc_sim* sim, int64_t n);

/* run!(sim, n; every, callback, graph): src/simulation.jl:220-235 and the CUDA
 * graph driver ext/FourierContourCellsCUDAExt.jl:144-180.  Results equal fcc_step. */
fcc_status fcc_run(fcc_sim* sim, int64_t n, int64_t every, fcc_callback cb, void* user, int32_t graph);

/* update_neighbors!(sim; force): src/simulation.jl:132-142. */
fcc_status fcc_update_neighbors(fcc_sim* sim, int32_t force);

/* compute_gradients!(sim): src/simulation.jl:150-158 (frame = true). */
fcc_status fcc_compute_gradients(fcc_sim* sim);

/* The fields of sim.bodies plus the device clock (Philox draw index), sim.t and sim.step. */
fcc_status fcc_get_state(fcc_sim* sim, fcc_bodies_host* out, int64_t* clock, double* t, int64_t* step);

/* Overwrite the body state (x, y, theta, imgx, imgy, coef; R0, type and parent
 * must match the created ones) and the clock; then enforce_shape!,
 * update_geometry! and an invalidated neighbour list, like the tests' refresh!
 * (test/runtests.jl:9-15). `clock < 0` keeps the clock.  The arrays are read
 * once, as they are; the call returns when they are no longer needed. */
fcc_status fcc_set_state(fcc_sim* sim, const fcc_bodies_host* in, int64_t clock);

/* Page-locked host memory for the arrays of fcc_bodies_host (no counterpart
 * in the reference, whose host arrays are Julia Arrays and whose state stays
 * in CuArrays).  fcc_set_state and fcc_get_state copy the caller's arrays to
 * and from the device as they are, converting on the device; from memory
 * allocated here those copies are direct DMA transfers, from ordinary
 * (pageable) memory the CUDA driver stages them through its own buffers.
 * A maintainer binding Julia would instead pin with CUDA.Mem.pin. */
fcc_status fcc_host_alloc(int64_t bytes, void** out);
fcc_status fcc_host_free(void* ptr);

/* sim.dt = dt (test/test_cuda.jl:156-162). */
fcc_status fcc_set_dt(fcc_sim* sim, double dt);

fcc_status fcc_get_gradients(fcc_sim* sim, const fcc_gradients_host* out);
fcc_status fcc_get_geometry(fcc_sim* sim, const fcc_geometry_host* out);

/* Sizes for fcc_get_neighbors: grid cells, capacity, and sim.neighbors.builds. */
fcc_status fcc_neighbor_dims(fcc_sim* sim, int32_t* ncx, int32_t* ncy, int32_t* cap, int64_t* builds, int32_t* valid);
fcc_status fcc_get_neighbors(fcc_sim* sim, const fcc_neighbors_host* out);

/* perimeters / areas / shape_index (src/observables.jl:7-18), FP64 node sums
 * on the device.  type = 0: all bodies; else bodies of that type, in body
 * order; *count receives the number of values written. */
fcc_status fcc_perimeters(fcc_sim* sim, int32_t type, double* out, int64_t* count);
fcc_status fcc_areas(fcc_sim* sim, int32_t type, double* out, int64_t* count);
fcc_status fcc_shape_index(fcc_sim* sim, int32_t type, double* out, int64_t* count);

/* body_energy(sim): src/observables.jl:47 (sum of Ebody of the last gradient evaluation). */
fcc_status fcc_body_energy(fcc_sim* sim, double* out);

/* philox_noise!(xi, key, n): src/random.jl:113-130.  Fills out (3 x nbodies,
 * column-major) with the first three standard normals of philox_normals for
 * bodies 1..nbodies and draw index `draw`, in precision 32 or 64. */
fcc_status fcc_philox_noise(uint64_t seed, uint64_t draw, int64_t nbodies, int32_t precision, double* out);

/* Standalone neighbour build on caller arrays (no simulation handle):
 * update_celllist! + the neighbour kernel (src/neighbors.jl:81-92, 148-174) on
 * x, y, rmax (length n, precision 32 or 64).  `range` is the contact range
 * plus skin.  Outputs are 1-based; count[i] may exceed cap (overflow, as the
 * reference's kernel counts without storing).  Grid sizes follow
 * CellList(box, cutoff, n).  Device scratch is allocated per call. */
fcc_status fcc_build_neighbors(int32_t precision, int64_t n, const double* x, const double* y,
                               const double* rmax, double Lx, double Ly, double cutoff, double range,
                               int32_t cap, int32_t* cellid, int32_t* perm, int32_t* start,
                               int32_t* stop, int32_t* idx, int32_t* count);

/* Neighbour build that allocates no device memory (no counterpart in the
 * reference, which allocates its lists itself).  For callers that cannot call
 * cudaMalloc — code that runs inside a memory pool or allocator it does not
 * own, or with a device-memory budget fixed up front — this does what
 * fcc_build_neighbors does, but on arrays already on the device: inputs x, y,
 * rmax (n values, float for precision 32, double for 64) and outputs cellid,
 * perm, count (n), start, stop (ncx*ncy) and idx (cap x n), in the same 1-based
 * layout.  All other scratch lives in one static device array of this
 * library, about 3.6 MB, which every GPU that loads the library holds until
 * the process exits; sizes beyond FCC_NOALLOC_MAX_BODIES bodies or
 * FCC_NOALLOC_MAX_CELLS grid cells, and a cutoff or box side that is not a
 * finite positive number, return FCC_ERR_ARGUMENT.  Work is queued on
 * `stream` (a cudaStream_t; NULL: the default stream) and the call returns
 * without synchronising.  The first call on a device looks up the scratch
 * array's device address and keeps it for the process (make that first call
 * before any stream capture; after cudaDeviceReset on that device the kept
 * address is stale and later calls there are invalid).  Every call reuses the
 * same scratch, so calls that overlap on the GPU (other streams, other
 * threads) race: serialise them. */
#define FCC_NOALLOC_MAX_BODIES 16384
#define FCC_NOALLOC_MAX_CELLS 16384
fcc_status fcc_build_neighbors_noalloc(int32_t precision, int64_t n, const void* x, const void* y, const void* rmax,
                                       double Lx, double Ly, double cutoff, double range, int32_t cap,
                                       int32_t* cellid, int32_t* perm, int32_t* start, int32_t* stop, int32_t* idx,
                                       int32_t* count, void* stream);

/* Device timing of the last fcc_step/fcc_run call (CUDA events on the handle's
 * stream): elapsed milliseconds, launches of this library's kernels, and
 * steps executed. */
fcc_status fcc_last_timing(fcc_sim* sim, double* ms, int64_t* launches, int64_t* steps);

/* Health of a simulation (no counterpart in the reference, which neither
 * detects non-finite states nor waits on the device): *nonfinite = 1 once a
 * step produced a non-finite position, angle or contour extent (sticky until
 * fcc_set_state); *barrier_error = 1 if a grid-barrier wait of the persistent
 * step kernel ran out of polls (the step call then failed with
 * FCC_ERR_DEVICE). */
fcc_status fcc_health(fcc_sim* sim, int32_t* nonfinite, int32_t* barrier_error);

/* Self-test of the bounded grid-barrier waits (no counterpart in the
 * reference): launches `blocks` blocks of which the last never arrives, so
 * the others' waits run out after a fixed number of polls, first at a
 * generation-word barrier (pools, parent drag), then at a flat barrier (the
 * step barrier of a lone simulation); *error = 1 when both waits ended with
 * the error status (the expected result for blocks >= 2), 0 when neither did
 * (one block, which waits for no one), 2 when only one did; *ms the kernel's
 * duration.  The device stays usable afterwards. */
fcc_status fcc_barrier_selftest(int32_t blocks, int32_t* error, double* ms);

/* ------------------------------------------------------------------ pool --
 * Many simulations packed into one engine: their bodies, grid cells and
 * neighbour lists share one device arena, and one persistent step kernel
 * launch advances all of them.  The reference runs concurrent simulations as
 * independent `Simulation`s on separate tasks/streams (README.md:255-262);
 * this is the batched form of that, for monolayers of uneven N (batching) and
 * for a request loop that admits and retires simulations while others run
 * (serving).  Each simulation keeps the semantics of fcc_create/fcc_run: its
 * own box, types, terms, dt, seed and Philox stream, its own neighbour-list
 * rebuilds, and results equal to running it alone with the same kernel
 * variant (fcc_pool_variant) — bit for bit.
 *
 * A pool is sized once (fcc_pool_bytes gives its device footprint, so a caller
 * sizes it from an HBM budget).  Every simulation's bodies start at a multiple
 * of FCC_POOL_ALIGN in the arena; the arena is kept dense (retired
 * simulations are compacted away before the next run). */
#define FCC_POOL_ALIGN 8

typedef struct fcc_pool fcc_pool;

typedef struct {
    int32_t precision;    /* 32 or 64, for every simulation of the pool */
    int32_t ntheta;       /* contour nodes, for every simulation of the pool */
    int64_t max_bodies;   /* arena capacity in bodies (each simulation padded to FCC_POOL_ALIGN) */
    int64_t max_cells;    /* arena capacity in grid cells */
    int32_t max_sims;     /* simulation slots */
    int32_t nl_capacity;  /* initial neighbours per body (0: 32); grows on overflow */
    int32_t max_children; /* children per body (0: 1) */
    int32_t max_bonds;    /* bonds per body (0: 1) */
} fcc_pool_params;

/* Device bytes a pool of these limits holds (both arena copies, lists, slots). */
fcc_status fcc_pool_bytes(const fcc_pool_params* params, int64_t* bytes);
fcc_status fcc_pool_create(const fcc_pool_params* params, fcc_pool** out);
fcc_status fcc_pool_destroy(fcc_pool* pool);

/* Admit one simulation (the arguments of fcc_create; params->precision and
 * params->ntheta must equal the pool's) that will run `horizon` steps.
 * FCC_ERR_FULL: no free slot, bodies or cells now (nothing changed). */
fcc_status fcc_pool_add(fcc_pool* pool, const fcc_params* params, const fcc_bodies_host* bodies, int64_t horizon,
                        int32_t* slot);
/* Admit a simulation resumed from a checkpoint: `bodies`, `clock` and `t` as
 * fcc_get_state / fcc_pool_get_state returned them (the clock is the Philox
 * draw index, src/random.jl:103; t is sim.t, which differs from clock * dt
 * once dt has changed); it holds when its clock reaches `horizon`, and its
 * steps done count from `clock`.  t < 0 takes clock * dt.  The state is
 * loaded with the same arithmetic as fcc_set_state (no counterpart in the
 * reference: the serving loop evicts and re-admits with it). */
fcc_status fcc_pool_add_at(fcc_pool* pool, const fcc_params* params, const fcc_bodies_host* bodies, int64_t clock,
                           double t, int64_t horizon, int32_t* slot);
/* Retire a simulation; its room is reclaimed before the next run or add. */
fcc_status fcc_pool_remove(fcc_pool* pool, int32_t slot);

/* Advance every admitted simulation by min(n, horizon - steps done) steps in
 * persistent multi-step launches of the packed step kernel. */
fcc_status fcc_pool_run(fcc_pool* pool, int64_t n);

/* Steps done and horizon of a slot; *active = 0 for a free slot. */
fcc_status fcc_pool_slot(fcc_pool* pool, int32_t slot, int32_t* active, int64_t* steps, int64_t* horizon);
/* Bodies, cells and slots in use, and the capacities. */
fcc_status fcc_pool_usage(fcc_pool* pool, int64_t* bodies, int64_t* cells, int32_t* sims, int64_t* max_bodies,
                          int64_t* max_cells, int32_t* max_sims);

/* fcc_get_state / fcc_shape_index (perimeters: which = 0, areas: 1, shape
 * index: 2) and sim.neighbors.builds of one slot. */
fcc_status fcc_pool_get_state(fcc_pool* pool, int32_t slot, fcc_bodies_host* out, int64_t* clock, double* t,
                              int64_t* step);
fcc_status fcc_pool_observable(fcc_pool* pool, int32_t slot, int32_t which, int32_t type, double* out,
                               int64_t* count);
fcc_status fcc_pool_builds(fcc_pool* pool, int32_t slot, int64_t* builds);

/* Launch configuration: kernel variant (index into the library's table; -1:
 * the autotuned or default choice) and steps per launch (0: 512). */
fcc_status fcc_pool_config(fcc_pool* pool, int32_t variant, int32_t steps_per_launch);
fcc_status fcc_pool_variant(fcc_pool* pool, int32_t* variant, int32_t* lanes, int32_t* slots, int32_t* block,
                            int32_t* min_blocks, int32_t* grid);

/* Device timing of the last fcc_pool_run: milliseconds, launches, and
 * body-steps executed (summed over simulations). */
fcc_status fcc_pool_last_timing(fcc_pool* pool, double* ms, int64_t* launches, int64_t* body_steps);

/* Autotuner: time every candidate kernel variant for `steps` steps of the
 * pool's current simulations, from a snapshot that is restored afterwards
 * (tuning leaves the trajectories untouched), and keep the fastest for this
 * size bucket (packed bodies rounded up to a power of two) in a process-wide
 * table that later runs of any pool of that bucket use unless fcc_pool_config
 * fixed a variant.  reorder = 0: only variants of the current one's family
 * (same lanes x node slots and measured identical rounding: results stay
 * bit-identical); 1: every variant (results agree to FP32 rounding).  *variant = -1 when
 * a neighbour list would have to regrow first (nothing tuned). */
fcc_status fcc_pool_tune(fcc_pool* pool, int64_t steps, int32_t reorder, int32_t* variant, double* us_per_step);

/* CUDA graph of a run round (release upload, persistent launches, status
 * download), recorded once per launch configuration and replayed:
 * enable = 1 / 0 switches it on (default) / off, -1 only queries.  *active = 0
 * when off or when this runtime could not record the round (then rounds are
 * launched directly); *replays counts graph launches. */
fcc_status fcc_pool_graph(fcc_pool* pool, int32_t enable, int32_t* active, int64_t* replays);

/* Message of the last error on this thread. */
const char* fcc_last_error(void);

/* Library build tag (architecture and kernel variants). */
const char* fcc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FCC_H */
