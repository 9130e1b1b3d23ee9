// fcc_pool.cu — packed multi-simulation engine (the fcc_pool_* entry points of
// include/fcc.h).  Included by fcc_lib.cu: it reuses the step kernel, the
// launch-variant table, SimSpec and the status helpers of that file.
//
// Layout.  The bodies of every admitted simulation occupy one contiguous range
// of a device arena, starting at a multiple of FCC_POOL_ALIGN and padded to a
// multiple of it (padding bodies have sim_of = -1); its grid cells occupy one
// contiguous range of the cell arrays.  Body, cell and neighbour ids inside the
// arena are global (arena) ids; each simulation's SimDesc carries body_off and
// cell_off, so every per-simulation quantity the kernels derive (Philox body
// index i = g - body_off + 1, cell index, the stable cell sort) equals the one
// of the same simulation run alone.  A warp group of the step kernel (32/L
// bodies, L <= 16 lanes per body) never straddles two simulations.
//
// Retired simulations leave holes; before the next run or admission the arena
// is compacted by one gather pass into a second arena copy (ids rebased by the
// move), and the copies swap.  A neighbour-list overflow regrows the capacity
// by the same gather with a wider list stride, so the lists of the other
// simulations survive and only the overflowed one rebuilds — as it would alone.

namespace {

constexpr int POOL_ALIGN = FCC_POOL_ALIGN;

// Raw pointers of one arena copy (kernel arguments).
template <class T>
struct ArenaPtrs {
    T* rec0;
    T* rec1;
    T* coef;
    T* R0;
    T* x0;
    T* y0;
    T* rmax0;
    int* imgx;
    int* imgy;
    int* sim_of;
    int* nb_count;
    int* nb_idx;
    int* cellid;
    int* perm;
    int* ch_count;
    int* ch_idx;
    int* bd_count;
    int* bd_idx;
    int* cstart;
    int* cstop;
    int* cell_sim;
    int cap, ccap, bcap;
};

template <class T>
struct Arena {
    DBuf<T> rec0, rec1, coef, R0, x0, y0, rmax0;
    DBuf<int> imgx, imgy, sim_of, nb_count, nb_idx, cellid, perm, ch_count, ch_idx, bd_count, bd_idx;
    DBuf<int> cstart, cstop, cell_sim;
    int cap = 0, ccap = 0, bcap = 0;

    static size_t bytes(size_t nb, size_t nc, int cap, int ccap, int bcap) {
        return nb * (sizeof(T) * (2 * RECW + NCM + 4) + sizeof(int) * (10 + (size_t)cap + ccap + bcap)) +
               nc * sizeof(int) * 3;
    }
    fcc_status alloc(size_t nb, size_t nc, int cap_, int ccap_, int bcap_, cudaStream_t st) {
        cap = cap_;
        ccap = ccap_;
        bcap = bcap_;
        for (DBuf<T>* b : {&rec0, &rec1}) FCC_TRY(b->alloc(nb * RECW, st));
        FCC_TRY(coef.alloc(nb * NCM, st));
        for (DBuf<T>* b : {&R0, &x0, &y0, &rmax0}) FCC_TRY(b->alloc(nb, st));
        for (DBuf<int>* b : {&imgx, &imgy, &sim_of, &nb_count, &cellid, &perm, &ch_count, &bd_count})
            FCC_TRY(b->alloc(nb, st));
        FCC_TRY(nb_idx.alloc(nb * cap, st));
        FCC_TRY(ch_idx.alloc(nb * ccap, st));
        FCC_TRY(bd_idx.alloc(nb * bcap, st));
        for (DBuf<int>* b : {&cstart, &cstop, &cell_sim}) FCC_TRY(b->alloc(nc, st));
        return FCC_OK;
    }
    ArenaPtrs<T> ptrs() {
        return ArenaPtrs<T>{rec0.p,     rec1.p,   coef.p,   R0.p,     x0.p,     y0.p,       rmax0.p,
                            imgx.p,     imgy.p,   sim_of.p, nb_count.p, nb_idx.p, cellid.p, perm.p,
                            ch_count.p, ch_idx.p, bd_count.p, bd_idx.p, cstart.p, cstop.p,  cell_sim.p,
                            cap,        ccap,     bcap};
    }
};

// One live simulation's move in a compaction: its bodies [old_off, old_off +
// npad) go to [new_off, ...), its cells [old_coff, old_coff + ncells) to
// [new_coff, ...).  Entries are sorted by new_off and cover the new arena.
struct MoveRange {
    int new_off, old_off, npad, new_coff, old_coff, ncells;
};

__device__ __forceinline__ int find_move(const MoveRange* mv, int nmv, int g, bool cells) {
    int lo = 0, hi = nmv - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((cells ? mv[mid].new_coff : mv[mid].new_off) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Gather the bodies of the live simulations into the other arena copy with
// rebased ids.  The current record's w field carries the parent id (rebased);
// the other record buffer is rewritten in full by the next step.
template <class T>
__global__ void k_pool_gather_bodies(ArenaPtrs<T> src, ArenaPtrs<T> dst, const MoveRange* __restrict__ mv, int nmv,
                                     int newN, int par) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= newN) return;
    const MoveRange m = mv[find_move(mv, nmv, g, false)];
    const int delta = m.old_off - m.new_off;
    const int cdelta = m.old_coff - m.new_coff;
    const int o = g + delta;
    const int so = src.sim_of[o];
    dst.sim_of[g] = so;
    T* rc_src = par ? src.rec1 : src.rec0;
    T* rc_dst = par ? dst.rec1 : dst.rec0;
    T* rn_src = par ? src.rec0 : src.rec1;
    T* rn_dst = par ? dst.rec0 : dst.rec1;
    for (int r = 0; r < RECW; ++r) {
        T v = rc_src[(size_t)o * RECW + r];
        if (r == R_W && so >= 0) {
            const int w = unpack_w(v);
            T* tag = nullptr;
            v = pack_w((((w >> 3) - delta) << 3) | (w & 7), tag);
        }
        rc_dst[(size_t)g * RECW + r] = v;
        rn_dst[(size_t)g * RECW + r] = rn_src[(size_t)o * RECW + r];
    }
    for (int r = 0; r < NCM; ++r) dst.coef[(size_t)g * NCM + r] = src.coef[(size_t)o * NCM + r];
    dst.R0[g] = src.R0[o];
    dst.x0[g] = src.x0[o];
    dst.y0[g] = src.y0[o];
    dst.rmax0[g] = src.rmax0[o];
    dst.imgx[g] = src.imgx[o];
    dst.imgy[g] = src.imgy[o];
    dst.perm[g] = src.perm[o] - delta;  // perm is indexed by arena position
    if (so < 0) {
        dst.nb_count[g] = 0;
        dst.ch_count[g] = 0;
        dst.bd_count[g] = 0;
        return;
    }
    dst.cellid[g] = src.cellid[o] - cdelta;
    const int cnt = src.nb_count[o];
    dst.nb_count[g] = cnt;
    const int nq = min(cnt, min(src.cap, dst.cap));
    for (int q = 0; q < nq; ++q) dst.nb_idx[(size_t)g * dst.cap + q] = src.nb_idx[(size_t)o * src.cap + q] - delta;
    const int cc = src.ch_count[o];
    dst.ch_count[g] = cc;
    for (int q = 0; q < cc; ++q) dst.ch_idx[(size_t)g * dst.ccap + q] = src.ch_idx[(size_t)o * src.ccap + q] - delta;
    const int bc = src.bd_count[o];
    dst.bd_count[g] = bc;
    for (int q = 0; q < bc; ++q) dst.bd_idx[(size_t)g * dst.bcap + q] = src.bd_idx[(size_t)o * src.bcap + q] - delta;
}

template <class T>
__global__ void k_pool_gather_cells(ArenaPtrs<T> src, ArenaPtrs<T> dst, const MoveRange* __restrict__ mv, int nmv,
                                    int newC) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= newC) return;
    const MoveRange m = mv[find_move(mv, nmv, c, true)];
    const int delta = m.old_off - m.new_off;
    const int o = c + (m.old_coff - m.new_coff);
    dst.cstart[c] = src.cstart[o] - delta;
    dst.cstop[c] = src.cstop[o] - delta;
    dst.cell_sim[c] = src.cell_sim[o];
}

// Slot set-up on the device: simulation ids of the slot's bodies (padding -1)
// and cells, children and bond partners rebased to arena ids.
__global__ void k_pool_slot_ids(int* sim_of, int* cell_sim, int* ch_count, int* ch_idx, int* bd_count, int* bd_idx,
                                const int* __restrict__ chc, const int* __restrict__ chi, const int* __restrict__ bdc,
                                const int* __restrict__ bdi, int slot, int off, int n, int npad, int coff, int ncells,
                                int ccap_src, int ccap, int bcap_src, int bcap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ncells) cell_sim[coff + i] = slot;
    if (i >= npad) return;
    const int g = off + i;
    sim_of[g] = i < n ? slot : -1;
    const int cc = i < n ? chc[i] : 0;
    ch_count[g] = cc;
    for (int q = 0; q < cc; ++q) ch_idx[(size_t)g * ccap + q] = chi[(size_t)i * ccap_src + q] + off;
    const int bc = i < n ? bdc[i] : 0;
    bd_count[g] = bc;
    for (int q = 0; q < bc; ++q) bd_idx[(size_t)g * bcap + q] = bdi[(size_t)i * bcap_src + q] + off;
}

struct PoolBase {
    virtual ~PoolBase() = default;
    virtual fcc_status add(const fcc_params* p, const fcc_bodies_host* b, int64_t horizon, int64_t clock0, double t0,
                           int32_t* slot) = 0;
    virtual fcc_status remove(int32_t slot) = 0;
    virtual fcc_status run(int64_t n) = 0;
    virtual fcc_status slot_info(int32_t slot, int32_t* active, int64_t* steps, int64_t* horizon) = 0;
    virtual fcc_status usage(int64_t*, int64_t*, int32_t*, int64_t*, int64_t*, int32_t*) = 0;
    virtual fcc_status get_state(int32_t slot, fcc_bodies_host* out, int64_t* clock, double* t, int64_t* step) = 0;
    virtual fcc_status observable(int32_t slot, int which, int32_t type, double* out, int64_t* count) = 0;
    virtual fcc_status slot_builds(int32_t slot, int64_t* b) = 0;
    virtual fcc_status config(int32_t variant, int32_t spl) = 0;
    virtual fcc_status variant_info(int32_t*, int32_t*, int32_t*, int32_t*, int32_t*, int32_t*) = 0;
    virtual fcc_status timing(double* ms, int64_t* launches, int64_t* body_steps) = 0;
    virtual fcc_status tune(int64_t steps, bool reorder, int32_t* chosen, double* best_us) = 0;
    virtual fcc_status graph_mode(int32_t enable, int32_t* active, int64_t* replays) = 0;
};

template <class T>
size_t pool_bytes(const fcc_pool_params& q) {
    const int cap = q.nl_capacity > 0 ? q.nl_capacity : 32;
    const int ccap = q.max_children > 0 ? q.max_children : 1;
    const int bcap = q.max_bonds > 0 ? q.max_bonds : 1;
    const size_t nb = (size_t)q.max_bodies, nc = (size_t)q.max_cells, ns = (size_t)std::max(q.max_sims, 2);
    const size_t transient = nb * (sizeof(T) * (4 + NCM) + sizeof(int)) + nc * sizeof(int);
    const size_t per_sim = ns * (sizeof(SimDesc<T>) + 2 * sizeof(int) + 3 * sizeof(long long));
    return 2 * Arena<T>::bytes(nb, nc, cap, ccap, bcap) + transient + per_sim;
}

template <class T>
struct Pool final : PoolBase {
    int device = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int nth = 0, cap = 32, ccap = 1, bcap = 1;
    int64_t max_bodies = 0, max_cells = 0;
    int max_sims = 0, nslots = 0;  // nslots = max(max_sims, 2): a pool never takes the one-simulation kernel path
    std::unique_ptr<Arena<T>> A, B;  // A holds the state; B is the compaction target
    DBuf<SimDesc<T>> sims;
    DBuf<int> flags, maxcount, slot_scr, ccount;
    DBuf<long long> clock, stop, builds;
    DBuf<GridSync> sync;
    DBuf<T> gx, gy, gth, E, glab, cs, basis;
    DBuf<float> mtab;  // FP32: tensor-core fragment table
    DBuf<MoveRange> moves;
    std::vector<SimDesc<T>> desc_stage;  // host staging of the descriptors a compaction rebases
    // device staging of an admission (bodies, child and bond lists), reused
    Stage<double> st_xch;  // host state exchange: x, y, theta, coefficients as the caller's doubles
    Stage<int> st_w, st_chc, st_chi, st_bdc, st_bdi;
    ObsArea obs;  // perimeters / areas / shape indices: reused device and pinned host buffers

    struct Slot {
        bool used = false;
        SimSpec<T> spec;
        int64_t off = 0, npad = 0;
        int coff = 0, ncells = 0;
        long long clock_h = 0, horizon = 0;
        T t_h = T(0);
        int64_t step_h = 0, builds_adjust = 0;
        int flags_h = 0;
    };
    std::vector<Slot> slots;
    std::vector<int> order;  // used slots in arena order
    int64_t Ntot = 0;
    int64_t Ctot = 0;
    bool dirty = false;
    long long gstep = 0;
    int nsplit = 0;
    // pinned status read-back
    int* fl_h = nullptr;
    int* mc_h = nullptr;
    long long* clk_h = nullptr;
    long long* bld_h = nullptr;
    long long* stop_h = nullptr;
    GridSync* sy_h = nullptr;
    int* fl_in_h = nullptr;  // release values uploaded at the start of a round
    int* any_h = nullptr;
    // CUDA graph of one round
    bool use_graph = true, graph_ok = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<long long> graph_key;
    int64_t graph_launches = 0;
    // launch configuration
    int variant = -1;  // -1: default (variant 0)
    int spl = 512;
    int grid = 0;
    double last_ms = 0;
    int64_t last_launches = 0, last_body_steps = 0;

    ~Pool() override {
        if (stream) cudaStreamSynchronize(stream);
        drop_graph();
        for (void* p : {(void*)fl_h, (void*)mc_h, (void*)clk_h, (void*)bld_h, (void*)stop_h, (void*)sy_h,
                        (void*)fl_in_h, (void*)any_h})
            if (p) cudaFreeHost(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    int par() const { return (int)(gstep & 1); }
    const Variant& var() const { return VARIANTS[variant < 0 ? 0 : variant]; }
    bool split() const { return nsplit > 0; }
    void* step_kernel() const { return (sizeof(T) == 4 ? var().f32 : var().f64)(nth <= var().L * var().S, split()); }
    size_t stage_bytes() const {
        return basis_table_bytes<T>() + (size_t)(var().blk / 32) * (sizeof(T) == 4 ? var().stage32 : var().stage64);
    }

    fcc_status init(const fcc_pool_params& q) {
        if (q.ntheta < 3) return fail(FCC_ERR_ARGUMENT, "pool: ntheta must be at least 3");
        if (q.max_bodies < 0 || q.max_cells < 0 || q.max_sims < 1)
            return fail(FCC_ERR_ARGUMENT, "pool: max_bodies and max_cells must be >= 0 and max_sims >= 1");
        if (q.max_bodies > (1ll << 30) || q.max_cells > (1ll << 30))
            return fail(FCC_ERR_UNSUPPORTED, "pool: at most 2^30 bodies and 2^30 cells");
        nth = q.ntheta;
        cap = q.nl_capacity > 0 ? q.nl_capacity : 32;
        ccap = q.max_children > 0 ? q.max_children : 1;
        bcap = q.max_bonds > 0 ? q.max_bonds : 1;
        max_bodies = q.max_bodies / POOL_ALIGN * POOL_ALIGN;
        max_cells = q.max_cells;
        max_sims = q.max_sims;
        nslots = std::max(max_sims, 2);
        CUDA_TRY(cudaGetDevice(&device));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        int coop = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        if (!coop) return fail(FCC_ERR_UNSUPPORTED, "device lacks cooperative launch");
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreate(&ev0));
        CUDA_TRY(cudaEventCreate(&ev1));
        CUDA_TRY(cudaMallocHost(&fl_h, nslots * sizeof(int)));
        CUDA_TRY(cudaMallocHost(&mc_h, nslots * sizeof(int)));
        CUDA_TRY(cudaMallocHost(&clk_h, nslots * sizeof(long long)));
        CUDA_TRY(cudaMallocHost(&bld_h, nslots * sizeof(long long)));
        CUDA_TRY(cudaMallocHost(&stop_h, nslots * sizeof(long long)));
        CUDA_TRY(cudaMallocHost(&sy_h, sizeof(GridSync)));
        CUDA_TRY(cudaMallocHost(&fl_in_h, nslots * sizeof(int)));
        CUDA_TRY(cudaMallocHost(&any_h, sizeof(int)));
        A = std::make_unique<Arena<T>>();
        B = std::make_unique<Arena<T>>();
        const size_t nb = (size_t)max_bodies, nc = (size_t)max_cells;
        FCC_TRY(A->alloc(nb, nc, cap, ccap, bcap, stream));
        FCC_TRY(B->alloc(nb, nc, cap, ccap, bcap, stream));
        FCC_TRY(sims.alloc(nslots, stream));
        for (DBuf<int>* b : {&flags, &maxcount}) FCC_TRY(b->alloc(nslots, stream));
        for (DBuf<long long>* b : {&clock, &stop, &builds}) FCC_TRY(b->alloc(nslots, stream));
        FCC_TRY(sync.alloc(1, stream));
        FCC_TRY(slot_scr.alloc(nb, stream));
        FCC_TRY(ccount.alloc(nc, stream));
        for (DBuf<T>* b : {&gx, &gy, &gth, &E}) FCC_TRY(b->alloc(nb, stream));
        FCC_TRY(glab.alloc(nb * NCM, stream));
        FCC_TRY(moves.alloc(nslots, stream));
        std::vector<T> csh(2 * (size_t)nth);
        for (int k = 0; k < nth; ++k) {  // FourierBasis.cs, src/basis.jl:50-52
            const double phi = k * (2 * PI / nth);
            csh[2 * k] = (T)std::cos(phi);
            csh[2 * k + 1] = (T)std::sin(phi);
        }
        FCC_TRY(cs.upload(csh, stream));
        FCC_TRY(basis.upload(mode_table<T>(nth), stream));
        if (sizeof(T) == 4 && nth <= BASIS_NODES) FCC_TRY(mtab.upload(mma_table(nth), stream));
        slots.assign(nslots, Slot{});
        for (int s = 0; s < nslots; ++s) stop_h[s] = 0;
        return sync_stream();
    }

    fcc_status sync_stream() {
        CUDA_TRY(cudaStreamSynchronize(stream));
        return FCC_OK;
    }

    DevPtrs<T> ptrs() {
        Arena<T>& a = *A;
        DevPtrs<T> d{};
        d.sims = sims.p;
        d.nsims = nslots;
        d.Ntot = (int)Ntot;
        d.Ctot = (int)Ctot;
        d.nth = nth;
        d.cap = a.cap;
        d.sim_of = a.sim_of.p;
        d.rec0 = a.rec0.p;
        d.rec1 = a.rec1.p;
        d.coef = a.coef.p;
        d.imgx = a.imgx.p;
        d.imgy = a.imgy.p;
        d.R0 = a.R0.p;
        d.x0 = a.x0.p;
        d.y0 = a.y0.p;
        d.rmax0 = a.rmax0.p;
        d.nb_idx = a.nb_idx.p;
        d.nb_count = a.nb_count.p;
        d.cellid = a.cellid.p;
        d.slot = slot_scr.p;
        d.perm = a.perm.p;
        d.cstart = a.cstart.p;
        d.cstop = a.cstop.p;
        d.ccount = ccount.p;
        d.cell_sim = a.cell_sim.p;
        d.ccap = a.ccap;
        d.ch_idx = a.ch_idx.p;
        d.ch_count = a.ch_count.p;
        d.bcap = a.bcap;
        d.bd_idx = a.bd_idx.p;
        d.bd_count = a.bd_count.p;
        d.flags = flags.p;
        d.clock = clock.p;
        d.stop = stop.p;
        d.builds = builds.p;
        d.maxcount = maxcount.p;
        d.sync = sync.p;
        d.cs = cs.p;
        d.basis = basis.p;
        d.mtab = mtab.p;
        d.gx = gx.p;
        d.gy = gy.p;
        d.gth = gth.p;
        d.glab = glab.p;
        d.E = E.p;
        return d;
    }

    // ------------------------------------------------------- admission --
    fcc_status add(const fcc_params* p, const fcc_bodies_host* b, int64_t horizon, int64_t clock0, double t0,
                   int32_t* slot_out) override {
        Range range("fcc pool add");
        if (!p || !b || !slot_out) return fail(FCC_ERR_ARGUMENT, "null argument");
        if (clock0 < 0) return fail(FCC_ERR_ARGUMENT, "pool: clock must be >= 0");
        if (std::isnan(t0)) return fail(FCC_ERR_ARGUMENT, "pool: t must not be NaN");
        if (p->precision != (sizeof(T) == 4 ? 32 : 64))
            return fail(FCC_ERR_ARGUMENT, "pool: the simulation's precision differs from the pool's");
        if (p->ntheta != nth) return fail(FCC_ERR_DIMENSION, "pool: the simulation's ntheta differs from the pool's");
        if (horizon < 0) return fail(FCC_ERR_ARGUMENT, "pool: horizon must be >= 0");
        if (b->n > 0 && (!b->x || !b->y || !b->theta || !b->coef))
            return fail(FCC_ERR_ARGUMENT, "pool: x, y, theta and coef are required");
        SimSpec<T> sp;
        FCC_TRY(make_spec(p, b, sp));
        if (sp.desc.nub + sp.desc.nuc + sp.desc.nubd > 0)
            return fail(FCC_ERR_UNSUPPORTED, "pool: simulations with compiled user terms run alone (fcc_create)");
        if (sp.ccap > ccap || sp.bcap > bcap)
            return fail(FCC_ERR_UNSUPPORTED, "pool: more children or bonds per body than the pool was made for");
        FCC_TRY(compact());
        int s = -1;
        for (int u = 0; u < max_sims; ++u)
            if (!slots[u].used) {
                s = u;
                break;
            }
        const int64_t N = sp.N;
        const int64_t npad = (N + POOL_ALIGN - 1) / POOL_ALIGN * POOL_ALIGN;
        const int64_t nce = (int64_t)sp.ncx * sp.ncy;
        if (s < 0 || Ntot + npad > max_bodies || Ctot + nce > max_cells)
            return fail(FCC_ERR_FULL, "pool: no room for " + std::to_string(N) + " bodies and " + std::to_string(nce) +
                                          " cells now (" + std::to_string(max_bodies - Ntot) + " bodies, " +
                                          std::to_string(max_cells - Ctot) + " cells free)");
        Slot& S = slots[s];
        S = Slot{};
        S.used = true;
        S.off = Ntot;
        S.npad = npad;
        S.coff = (int)Ctot;
        S.ncells = (int)nce;
        S.horizon = horizon;
        // a resumed simulation counts its steps from its clock, so that steps
        // done and the horizon are both measured on the clock; its time is the
        // checkpoint's (t0), or clock * dt when the caller has none (t0 < 0:
        // exact only if dt never changed before the checkpoint)
        S.clock_h = clock0;
        S.step_h = clock0;
        S.t_h = t0 >= 0 ? (T)t0 : (T)((double)clock0 * (double)sp.desc.dt);
        sp.desc.body_off = (int)S.off;
        sp.desc.cell_off = S.coff;
        S.spec = std::move(sp);
        const SimSpec<T>& P = S.spec;
        Arena<T>& a = *A;
        CUDA_TRY(cudaMemcpyAsync(sims.p + s, &P.desc, sizeof(SimDesc<T>), cudaMemcpyHostToDevice, stream));
        if (N > 0) {
            const size_t n = (size_t)N;
            CUDA_TRY(cudaMemcpyAsync(a.R0.p + S.off, P.R0.data(), n * sizeof(T), cudaMemcpyHostToDevice, stream));
            if (b->imgx) CUDA_TRY(cudaMemcpyAsync(a.imgx.p + S.off, b->imgx, n * sizeof(int), cudaMemcpyHostToDevice, stream));
            else CUDA_TRY(cudaMemsetAsync(a.imgx.p + S.off, 0, n * sizeof(int), stream));
            if (b->imgy) CUDA_TRY(cudaMemcpyAsync(a.imgy.p + S.off, b->imgy, n * sizeof(int), cudaMemcpyHostToDevice, stream));
            else CUDA_TRY(cudaMemsetAsync(a.imgy.p + S.off, 0, n * sizeof(int), stream));
        }
        {
            FCC_TRY(st_chc.upload(P.chc, stream));
            FCC_TRY(st_chi.upload(P.chi, stream));
            FCC_TRY(st_bdc.upload(P.bdc, stream));
            FCC_TRY(st_bdi.upload(P.bdi, stream));
            const int64_t cnt = std::max<int64_t>(npad, nce);
            if (cnt > 0)
                k_pool_slot_ids<<<(int)((cnt + 255) / 256), 256, 0, stream>>>(
                    a.sim_of.p, a.cell_sim.p, a.ch_count.p, a.ch_idx.p, a.bd_count.p, a.bd_idx.p, st_chc.p(),
                    st_chi.p(), st_bdc.p(), st_bdi.p(), s, (int)S.off, (int)N, (int)npad, S.coff, (int)nce, P.ccap,
                    a.ccap, P.bcap, a.bcap);
            CUDA_TRY(cudaGetLastError());
            FCC_TRY(sync_stream());
        }
        Ntot += npad;
        Ctot += nce;
        order.push_back(s);
        if (P.split) ++nsplit;
        FCC_TRY(load_bodies(s, b));
        // held until the next run releases it; the list is invalid, so the
        // release rebuilds it
        S.flags_h = F_ACTIVE | F_HOLD | (P.has_contact ? F_CONTACT : 0);
        const long long zero = 0;
        CUDA_TRY(cudaMemcpyAsync(flags.p + s, &S.flags_h, sizeof(int), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(clock.p + s, &S.clock_h, sizeof(long long), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(builds.p + s, &zero, sizeof(long long), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemsetAsync(maxcount.p + s, 0, sizeof(int), stream));
        *slot_out = s;
        return sync_stream();
    }

    // enforce_shape! and lab frame of a slot's host state (k_init):
    // the caller's double arrays are copied as they are and converted on the
    // device
    fcc_status load_bodies(int s, const fcc_bodies_host* b) {
        Slot& S = slots[s];
        const SimSpec<T>& P = S.spec;
        const size_t n = (size_t)P.N;
        if (n == 0) return FCC_OK;
        std::vector<int> w(n);
        for (size_t i = 0; i < n; ++i) w[i] = (((int)S.off + P.parent[i] - 1) << 3) | (P.type[i] - 1);
        FCC_TRY(st_xch.reserve(n * (3 + (size_t)P.nc), stream));
        double* dx = st_xch.p();
        CUDA_TRY(cudaMemcpyAsync(dx, b->x, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(dx + n, b->y, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(dx + 2 * n, b->theta, n * sizeof(double), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(dx + 3 * n, b->coef, n * P.nc * sizeof(double), cudaMemcpyHostToDevice, stream));
        FCC_TRY(st_w.upload(w, stream));
        const DevPtrs<T> d = ptrs();
        const int blocks = (int)((n + INIT_BLOCK - 1) / INIT_BLOCK);
        k_init<T><<<blocks, INIT_BLOCK, init_smem_bytes(P.nc), stream>>>(d, par(), (int)S.off, (int)n, dx, dx + n,
                                                                          dx + 2 * n, dx + 3 * n, P.nc, P.K, st_w.p(),
                                                                          nullptr, nullptr);
        CUDA_TRY(cudaGetLastError());
        return sync_stream();
    }

    fcc_status remove(int32_t s) override {
        if (s < 0 || s >= max_sims || !slots[s].used) return fail(FCC_ERR_ARGUMENT, "pool: no simulation in this slot");
        const int zero = 0;
        CUDA_TRY(cudaMemcpyAsync(flags.p + s, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
        if (slots[s].spec.split) --nsplit;
        slots[s].used = false;
        slots[s].spec = SimSpec<T>{};
        order.erase(std::find(order.begin(), order.end(), s));
        dirty = true;
        return sync_stream();
    }

    // ------------------------------------------------------ compaction --
    // Gather every live simulation into B at dense offsets (list capacity
    // newcap), swap the arena copies, rebase the descriptors.
    fcc_status gather(int newcap) {
        Range range("fcc pool compact");
        std::vector<MoveRange> mv;
        int64_t nb = 0, nc = 0;
        for (int s : order) {
            Slot& S = slots[s];
            mv.push_back(MoveRange{(int)nb, (int)S.off, (int)S.npad, (int)nc, S.coff, S.ncells});
            nb += S.npad;
            nc += S.ncells;
        }
        if (B->cap != newcap || B->ccap != ccap || B->bcap != bcap)
            FCC_TRY(B->alloc((size_t)max_bodies, (size_t)max_cells, newcap, ccap, bcap, stream));
        if (!mv.empty()) {
            CUDA_TRY(cudaMemcpyAsync(moves.p, mv.data(), mv.size() * sizeof(MoveRange), cudaMemcpyHostToDevice, stream));
            if (nb > 0)
                k_pool_gather_bodies<T><<<(int)((nb + 255) / 256), 256, 0, stream>>>(A->ptrs(), B->ptrs(), moves.p,
                                                                                   (int)mv.size(), (int)nb, par());
            if (nc > 0)
                k_pool_gather_cells<T><<<(int)((nc + 255) / 256), 256, 0, stream>>>(A->ptrs(), B->ptrs(), moves.p,
                                                                                  (int)mv.size(), (int)nc);
            CUDA_TRY(cudaGetLastError());
        }
        std::swap(A, B);
        cap = newcap;
        size_t k = 0;
        int lo = nslots, hi = -1;  // the rebased descriptors go up in one copy
        for (int s : order) {
            Slot& S = slots[s];
            S.off = mv[k].new_off;
            S.coff = mv[k].new_coff;
            ++k;
            S.spec.desc.body_off = (int)S.off;
            S.spec.desc.cell_off = S.coff;
            lo = std::min(lo, s);
            hi = std::max(hi, s);
        }
        if (hi >= lo) {
            desc_stage.resize((size_t)(hi - lo + 1));
            for (int s = lo; s <= hi; ++s)
                if (slots[s].used) desc_stage[(size_t)(s - lo)] = slots[s].spec.desc;
            // slots between lo and hi that are not in use get a copy they never read
            CUDA_TRY(cudaMemcpyAsync(sims.p + lo, desc_stage.data(), desc_stage.size() * sizeof(SimDesc<T>),
                                     cudaMemcpyHostToDevice, stream));
        }
        Ntot = nb;
        Ctot = nc;
        dirty = false;
        return sync_stream();
    }

    fcc_status compact() {
        if (!dirty) return FCC_OK;
        return gather(cap);
    }

    // ------------------------------------------------------------- run --
    fcc_status configure() {
        if (variant >= 0 && sizeof(T) != 4 && !VARIANTS[variant].f64)
            return fail(FCC_ERR_UNSUPPORTED, "pool: this kernel variant has no FP64 build");
        const int smem = (int)stage_bytes();
        CUDA_TRY(cudaFuncSetAttribute(step_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel(), var().blk, smem));
        if (per_sm < 1) return fail(FCC_ERR_UNSUPPORTED, "step kernel does not fit on an SM");
        const int bpw = 32 / var().L;
        const int64_t groups = (Ntot + bpw - 1) / bpw;
        const int64_t want = std::max<int64_t>(1, (groups + var().blk / 32 - 1) / (var().blk / 32));
        grid = (int)std::min<int64_t>(want, (int64_t)per_sm * nsm);
        return FCC_OK;
    }

    // Status of every slot into pinned host buffers (queued on the stream).
    fcc_status enqueue_status() {
        const int ns = nslots;
        CUDA_TRY(cudaMemcpyAsync(fl_h, flags.p, ns * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(mc_h, maxcount.p, ns * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(clk_h, clock.p, ns * sizeof(long long), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(bld_h, builds.p, ns * sizeof(long long), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(sy_h, sync.p, sizeof(GridSync), cudaMemcpyDeviceToHost, stream));
        return FCC_OK;
    }

    // Host mirror from the status read back (after the stream synchronised).
    fcc_status process_status() {
        if (sy_h->error) return fail(FCC_ERR_DEVICE, "a grid barrier wait timed out in the step kernel");
        for (int s : order) {
            Slot& S = slots[s];
            S.flags_h = fl_h[s];
            const long long executed = clk_h[s] - S.clock_h;
            for (long long q = 0; q < executed; ++q) S.t_h += S.spec.desc.dt;
            S.step_h += executed;
            last_body_steps += executed * S.spec.N;
            S.clock_h = clk_h[s];
        }
        return FCC_OK;
    }

    // Release every simulation that has steps left up to its target, with
    // the rebuild decision bookkeeping() takes after a step
    // (src/simulation.jl:132-142), into the pinned upload buffers.  Returns the
    // most steps any one needs.
    int64_t release(const std::vector<long long>& target) {
        int any = 0;
        int64_t most = 0;
        for (int s = 0; s < nslots; ++s) {
            fl_in_h[s] = 0;
            stop_h[s] = 0;
        }
        for (int s : order) {
            Slot& S = slots[s];
            int f = S.flags_h & ~F_HOLD;
            stop_h[s] = target[s];
            if (target[s] <= S.clock_h) {
                f |= F_HOLD;
            } else {
                most = std::max<int64_t>(most, target[s] - S.clock_h);
                const bool need = (f & F_CONTACT) && !(f & F_FROZEN) &&
                                  ((f & F_REBUILD) || !(f & F_VALID) || (f & F_NEED) || S.spec.desc.skin == T(0));
                if (need) {
                    f = (f & ~F_REBUILD) | F_NEED;
                    any = 1;
                }
            }
            S.flags_h = f;
            fl_in_h[s] = f;
        }
        *any_h = any;
        return most;
    }

    // One round: upload the release, `most` steps in launches of at most
    // `spl` steps, download the status.  Recorded once as a CUDA graph and
    // replayed while the launch configuration, the arena and the record
    // parity are unchanged (the graph's copies read and write the pinned
    // buffers, so new release values go in without re-recording).
    fcc_status enqueue_round(int64_t most, long long g0) {
        const int ns = nslots;
        CUDA_TRY(cudaMemcpyAsync(flags.p, fl_in_h, ns * sizeof(int), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(stop.p, stop_h, ns * sizeof(long long), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(&sync.p->any_need, any_h, sizeof(int), cudaMemcpyHostToDevice, stream));
        DevPtrs<T> d = ptrs();
        long long g = g0;
        for (int64_t left = most; left > 0;) {
            int k = (int)std::min<int64_t>(spl, left);
            int p0 = (int)(g & 1);
            void* args[] = {&d, &k, &p0};
            CUDA_TRY(cudaLaunchCooperativeKernel(step_kernel(), dim3(grid), dim3(var().blk), args, stage_bytes(), stream));
            g += k;
            left -= k;
        }
        return enqueue_status();
    }

    fcc_status run_round(int64_t most) {
        Range range("fcc pool round");
        FCC_TRY(configure());
        const int64_t nl = (most + spl - 1) / spl;
        if (use_graph && graph_ok) {
            const std::vector<long long> key = {(long long)(uintptr_t)A.get(), (long long)Ntot, (long long)Ctot,
                                                (long long)grid, (long long)variant, (long long)split(),
                                                (long long)cap, (long long)par(), (long long)most, (long long)spl};
            if (key != graph_key) {
                drop_graph();
                cudaGraph_t g = nullptr;
                CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                const fcc_status st = enqueue_round(most, gstep);
                const cudaError_t e = cudaStreamEndCapture(stream, &g);
                if (st == FCC_OK && e == cudaSuccess && g &&
                    cudaGraphInstantiate(&graph_exec, g, 0) == cudaSuccess) {
                    graph = g;
                    graph_key = key;
                } else {
                    // this runtime does not record the round (e.g. the
                    // cooperative launch): launch it directly from now on
                    if (g) cudaGraphDestroy(g);
                    graph_exec = nullptr;
                    graph_ok = false;
                    cudaGetLastError();
                }
            }
            if (graph_ok) {
                CUDA_TRY(cudaGraphLaunch(graph_exec, stream));
                ++graph_launches;
            } else {
                FCC_TRY(enqueue_round(most, gstep));
            }
        } else {
            FCC_TRY(enqueue_round(most, gstep));
        }
        gstep += most;
        last_launches += nl;
        CUDA_TRY(cudaStreamSynchronize(stream));
        return process_status();
    }

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        graph_key.clear();
    }

    // Neighbour-list overflow of some simulations: regrow the shared capacity
    // to twice the largest count, keeping every list, and rebuild the
    // overflowed ones (src/neighbors.jl:226-233).
    fcc_status regrow() {
        int mc = 0;
        for (int s : order)
            if (slots[s].flags_h & F_FROZEN) mc = std::max(mc, mc_h[s]);
        FCC_TRY(gather(std::max(2 * mc, cap + 1)));
        for (int s : order) {
            Slot& S = slots[s];
            if (!(S.flags_h & F_FROZEN)) continue;
            S.builds_adjust -= 1;  // the overflowed build is repeated
            S.flags_h = (S.flags_h & ~(F_FROZEN | F_VALID | F_REBUILD)) | F_NEED;
        }
        return FCC_OK;
    }

    // Advance every simulation to its target clock (rounds until no
    // simulation is frozen by a list overflow); all hold afterwards.
    fcc_status advance_to(const std::vector<long long>& target) {
        for (int round = 0;; ++round) {
            const int64_t most = release(target);
            if (most == 0) break;
            FCC_TRY(run_round(most));
            bool frozen = false;
            for (int s : order) frozen |= (slots[s].flags_h & F_FROZEN) != 0;
            if (frozen && tuning) return fail(FCC_ERR_FULL, "pool: a neighbour list overflowed during tuning");
            if (frozen) FCC_TRY(regrow());
            else {
                for (int s : order)
                    if (slots[s].clock_h < target[s])
                        return fail(FCC_ERR_DEVICE, "pool: the step kernel did not advance a simulation's clock");
                break;
            }
            if (round > 64) return fail(FCC_ERR_DEVICE, "pool: neighbour lists did not fit after regrowth");
        }
        for (int s : order) slots[s].flags_h |= F_HOLD;
        for (int s = 0; s < nslots; ++s) fl_in_h[s] = 0;
        for (int s : order) fl_in_h[s] = slots[s].flags_h;
        CUDA_TRY(cudaMemcpyAsync(flags.p, fl_in_h, nslots * sizeof(int), cudaMemcpyHostToDevice, stream));
        return sync_stream();
    }

    fcc_status run(int64_t n) override {
        last_launches = 0;
        last_body_steps = 0;
        last_ms = 0;
        if (n <= 0) return FCC_OK;
        FCC_TRY(compact());
        FCC_TRY(apply_tuned());
        std::vector<long long> target(nslots, 0);
        for (int s : order) {
            const Slot& S = slots[s];
            target[s] = S.clock_h + std::min<long long>(n, std::max<long long>(0, S.horizon - S.clock_h));
        }
        CUDA_TRY(cudaEventRecord(ev0, stream));
        FCC_TRY(advance_to(target));
        CUDA_TRY(cudaEventRecord(ev1, stream));
        CUDA_TRY(cudaEventSynchronize(ev1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        return FCC_OK;
    }

    // ------------------------------------------------------- autotuner --
    // Launch shapes are chosen per size bucket (packed bodies rounded up to a
    // power of two, precision): each candidate variant runs `steps` steps of
    // the live pool from a snapshot, the fastest is kept, and the snapshot is
    // restored, so tuning leaves no trace in the trajectories.  By default the
    // candidates are the current variant's family (block size and register
    // budget differ, the rounding is measured identical, so results stay
    // bit-identical); `reorder` admits every variant (other lane counts sum
    // node quadratures in another order: results then agree with the default
    // to FP32 rounding, not bit for bit).
    static std::map<std::pair<int, int>, int>& tune_table() {
        static std::map<std::pair<int, int>, int> t;
        return t;
    }
    static std::mutex& tune_mutex() {
        static std::mutex m;
        return m;
    }
    std::pair<int, int> bucket() const {
        int b = 0;
        while ((1ll << b) < std::max<int64_t>(Ntot, 1)) ++b;
        return {(int)sizeof(T), b};
    }
    bool tuned = false;     // variant came from the table or a tune call
    bool tuning = false;    // inside a tune trial (the snapshot in B must survive)
    bool user_set = false;  // fcc_pool_config chose the variant

    fcc_status apply_tuned() {
        if (user_set) return FCC_OK;
        std::lock_guard<std::mutex> lk(tune_mutex());
        auto it = tune_table().find(bucket());
        if (it != tune_table().end()) {
            variant = it->second;
            tuned = true;
        } else {
            variant = -1;
            tuned = false;
        }
        return FCC_OK;
    }

    // Identity copy of the live arena ranges from one copy to the other.
    fcc_status copy_arena(Arena<T>& src, Arena<T>& dst) {
        if (dst.cap != src.cap || dst.ccap != src.ccap || dst.bcap != src.bcap)
            FCC_TRY(dst.alloc((size_t)max_bodies, (size_t)max_cells, src.cap, src.ccap, src.bcap, stream));
        std::vector<MoveRange> mv;
        for (int s : order) {
            const Slot& S = slots[s];
            mv.push_back(MoveRange{(int)S.off, (int)S.off, (int)S.npad, S.coff, S.coff, S.ncells});
        }
        if (mv.empty()) return FCC_OK;
        CUDA_TRY(cudaMemcpyAsync(moves.p, mv.data(), mv.size() * sizeof(MoveRange), cudaMemcpyHostToDevice, stream));
        if (Ntot > 0)
            k_pool_gather_bodies<T><<<(int)((Ntot + 255) / 256), 256, 0, stream>>>(src.ptrs(), dst.ptrs(), moves.p,
                                                                                 (int)mv.size(), (int)Ntot, par());
        if (Ctot > 0)
            k_pool_gather_cells<T><<<(int)((Ctot + 255) / 256), 256, 0, stream>>>(src.ptrs(), dst.ptrs(), moves.p,
                                                                                (int)mv.size(), (int)Ctot);
        CUDA_TRY(cudaGetLastError());
        return sync_stream();
    }

    fcc_status graph_mode(int32_t enable, int32_t* active, int64_t* replays) override {
        if (enable >= 0) {
            use_graph = enable != 0;
            drop_graph();
        }
        if (active) *active = (use_graph && graph_ok) ? 1 : 0;
        if (replays) *replays = graph_launches;
        return FCC_OK;
    }

    fcc_status tune(int64_t steps, bool reorder, int32_t* chosen, double* best_us) override {
        Range range("fcc pool tune");
        FCC_TRY(compact());
        if (order.empty()) return fail(FCC_ERR_ARGUMENT, "pool: nothing to tune on (no simulations)");
        if (steps < 1) return fail(FCC_ERR_ARGUMENT, "pool: tune needs at least one step");
        // snapshot: arena into B, per-slot device state and the host mirror
        FCC_TRY(copy_arena(*A, *B));
        const int ns = nslots;
        std::vector<int> f0(ns), m0(ns);
        std::vector<long long> c0(ns), b0(ns), st0(ns);
        CUDA_TRY(cudaMemcpyAsync(f0.data(), flags.p, ns * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(m0.data(), maxcount.p, ns * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(c0.data(), clock.p, ns * sizeof(long long), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(b0.data(), builds.p, ns * sizeof(long long), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(st0.data(), stop.p, ns * sizeof(long long), cudaMemcpyDeviceToHost, stream));
        FCC_TRY(sync_stream());
        const std::vector<Slot> mirror = slots;
        const long long gstep0 = gstep;
        const int cap0 = cap, variant0 = variant;
        const Variant& cur = VARIANTS[variant < 0 ? 0 : variant];
        auto restore = [&]() -> fcc_status {
            if (A->cap != cap0) {
                FCC_TRY(A->alloc((size_t)max_bodies, (size_t)max_cells, cap0, ccap, bcap, stream));
            }
            cap = cap0;
            gstep = gstep0;
            FCC_TRY(copy_arena(*B, *A));
            slots = mirror;
            CUDA_TRY(cudaMemcpyAsync(flags.p, f0.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(maxcount.p, m0.data(), ns * sizeof(int), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(clock.p, c0.data(), ns * sizeof(long long), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(builds.p, b0.data(), ns * sizeof(long long), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(stop.p, st0.data(), ns * sizeof(long long), cudaMemcpyHostToDevice, stream));
            for (int s = 0; s < nslots; ++s) fl_in_h[s] = f0[s];
            return sync_stream();
        };
        int best = -1;
        double best_t = 1e300;
        // every candidate is timed twice, in alternation, and keeps its faster
        // time: the first launch of a kernel (lazy module loading) and clock
        // ramps do not decide the choice
        for (int pass = 0; pass < 2; ++pass)
        for (int v = 0; v < NVARIANTS; ++v) {
            const Variant& c = VARIANTS[v];
            if (sizeof(T) != 4 && !c.f64) continue;
            if (!reorder && c.family != cur.family) continue;
            variant = v;
            drop_graph();
            std::vector<long long> target(nslots, 0);
            for (int s : order) target[s] = slots[s].clock_h + steps;
            CUDA_TRY(cudaEventRecord(ev0, stream));
            tuning = true;
            const fcc_status st = advance_to(target);
            tuning = false;
            CUDA_TRY(cudaEventRecord(ev1, stream));
            CUDA_TRY(cudaEventSynchronize(ev1));
            float ms = 0;
            CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
            FCC_TRY(restore());
            if (st == FCC_ERR_FULL) {  // lists must regrow first: leave the launch shape untuned
                drop_graph();
                variant = variant0;
                if (chosen) *chosen = -1;
                if (best_us) *best_us = 0;
                return FCC_OK;
            }
            if (st != FCC_OK) return st;
            if (ms < best_t) {
                best_t = ms;
                best = v;
            }
        }
        drop_graph();
        variant = variant0;
        if (best < 0) return fail(FCC_ERR_UNSUPPORTED, "pool: no kernel variant to tune");
        {
            std::lock_guard<std::mutex> lk(tune_mutex());
            tune_table()[bucket()] = best;
        }
        user_set = false;
        FCC_TRY(apply_tuned());
        if (chosen) *chosen = best;
        if (best_us) *best_us = best_t * 1e3 / (double)steps;
        return FCC_OK;
    }

    // ------------------------------------------------------- queries --
    fcc_status check_slot(int32_t s) const {
        if (s < 0 || s >= max_sims || !slots[s].used) return fail(FCC_ERR_ARGUMENT, "pool: no simulation in this slot");
        return FCC_OK;
    }

    fcc_status slot_info(int32_t s, int32_t* active, int64_t* steps, int64_t* horizon) override {
        const bool ok = s >= 0 && s < max_sims && slots[s].used;
        if (active) *active = ok ? 1 : 0;
        if (steps) *steps = ok ? slots[s].step_h : 0;
        if (horizon) *horizon = ok ? slots[s].horizon : 0;
        return FCC_OK;
    }

    fcc_status usage(int64_t* nb, int64_t* nc, int32_t* ns, int64_t* mb, int64_t* mc, int32_t* ms) override {
        FCC_TRY(compact());
        if (nb) *nb = Ntot;
        if (nc) *nc = Ctot;
        if (ns) *ns = (int32_t)order.size();
        if (mb) *mb = max_bodies;
        if (mc) *mc = max_cells;
        if (ms) *ms = max_sims;
        return FCC_OK;
    }

    fcc_status get_state(int32_t s, fcc_bodies_host* o, int64_t* clk, double* t, int64_t* stp) override {
        FCC_TRY(check_slot(s));
        FCC_TRY(compact());
        const Slot& S = slots[s];
        const SimSpec<T>& P = S.spec;
        const int64_t N = P.N;
        if (o) {
            if (o->n != N || o->ncoef != P.nc) return fail(FCC_ERR_DIMENSION, "state buffers do not match the simulation");
            Arena<T>& a = *A;
            const size_t n = (size_t)N;
            if (n > 0) {
                FCC_TRY(st_xch.reserve(n * (3 + (size_t)P.nc), stream));
                double* dx = st_xch.p();
                k_store_host<T><<<(int)std::min<size_t>((n * P.nc + 255) / 256, (size_t)nsm * 8), 256, 0, stream>>>(
                    ptrs(), par(), (int)S.off, (int)n, dx, dx + n, dx + 2 * n, dx + 3 * n, P.nc, P.K, nullptr, nullptr);
                CUDA_TRY(cudaGetLastError());
                if (o->x) CUDA_TRY(cudaMemcpyAsync(o->x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                if (o->y) CUDA_TRY(cudaMemcpyAsync(o->y, dx + n, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                if (o->theta)
                    CUDA_TRY(cudaMemcpyAsync(o->theta, dx + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                if (o->coef)
                    CUDA_TRY(cudaMemcpyAsync(o->coef, dx + 3 * n, n * P.nc * sizeof(double), cudaMemcpyDeviceToHost,
                                             stream));
                if (o->imgx)
                    CUDA_TRY(cudaMemcpyAsync(o->imgx, a.imgx.p + S.off, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
                if (o->imgy)
                    CUDA_TRY(cudaMemcpyAsync(o->imgy, a.imgy.p + S.off, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
            }
            for (size_t i = 0; i < n; ++i) {
                if (o->R0) o->R0[i] = (double)P.R0[i];
                if (o->type) o->type[i] = P.type[i];
                if (o->parent) o->parent[i] = P.parent[i];
            }
            FCC_TRY(sync_stream());
        }
        if (clk) *clk = S.clock_h;
        if (t) *t = (double)S.t_h;
        if (stp) *stp = S.step_h;
        return FCC_OK;
    }

    fcc_status observable(int32_t s, int which, int32_t typ, double* out, int64_t* count) override {
        FCC_TRY(check_slot(s));
        if (which < 0 || which > 2) return fail(FCC_ERR_ARGUMENT, "pool: which must be 0, 1 or 2");
        FCC_TRY(compact());
        const Slot& S = slots[s];
        const int64_t N = S.spec.N;
        const double* v = nullptr;
        if (N > 0) {
            FCC_TRY(obs.reserve(3 * (size_t)N, stream));
            k_observables<T><<<(int)((N + 127) / 128), 128, 0, stream>>>(ptrs(), par(), (int)S.off, (int)N, obs.dev.p);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaMemcpyAsync(obs.host, obs.dev.p, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, stream));
            FCC_TRY(sync_stream());
            v = obs.host;
        }
        int64_t w = 0;
        for (int64_t i = 0; i < N; ++i) {
            if (typ != 0 && S.spec.type[i] != typ) continue;
            if (out) out[w] = v[3 * i + which];
            ++w;
        }
        if (count) *count = w;
        return FCC_OK;
    }

    fcc_status slot_builds(int32_t s, int64_t* b) override {
        FCC_TRY(check_slot(s));
        long long v = 0;
        CUDA_TRY(cudaMemcpyAsync(&v, builds.p + s, sizeof(long long), cudaMemcpyDeviceToHost, stream));
        FCC_TRY(sync_stream());
        if (b) *b = v + slots[s].builds_adjust;
        return FCC_OK;
    }

    fcc_status config(int32_t v, int32_t steps) override {
        if (v < -1 || v >= NVARIANTS) return fail(FCC_ERR_ARGUMENT, "pool: no such kernel variant");
        if (v >= 0 && sizeof(T) != 4 && !VARIANTS[v].f64)
            return fail(FCC_ERR_UNSUPPORTED, "pool: this kernel variant has no FP64 build");
        if (steps < 0) return fail(FCC_ERR_ARGUMENT, "pool: steps per launch must be >= 0");
        variant = v;
        user_set = v >= 0;
        spl = steps > 0 ? steps : 512;
        drop_graph();
        return FCC_OK;
    }

    fcc_status variant_info(int32_t* v, int32_t* L, int32_t* S_, int32_t* blk, int32_t* minb, int32_t* g) override {
        if (v) *v = variant < 0 ? 0 : variant;
        if (L) *L = var().L;
        if (S_) *S_ = var().S;
        if (blk) *blk = var().blk;
        if (minb) *minb = sizeof(T) == 4 ? var().minb : 1;
        if (g) *g = grid;
        return FCC_OK;
    }

    fcc_status timing(double* ms, int64_t* launches, int64_t* body_steps) override {
        if (ms) *ms = last_ms;
        if (launches) *launches = last_launches;
        if (body_steps) *body_steps = last_body_steps;
        return FCC_OK;
    }
};

}  // namespace

struct fcc_pool {
    std::unique_ptr<PoolBase> impl;
    int device = 0;
};

extern "C" {

fcc_status fcc_pool_bytes(const fcc_pool_params* q, int64_t* bytes) {
    if (!q || !bytes) return fail(FCC_ERR_ARGUMENT, "null argument");
    if (q->precision == 32) *bytes = (int64_t)pool_bytes<float>(*q);
    else if (q->precision == 64) *bytes = (int64_t)pool_bytes<double>(*q);
    else return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    return FCC_OK;
}

fcc_status fcc_pool_create(const fcc_pool_params* q, fcc_pool** out) {
    if (!out) return fail(FCC_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!q) return fail(FCC_ERR_ARGUMENT, "null params");
    std::unique_ptr<fcc_pool> h(new fcc_pool);
    fcc_status st;
    if (q->precision == 64) {
        auto e = std::make_unique<Pool<double>>();
        st = e->init(*q);
        h->impl = std::move(e);
    } else if (q->precision == 32) {
        auto e = std::make_unique<Pool<float>>();
        st = e->init(*q);
        h->impl = std::move(e);
    } else {
        return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    }
    if (st != FCC_OK) return st;
    cudaGetDevice(&h->device);
    *out = h.release();
    return FCC_OK;
}

fcc_status fcc_pool_destroy(fcc_pool* pool) {
    if (pool) cudaSetDevice(pool->device);
    delete pool;
    return FCC_OK;
}

#define POOL_CALL(expr)                                                  \
    do {                                                                 \
        if (!pool) return fail(FCC_ERR_ARGUMENT, "null pool");           \
        cudaError_t e_ = cudaSetDevice(pool->device);                    \
        if (e_ != cudaSuccess) return cuda_fail(e_, "cudaSetDevice");    \
        return pool->impl->expr;                                         \
    } while (0)

fcc_status fcc_pool_add(fcc_pool* pool, const fcc_params* params, const fcc_bodies_host* bodies, int64_t horizon,
                        int32_t* slot) {
    POOL_CALL(add(params, bodies, horizon, 0, 0.0, slot));
}
fcc_status fcc_pool_add_at(fcc_pool* pool, const fcc_params* params, const fcc_bodies_host* bodies, int64_t clock,
                           double t, int64_t horizon, int32_t* slot) {
    POOL_CALL(add(params, bodies, horizon, clock, t, slot));
}
fcc_status fcc_pool_remove(fcc_pool* pool, int32_t slot) { POOL_CALL(remove(slot)); }
fcc_status fcc_pool_run(fcc_pool* pool, int64_t n) { POOL_CALL(run(n)); }
fcc_status fcc_pool_slot(fcc_pool* pool, int32_t slot, int32_t* active, int64_t* steps, int64_t* horizon) {
    POOL_CALL(slot_info(slot, active, steps, horizon));
}
fcc_status fcc_pool_usage(fcc_pool* pool, int64_t* bodies, int64_t* cells, int32_t* sims, int64_t* max_bodies,
                          int64_t* max_cells, int32_t* max_sims) {
    POOL_CALL(usage(bodies, cells, sims, max_bodies, max_cells, max_sims));
}
fcc_status fcc_pool_get_state(fcc_pool* pool, int32_t slot, fcc_bodies_host* out, int64_t* clock, double* t,
                              int64_t* step) {
    POOL_CALL(get_state(slot, out, clock, t, step));
}
fcc_status fcc_pool_observable(fcc_pool* pool, int32_t slot, int32_t which, int32_t type, double* out,
                               int64_t* count) {
    POOL_CALL(observable(slot, which, type, out, count));
}
fcc_status fcc_pool_builds(fcc_pool* pool, int32_t slot, int64_t* nbuilds) { POOL_CALL(slot_builds(slot, nbuilds)); }
fcc_status fcc_pool_config(fcc_pool* pool, int32_t variant, int32_t steps_per_launch) {
    POOL_CALL(config(variant, steps_per_launch));
}
fcc_status fcc_pool_variant(fcc_pool* pool, int32_t* variant, int32_t* lanes, int32_t* slots, int32_t* block,
                            int32_t* min_blocks, int32_t* grid) {
    POOL_CALL(variant_info(variant, lanes, slots, block, min_blocks, grid));
}
fcc_status fcc_pool_last_timing(fcc_pool* pool, double* ms, int64_t* launches, int64_t* body_steps) {
    POOL_CALL(timing(ms, launches, body_steps));
}
fcc_status fcc_pool_tune(fcc_pool* pool, int64_t steps, int32_t reorder, int32_t* variant, double* us_per_step) {
    POOL_CALL(tune(steps, reorder != 0, variant, us_per_step));
}
fcc_status fcc_pool_graph(fcc_pool* pool, int32_t enable, int32_t* active, int64_t* replays) {
    POOL_CALL(graph_mode(enable, active, replays));
}

}  // extern "C"
