// fcc_noalloc.cu — neighbour build that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside a device-memory
// pool it does not own, allocators that forbid foreign allocations in a
// serving process, or embedders whose memory budget is fixed up front.  fcc_build_neighbors_noalloc serves them: the caller
// passes its input and output arrays already on the device, and every other
// buffer the cell-list / neighbour-list kernels need lives in the static
// device array below, which each GPU that loads this library holds until the
// process exits.  Included by fcc_lib.cu (one translation unit).

namespace {

// Scratch of the no-allocation build: the body records, cell bookkeeping and
// run state of a one-simulation engine, for at most FCC_NOALLOC_MAX_BODIES
// bodies (records sized for FP64) and FCC_NOALLOC_MAX_CELLS grid cells.
constexpr size_t NA_REC = (size_t)FCC_NOALLOC_MAX_BODIES * RECW * sizeof(double);
constexpr size_t NA_BODY = (size_t)FCC_NOALLOC_MAX_BODIES * sizeof(int);
constexpr size_t NA_CELL = (size_t)FCC_NOALLOC_MAX_CELLS * sizeof(int);
constexpr size_t NA_DESC = (sizeof(SimDesc<double>) + 255) / 256 * 256;
constexpr size_t NA_OFF_REC = 0;
constexpr size_t NA_OFF_SIMOF = NA_OFF_REC + NA_REC;
constexpr size_t NA_OFF_CELLID = NA_OFF_SIMOF + NA_BODY;
constexpr size_t NA_OFF_SLOT = NA_OFF_CELLID + NA_BODY;
constexpr size_t NA_OFF_PERM = NA_OFF_SLOT + NA_BODY;
constexpr size_t NA_OFF_CCOUNT = NA_OFF_PERM + NA_BODY;
constexpr size_t NA_OFF_CSIM = NA_OFF_CCOUNT + NA_CELL;
constexpr size_t NA_OFF_CSTART = NA_OFF_CSIM + NA_CELL;
constexpr size_t NA_OFF_CSTOP = NA_OFF_CSTART + NA_CELL;
constexpr size_t NA_OFF_DESC = NA_OFF_CSTOP + NA_CELL;
constexpr size_t NA_OFF_STATE = NA_OFF_DESC + NA_DESC;  // flags, maxcount, clock, builds, sync
constexpr size_t NA_BYTES = NA_OFF_STATE + 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current (host code may not use the symbol itself).
unsigned char* g_noalloc_addr[64] = {nullptr};
std::mutex g_noalloc_mutex;

struct NaState {
    int flags, maxcount;
    long long clock, builds;
    GridSync sync;
};

// Clear what the build needs at zero (cell counts, body -> simulation map,
// cell -> simulation map, run state) and write the simulation descriptor.
template <class T>
__global__ void k_noalloc_setup(unsigned char* scr, SimDesc<T> desc, int n, int ncells) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    int* sim_of = reinterpret_cast<int*>(scr + NA_OFF_SIMOF);
    int* ccount = reinterpret_cast<int*>(scr + NA_OFF_CCOUNT);
    int* csim = reinterpret_cast<int*>(scr + NA_OFF_CSIM);
    for (int i = tid; i < n; i += nthr) sim_of[i] = 0;
    for (int c = tid; c < ncells; c += nthr) {
        ccount[c] = 0;
        csim[c] = 0;
    }
    if (tid == 0) {
        *reinterpret_cast<SimDesc<T>*>(scr + NA_OFF_DESC) = desc;
        NaState* st = reinterpret_cast<NaState*>(scr + NA_OFF_STATE);
        st->flags = F_ACTIVE | F_CONTACT | F_NEED;
        st->maxcount = 0;
        st->clock = 0;
        st->builds = 0;
        st->sync = GridSync{0, 0, 0, 1};
    }
}

// 0-based internal lists -> the reference's 1-based cell list and
// neighbour matrix (empty cells: start = 1, stop = 0; idx beyond count: 0).
__global__ void k_noalloc_finish(const unsigned char* scr, int n, int ncells, int cap, int32_t* cellid,
                                 int32_t* perm, int32_t* start, int32_t* stop, int32_t* idx, const int32_t* count) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    const int* icell = reinterpret_cast<const int*>(scr + NA_OFF_CELLID);
    const int* iperm = reinterpret_cast<const int*>(scr + NA_OFF_PERM);
    const int* cst = reinterpret_cast<const int*>(scr + NA_OFF_CSTART);
    const int* csp = reinterpret_cast<const int*>(scr + NA_OFF_CSTOP);
    for (int i = tid; i < n; i += nthr) {
        cellid[i] = icell[i] + 1;
        perm[i] = iperm[i] + 1;
        const int k = count[i];
        for (int q = 0; q < cap; ++q) {
            const size_t o = (size_t)i * cap + q;
            idx[o] = q < k ? idx[o] + 1 : 0;
        }
    }
    for (int c = tid; c < ncells; c += nthr) {
        const bool empty = csp[c] <= cst[c];
        start[c] = empty ? 1 : cst[c] + 1;
        stop[c] = empty ? 0 : csp[c];
    }
}

fcc_status noalloc_scratch(unsigned char** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(FCC_ERR_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return FCC_OK;
}

template <class T>
fcc_status build_neighbors_noalloc_t(int64_t n, const T* x, const T* y, const T* rmax, double Lx, double Ly,
                                     double cutoff, double range, int32_t cap, int32_t* cellid, int32_t* perm,
                                     int32_t* start, int32_t* stop, int32_t* idx, int32_t* count,
                                     cudaStream_t st) {
    SimDesc<T> s{};
    s.Lx = (T)Lx;
    s.Ly = (T)Ly;
    int64_t gx = 0, gy = 0;
    FCC_TRY(cell_grid_dims((double)s.Lx, (double)s.Ly, cutoff, &gx, &gy));
    if (gx * gy > FCC_NOALLOC_MAX_CELLS)
        return fail(FCC_ERR_ARGUMENT, "the cell grid (" + std::to_string(gx * gy) +
                                          " cells) exceeds FCC_NOALLOC_MAX_CELLS = " +
                                          std::to_string(FCC_NOALLOC_MAX_CELLS));
    const int ncx = (int)gx, ncy = (int)gy;
    s.wx = s.Lx / (T)ncx;
    s.wy = s.Ly / (T)ncy;
    s.ncx = ncx;
    s.ncy = ncy;
    s.ncells = ncx * ncy;
    s.n = (int)n;
    s.nbrange = (T)range;
    s.skin = T(0);
    unsigned char* scr = nullptr;
    FCC_TRY(noalloc_scratch(&scr));
    NaState* state = reinterpret_cast<NaState*>(scr + NA_OFF_STATE);
    DevPtrs<T> d{};
    d.sims = reinterpret_cast<const SimDesc<T>*>(scr + NA_OFF_DESC);
    d.nsims = 1;
    d.Ntot = (int)n;
    d.Ctot = s.ncells;
    d.cap = cap;
    d.sim_of = reinterpret_cast<const int*>(scr + NA_OFF_SIMOF);
    d.rec0 = d.rec1 = reinterpret_cast<T*>(scr + NA_OFF_REC);
    d.cellid = reinterpret_cast<int*>(scr + NA_OFF_CELLID);
    d.slot = reinterpret_cast<int*>(scr + NA_OFF_SLOT);
    d.perm = reinterpret_cast<int*>(scr + NA_OFF_PERM);
    d.cstart = reinterpret_cast<int*>(scr + NA_OFF_CSTART);
    d.cstop = reinterpret_cast<int*>(scr + NA_OFF_CSTOP);
    d.ccount = reinterpret_cast<int*>(scr + NA_OFF_CCOUNT);
    d.cell_sim = reinterpret_cast<const int*>(scr + NA_OFF_CSIM);
    d.nb_idx = idx;
    d.nb_count = count;
    d.flags = &state->flags;
    d.maxcount = &state->maxcount;
    d.clock = &state->clock;
    d.builds = &state->builds;
    d.sync = &state->sync;
    const int grid = (int)((n + 255) / 256);
    const int cgrid = (s.ncells + 255) / 256;
    k_noalloc_setup<T><<<std::max(grid, cgrid), 256, 0, st>>>(scr, s, (int)n, s.ncells);
    k_pack_head<T><<<grid, 256, 0, st>>>(d.rec0, x, y, rmax, (int)n);
    k_phase_count<T><<<grid, 256, 0, st>>>(d, 0);
    k_phase_scan<T><<<1, 1024, 0, st>>>(d);
    k_phase_scatter<T><<<grid, 256, 0, st>>>(d);
    k_phase_sort<T><<<cgrid, 256, 0, st>>>(d);
    k_phase_neighbors<T><<<grid, 256, 0, st>>>(d, 0);
    k_noalloc_finish<<<std::max(grid, cgrid), 256, 0, st>>>(scr, (int)n, s.ncells, cap, cellid, perm, start, stop,
                                                           idx, count);
    CUDA_TRY(cudaGetLastError());
    return FCC_OK;
}

}  // namespace

extern "C" fcc_status fcc_build_neighbors_noalloc(int32_t precision, int64_t n, const void* x, const void* y,
                                                  const void* rmax, double Lx, double Ly, double cutoff, double range,
                                                  int32_t cap, int32_t* cellid, int32_t* perm, int32_t* start,
                                                  int32_t* stop, int32_t* idx, int32_t* count, void* stream) {
    if (precision != 32 && precision != 64) return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    if (n < 0 || cap < 1) return fail(FCC_ERR_ARGUMENT, "n must be >= 0 and cap >= 1");
    if (n > FCC_NOALLOC_MAX_BODIES)
        return fail(FCC_ERR_ARGUMENT, "n = " + std::to_string(n) + " exceeds FCC_NOALLOC_MAX_BODIES = " +
                                          std::to_string(FCC_NOALLOC_MAX_BODIES));
    {  // the grid first: a cutoff or box that is not finite and positive, or a grid beyond the scratch
        int64_t gx = 0, gy = 0;
        const fcc_status g = cell_grid_dims(Lx, Ly, cutoff, &gx, &gy);
        if (g == FCC_ERR_UNSUPPORTED || (g == FCC_OK && gx * gy > FCC_NOALLOC_MAX_CELLS))
            return fail(FCC_ERR_ARGUMENT, "the cell grid exceeds FCC_NOALLOC_MAX_CELLS = " +
                                              std::to_string(FCC_NOALLOC_MAX_CELLS) + " cells");
        if (g != FCC_OK) return g;
    }
    if (n == 0) return FCC_OK;
    if (!x || !y || !rmax || !cellid || !perm || !start || !stop || !idx || !count)
        return fail(FCC_ERR_ARGUMENT, "null device array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == 64)
        return build_neighbors_noalloc_t<double>(n, static_cast<const double*>(x), static_cast<const double*>(y),
                                                 static_cast<const double*>(rmax), Lx, Ly, cutoff, range, cap, cellid,
                                                 perm, start, stop, idx, count, st);
    return build_neighbors_noalloc_t<float>(n, static_cast<const float*>(x), static_cast<const float*>(y),
                                            static_cast<const float*>(rmax), Lx, Ly, cutoff, range, cap, cellid, perm,
                                            start, stop, idx, count, st);
}
