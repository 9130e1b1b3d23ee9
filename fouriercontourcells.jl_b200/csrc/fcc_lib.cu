// fcc_lib.cu — host runtime of libfcc_b200: the C ABI of include/fcc.h.
//
// An Engine<T> owns the device state of one simulation (the body, cell and
// neighbour arrays of fcc_device.cuh), one CUDA stream and the launch
// configuration of the persistent step kernel.  Every reference entry point
// maps onto it: Simulation(...) -> fcc_create (src/simulation.jl:66-105),
// step! -> fcc_step (:165-173), run! -> fcc_run (:220-235 and
// ext/FourierContourCellsCUDAExt.jl:144-180), compute_gradients! ->
// fcc_compute_gradients (:150-158), update_neighbors! -> fcc_update_neighbors
// (:132-142), shape_index & co. -> fcc_shape_index (src/observables.jl:7-18).

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fcc.h"
#include "../../include/fcc_user_terms.h"
#include "fcc_kernels.cuh"

#ifndef FCC_NVTX
#define FCC_NVTX 1  // named ranges around the host phases for nsys / ncu timelines (free without a tool)
#endif
#if FCC_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

namespace fcc {
// A named range on the profiler timeline for the lifetime of the object.
struct Range {
#if FCC_NVTX
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
#else
    explicit Range(const char*) {}
#endif
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};
}  // namespace fcc

using namespace fcc;

namespace {

thread_local std::string g_err;

fcc_status fail(fcc_status code, const std::string& msg) {
    g_err = msg;
    return code;
}
fcc_status cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? FCC_ERR_NOMEM : FCC_ERR_CUDA;
}
#define CUDA_TRY(x)                                      \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #x); \
    } while (0)
#define FCC_TRY(x)                        \
    do {                                  \
        fcc_status s_ = (x);              \
        if (s_ != FCC_OK) return s_;      \
    } while (0)

// Device buffer owned by an engine.
template <class V>
struct DBuf {
    V* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    fcc_status alloc(size_t count, cudaStream_t st) {
        release();
        n = count;
        if (count == 0) return FCC_OK;
        CUDA_TRY(cudaMalloc(&p, count * sizeof(V)));
        CUDA_TRY(cudaMemsetAsync(p, 0, count * sizeof(V), st));
        return FCC_OK;
    }
    fcc_status upload(const std::vector<V>& h, cudaStream_t st) {
        FCC_TRY(alloc(h.size(), st));
        if (!h.empty()) CUDA_TRY(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st));
        return FCC_OK;
    }
};

// blocks of 256 threads for the neighbour phase (8 lanes per body), capped;
// the phase loops over the rest
inline int neighbor_grid(int64_t n) { return (int)std::min<int64_t>((n + 31) / 32, 148 * 64); }

// Device staging area for host data on its way to a kernel, reused across
// calls: it grows and never shrinks, so an admission allocates nothing once a
// simulation of that size has been seen (allocation and release of device
// memory synchronise the device and cost milliseconds).
template <class V>
struct Stage {
    DBuf<V> buf;
    fcc_status upload(const std::vector<V>& h, cudaStream_t st) {
        FCC_TRY(reserve(h.size(), st));
        if (!h.empty()) CUDA_TRY(cudaMemcpyAsync(buf.p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st));
        return FCC_OK;
    }
    fcc_status reserve(size_t count, cudaStream_t st) {
        if (count > buf.n) FCC_TRY(buf.alloc(count, st));
        return FCC_OK;
    }
    V* p() const { return buf.p; }
};

// The device's address of page-locked host memory that the device reads and
// writes in place (every page-locked allocation is mapped under unified
// addressing), or null for any other pointer (pageable memory, device
// memory, null).
template <class V>
V* mapped_view(V* p) {
    if (!p) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();  // not a pointer the runtime knows: not mapped
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
    return static_cast<V*>(a.devicePointer);
}

// Device output of k_observables and its pinned host copy, grown on demand
// and reused: an observable query allocates nothing after the first at its
// size (allocation and release of device memory synchronise the device and
// cost milliseconds).
struct ObsArea {
    DBuf<double> dev;
    double* host = nullptr;
    size_t cap = 0;
    ObsArea() = default;
    ObsArea(const ObsArea&) = delete;
    ObsArea& operator=(const ObsArea&) = delete;
    ~ObsArea() {
        if (host) cudaFreeHost(host);
    }
    fcc_status reserve(size_t n, cudaStream_t st) {
        if (n <= cap) return FCC_OK;
        if (host) cudaFreeHost(host);
        host = nullptr;
        cap = 0;
        FCC_TRY(dev.alloc(n, st));
        CUDA_TRY(cudaMallocHost(&host, n * sizeof(double)));
        cap = n;
        return FCC_OK;
    }
};

const double PI = 3.14159265358979323846;

// Launch configurations of the step kernel: lanes per body L, node slots per
// lane S (L*S >= 40 covers the nθ = 40 contour in one pass), and the minimum
// resident 256-thread blocks per SM the register budget is cut for.

template <class T, int L, int S, int BLK, int MB>
void* step_fn(bool one, bool split) {
    if (one)
        return split ? (void*)k_step<T, L, S, true, true, BLK, MB> : (void*)k_step<T, L, S, true, false, BLK, MB>;
    return split ? (void*)k_step<T, L, S, false, true, BLK, MB> : (void*)k_step<T, L, S, false, false, BLK, MB>;
}

// `family`: variants of one family give bit-identical trajectories (same
// lanes x node slots, and — measured, since the compiler may fuse either
// product of a*b + c*d differently under another register budget — the same
// rounding); the autotuner keeps within the family unless told to reorder.
struct Variant {
    int L, S, blk, minb;
    void* (*f32)(bool, bool);
    void* (*f64)(bool, bool);
    size_t stage32, stage64;  // shared-memory neighbour stage per warp
    int family;
};

const Variant VARIANTS[] = {
    {8, 5, 256, 2, step_fn<float, 8, 5, 256, 2>, step_fn<double, 8, 5, 256, 1>, stage_bytes_per_warp<float, 8>(),
     stage_bytes_per_warp<double, 8>(), 0},
    {4, 10, 256, 2, step_fn<float, 4, 10, 256, 2>, nullptr, stage_bytes_per_warp<float, 4>(), 0, 1},
    {16, 3, 256, 2, step_fn<float, 16, 3, 256, 2>, nullptr, stage_bytes_per_warp<float, 16>(), 0, 2},
    {8, 5, 128, 5, step_fn<float, 8, 5, 128, 5>, nullptr, stage_bytes_per_warp<float, 8>(), 0, 3},
    {16, 3, 128, 5, step_fn<float, 16, 3, 128, 5>, nullptr, stage_bytes_per_warp<float, 16>(), 0, 2},
    {8, 5, 224, 2, step_fn<float, 8, 5, 224, 2>, step_fn<double, 8, 5, 224, 1>, stage_bytes_per_warp<float, 8>(),
     stage_bytes_per_warp<double, 8>(), 0},
};
constexpr int NVARIANTS = sizeof(VARIANTS) / sizeof(VARIANTS[0]);
constexpr int LANES = 8, SLOTS = 5;  // compute_gradients and the FP64 step

// A simulation as set up from the reference's constructor arguments
// (src/simulation.jl:66-105), validated and converted to T, with local body
// ids: the part of an engine that does not depend on where its bodies sit.
template <class T>
struct SimSpec {
    SimDesc<T> desc{};  // body_off = cell_off = 0
    int64_t N = 0;
    int K = 0, nc = 0, nth = 0, ncx = 1, ncy = 1;
    bool has_contact = false, split = false;
    std::vector<int32_t> type, parent;
    std::vector<T> R0;
    std::vector<int> chc, chi, bdc, bdi;  // children and bond partners per body (local ids)
    int ccap = 1, bcap = 1;
};

// sqrt(2 D dt) of every type, evaluated in T exactly as the device would
// (the step reads them from the descriptor)
template <class T>
void set_noise_amplitudes(SimDesc<T>& s) {
    for (int t = 0; t < MT; ++t) {
        const T a = T(2) * s.Dr[t], b = T(2) * s.Dt[t];
        s.sigr[t] = std::sqrt(T(a * s.dt));
        s.sigt[t] = std::sqrt(T(b * s.dt));
    }
}

// Cell grid of CellList(box, cutoff, n) (src/neighbors.jl:27-45): floor(L /
// cutoff) cells per side, collapsed to 1 below 3.  The box sides and the
// cutoff must be finite and positive (the reference's floor(Int, L/cutoff)
// throws otherwise), and the side counts are formed in 64 bits, each capped,
// before anything narrows them.
fcc_status cell_grid_dims(double Lx, double Ly, double cutoff, int64_t* ncx, int64_t* ncy) {
    if (!(std::isfinite(cutoff) && cutoff > 0))
        return fail(FCC_ERR_ARGUMENT, "cutoff must be a finite positive number");
    if (!(std::isfinite(Lx) && Lx > 0 && std::isfinite(Ly) && Ly > 0))
        return fail(FCC_ERR_ARGUMENT, "box sides must be finite positive numbers");
    auto side = [&](double L, int64_t* out) -> fcc_status {
        const double m = std::floor(L / cutoff);
        if (!(m < (double)(1 << 28))) return fail(FCC_ERR_UNSUPPORTED, "cell grid too large");
        *out = m >= 3 ? (int64_t)m : 1;
        return FCC_OK;
    };
    FCC_TRY(side(Lx, ncx));
    return side(Ly, ncy);
}

template <class T>
fcc_status make_spec(const fcc_params* p, const fcc_bodies_host* b, SimSpec<T>& sp) {
    // validation in the order of src/simulation.jl:66-105
    if (!p || !b) return fail(FCC_ERR_ARGUMENT, "null argument");
    if (p->ntypes < 1 || p->ntypes > FCC_MAX_TYPES || !p->types)
        return fail(FCC_ERR_ARGUMENT, "types must hold 1..8 BodyType entries");
    for (int t = 0; t < p->ntypes; ++t) {
        if (p->types[t].parent_drag != 0 && p->types[t].parent_drag != 1)
            return fail(FCC_ERR_ARGUMENT, "drag must be :substrate or :parent");
        if (p->types[t].maxmode < 0) return fail(FCC_ERR_ARGUMENT, "a body type's maxmode must be >= 0");
    }
    if (p->nterms < 0 || p->nterms > FCC_MAX_TERMS || (p->nterms > 0 && !p->terms))
        return fail(FCC_ERR_ARGUMENT, "energy terms must be BodyTerms, ContactTerms or BondTerms");
    int nuser[3] = {0, 0, 0};
    for (int q = 0; q < p->nterms; ++q) {
        const fcc_term& ft = p->terms[q];
        if (ft.kind < FCC_TENSION || ft.kind > FCC_USER_BOND)
            return fail(FCC_ERR_ARGUMENT, "energy terms must be BodyTerms, ContactTerms or BondTerms");
        if (ft.kind >= FCC_USER_BODY) {
            const int k = ft.kind - FCC_USER_BODY;
            const int have = k == 0 ? fcc_user::n_body : k == 1 ? fcc_user::n_contact : fcc_user::n_bond;
            if (ft.user < 0 || ft.user >= have) return fail(FCC_ERR_ARGUMENT, "no compiled user term with this index");
            if (++nuser[k] > MUT)
                return fail(FCC_ERR_UNSUPPORTED, "at most " + std::to_string(MUT) + " user terms of each kind");
        }
        if (ft.ntypes_on < 0 || ft.ntypes_on > FCC_MAX_TYPES) return fail(FCC_ERR_ARGUMENT, "OnTypes: bad type list");
        if (ft.kind == FCC_OVERLAP && (ft.nJ < 1 || ft.nJ > FCC_MAX_TYPES))
            return fail(FCC_ERR_DIMENSION, "coupling tables must be square and equal-sized");
    }
    int64_t& N = sp.N;
    N = b->n;
    if (N < 0) return fail(FCC_ERR_DIMENSION, "inconsistent body array lengths");
    if (N > (1 << 27)) return fail(FCC_ERR_UNSUPPORTED, "at most 2^27 bodies per simulation");
    int32_t maxtype = 0;
    for (int64_t i = 0; i < N; ++i) {
        if (b->type[i] > p->ntypes) return fail(FCC_ERR_ARGUMENT, "body type without BodyType entry");
        if (b->type[i] < 1) return fail(FCC_ERR_ARGUMENT, "body type ids are 1-based");
        maxtype = std::max(maxtype, b->type[i]);
    }
    for (int q = 0; q < p->nterms; ++q) {
        const fcc_term& ft = p->terms[q];
        if (ft.kind == FCC_OVERLAP && ft.nJ > 1 && ft.nJ < maxtype)
            return fail(FCC_ERR_DIMENSION, "Overlap coupling table smaller than the number of body types");
    }
    for (int64_t i = 0; i < N; ++i) {  // check_parents, src/simulation.jl:108-118
        int64_t pp = b->parent[i];
        if (pp < 1 || pp > N)
            return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has parent " + std::to_string(pp) +
                                              " outside 1:" + std::to_string(N));
        if (!p->types[b->type[i] - 1].parent_drag) continue;
        if (pp == i + 1)
            return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has drag = :parent but is its own parent");
        if (p->types[b->type[pp - 1] - 1].parent_drag)
            return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has drag = :parent, but so has its parent " +
                                              std::to_string(pp) + " (one level only)");
    }
    int& K = sp.K;
    int& nth = sp.nth;
    int& nc = sp.nc;
    K = b->ncoef / 2;
    nth = p->ntheta;
    if (K + 1 < 2) return fail(FCC_ERR_ARGUMENT, "maxmode must be ≥ 2");
    if (!(nth > 2 * (K + 1))) return fail(FCC_ERR_ARGUMENT, "nθ must exceed 2·maxmode");
    nc = 2 * K + 1;
    if (b->ncoef != nc) return fail(FCC_ERR_DIMENSION, "coefficient rows must be odd: [a₀; aₙ; bₙ]");
    if (K > KM) return fail(FCC_ERR_UNSUPPORTED, "the kernels support maxmode ≤ 10");
    for (int t = 0; t < p->ntypes; ++t)
        if (p->types[t].maxmode > K + 1)
            return fail(FCC_ERR_ARGUMENT, "a body type's maxmode exceeds the simulation's (" + std::to_string(K + 1) + ")");
    if (!(p->skin >= 0)) return fail(FCC_ERR_ARGUMENT, "skin must be non-negative");

    // simulation descriptor (convert_precision: every parameter to T)
    SimDesc<T>& s = sp.desc;
    s = SimDesc<T>{};
    std::vector<T>& R0_h = sp.R0;
    int& ncx = sp.ncx;
    int& ncy = sp.ncy;
    bool& has_contact = sp.has_contact;
    bool& split = sp.split;
    has_contact = false;
    s.Lx = (T)p->Lx;
    s.Ly = (T)p->Ly;
    s.invLx = T(1) / s.Lx;
    s.invLy = T(1) / s.Ly;
    s.dt = (T)p->dt;
    s.skin = (T)p->skin;
    // contact_range (src/energies/contact.jl:54): the largest interaction
    // range of the contact terms, in T (0 for the built-in ones)
    s.crange = T(0);
    for (int q = 0; q < p->nterms; ++q)
        if (p->terms[q].kind == FCC_USER_CONTACT)
            s.crange = std::max(s.crange, fcc_user::contact_range<T>(p->terms[q].user, (T)p->terms[q].a,
                                                                    (T)p->terms[q].b));
    if (!(s.crange >= T(0))) return fail(FCC_ERR_ARGUMENT, "interaction ranges must be non-negative");
    s.nbrange = s.crange + s.skin;
    s.dphi = (T)(2 * PI / nth);
    R0_h.resize(N);
    double maxR0 = 0;
    for (int64_t i = 0; i < N; ++i) {
        R0_h[i] = (T)b->R0[i];
        maxR0 = std::max(maxR0, (double)R0_h[i]);
    }
    const double cutoff = 2 * maxR0 * (1 + SHAPE_BOUND) + (double)s.crange + p->skin;  // src/simulation.jl:90
    {
        int64_t gx = 0, gy = 0;
        FCC_TRY(cell_grid_dims((double)s.Lx, (double)s.Ly, cutoff, &gx, &gy));
        if (gx * gy > (1 << 28)) return fail(FCC_ERR_UNSUPPORTED, "cell grid too large");
        ncx = (int)gx;
        ncy = (int)gy;
    }
    s.wx = s.Lx / (T)ncx;
    s.wy = s.Ly / (T)ncy;
    s.ncx = ncx;
    s.ncy = ncy;
    s.cell_off = 0;
    s.ncells = ncx * ncy;
    s.body_off = 0;
    s.n = (int)N;
    s.nth = nth;
    s.K = K;
    s.k0 = (uint32_t)(p->seed & 0xffffffffu);
    s.k1 = (uint32_t)(p->seed >> 32);
    s.ntypes = p->ntypes;
    s.rewrap = (ncx < 3 || ncy < 3) ? 1 : 0;
    for (int t = 0; t < p->ntypes; ++t) {
        const fcc_body_type& bt = p->types[t];
        s.v0[t] = (T)bt.v0;
        s.Dr[t] = (T)bt.Dr;
        s.Dt[t] = (T)bt.Dt;
        s.mur[t] = (T)bt.mu_r;
        s.muth[t] = (T)bt.mu_theta;
        s.muab[t] = (T)bt.mu_ab;
        s.parent_drag[t] = bt.parent_drag;
        s.kmax[t] = bt.maxmode > 0 ? bt.maxmode - 1 : K;
    }
    set_noise_amplitudes(s);
    auto mask_of = [](const fcc_term& ft) {
        if (ft.ntypes_on == 0) return 0xffffffffu;
        uint32_t m = 0;
        for (int u = 0; u < ft.ntypes_on; ++u)
            if (ft.types_on[u] >= 1 && ft.types_on[u] <= FCC_MAX_TYPES) m |= 1u << (ft.types_on[u] - 1);
        return m;
    };
    // contact couplings summed over terms in the reference's order g1 + (g2 + ...)
    for (int r = 0; r < 2; ++r)
        for (int a = 0; a < MT; ++a)
            for (int c = 0; c < MT; ++c) s.cA[r][a][c] = T(0);
    for (int a = 0; a < MT; ++a) s.cB[a] = T(0);
    for (int q = p->nterms - 1; q >= 0; --q) {
        const fcc_term& ft = p->terms[q];
        const uint32_t mk = mask_of(ft);
        if (ft.kind == FCC_OVERLAP) {
            has_contact = true;
            for (int a = 0; a < MT; ++a) {
                if (!((mk >> a) & 1u)) continue;
                for (int c = 0; c < MT; ++c) {
                    const int ij = ft.nJ == 1 ? 0 : (a < ft.nJ && c < ft.nJ ? a + ft.nJ * c : -1);
                    if (ij < 0) continue;
                    s.cA[0][a][c] = (T)ft.J[ij] + s.cA[0][a][c];
                    s.cA[1][a][c] = (T)ft.Jrel[ij] + s.cA[1][a][c];
                }
            }
        } else if (ft.kind == FCC_LINEAR_REPULSION) {
            has_contact = true;
            for (int a = 0; a < MT; ++a)
                if ((mk >> a) & 1u) s.cB[a] = (T)ft.a + s.cB[a];
        }
    }
    s.nbt = 0;
    s.nbd = 0;
    s.nub = s.nuc = s.nubd = 0;
    for (int q = 0; q < p->nterms; ++q) {
        const fcc_term& ft = p->terms[q];
        if (ft.kind == FCC_USER_BODY) {
            const int u = s.nub++;
            s.ub_id[u] = ft.user;
            s.ub_mask[u] = mask_of(ft);
            s.ub_a[u] = (T)ft.a;
            s.ub_b[u] = (T)ft.b;
        } else if (ft.kind == FCC_USER_CONTACT) {
            const int u = s.nuc++;
            s.uc_id[u] = ft.user;
            s.uc_mask[u] = mask_of(ft);
            s.uc_a[u] = (T)ft.a;
            s.uc_b[u] = (T)ft.b;
            has_contact = true;
        } else if (ft.kind == FCC_USER_BOND) {
            const int u = s.nubd++;
            s.ubd_id[u] = ft.user;
            s.ubd_mask[u] = mask_of(ft);
            s.ubd_a[u] = (T)ft.a;
            s.ubd_b[u] = (T)ft.b;
        }
        if (ft.kind == FCC_TENSION || ft.kind == FCC_PERIMETER_ELASTICITY) {
            const int u = s.nbt++;
            s.bt_kind[u] = ft.kind == FCC_TENSION ? BT_TENSION : BT_PERIMETER;
            s.bt_mask[u] = mask_of(ft);
            s.bt_a[u] = (T)ft.a;
            // l0 = p0 * sqrt(π) * R0 (src/energies/body_terms.jl:34)
            s.bt_b[u] = ft.kind == FCC_TENSION ? T(0) : (T)ft.b * std::sqrt((T)PI);
        } else if (ft.kind == FCC_HARMONIC_BOND) {
            const int u = s.nbd++;
            s.bd_mask[u] = mask_of(ft);
            s.bd_k[u] = (T)ft.a;
            s.bd_r0[u] = (T)ft.b;
        }
    }
    s.has_contact = has_contact ? 1 : 0;
    s.has_noise = 0;
    for (int t = 0; t < p->ntypes; ++t)
        if (p->types[t].Dr != 0 || p->types[t].Dt != 0) s.has_noise = 1;
    split = false;
    for (int64_t i = 0; i < N; ++i)
        if (p->types[b->type[i] - 1].parent_drag) split = true;
    s.has_parent_drag = split ? 1 : 0;

    // children (src/bodies.jl:121-135) and bonds (src/energies/bonds.jl:52-71), local ids
    std::vector<int32_t>& type_h = sp.type;
    std::vector<int32_t>& parent_h = sp.parent;
    type_h.assign(b->type, b->type + N);
    parent_h.assign(b->parent, b->parent + N);
    std::vector<int>& chc = sp.chc;
    chc.assign(N, 0);
    for (int64_t k = 0; k < N; ++k)
        if (parent_h[k] != k + 1) chc[parent_h[k] - 1] += 1;
    int& ccap = sp.ccap;
    ccap = 1;
    for (int64_t k = 0; k < N; ++k) ccap = std::max(ccap, chc[k]);
    std::vector<int>& chi = sp.chi;
    chi.assign((size_t)ccap * N, 0);
    std::fill(chc.begin(), chc.end(), 0);
    for (int64_t k = 0; k < N; ++k) {
        const int pp = parent_h[k] - 1;
        if (pp == k) continue;
        chi[(size_t)pp * ccap + chc[pp]++] = (int)k;
    }
    std::vector<int>& bdc = sp.bdc;
    bdc.assign(N, 0);
    std::set<std::pair<int64_t, int64_t>> seen;
    for (int64_t q = 0; q < p->nbonds; ++q) {
        const int64_t i = p->bonds[2 * q], j = p->bonds[2 * q + 1];
        if (!(1 <= i && i <= N && 1 <= j && j <= N))
            return fail(FCC_ERR_ARGUMENT, "bond (" + std::to_string(i) + ", " + std::to_string(j) +
                                              ") refers to a body outside 1:" + std::to_string(N));
        if (i == j)
            return fail(FCC_ERR_ARGUMENT, "bond (" + std::to_string(i) + ", " + std::to_string(j) + ") connects a body to itself");
        auto key = std::make_pair(std::min(i, j), std::max(i, j));
        if (seen.count(key)) return fail(FCC_ERR_ARGUMENT, "duplicate bond (" + std::to_string(i) + ", " + std::to_string(j) + ")");
        seen.insert(key);
        bdc[i - 1] += 1;
        bdc[j - 1] += 1;
    }
    int& bcap = sp.bcap;
    bcap = 1;
    for (int64_t k = 0; k < N; ++k) bcap = std::max(bcap, bdc[k]);
    std::vector<int>& bdi = sp.bdi;
    bdi.assign((size_t)bcap * N, 0);
    std::fill(bdc.begin(), bdc.end(), 0);
    for (int64_t q = 0; q < p->nbonds; ++q) {
        const int64_t i = p->bonds[2 * q] - 1, j = p->bonds[2 * q + 1] - 1;
        bdi[(size_t)i * bcap + bdc[i]++] = (int)j;
        bdi[(size_t)j * bcap + bdc[j]++] = (int)i;
    }
    return FCC_OK;
}

// cos(n phi_k), sin(n phi_k), n cos(n phi_k), n sin(n phi_k) for the nodes
// phi_k = 2 pi k / nth and the modes n = 2..10, evaluated in double (the
// reference's FourierBasis rows, src/basis.jl:35-63) and rounded to T.
template <class T>
std::vector<T> mode_table(int nth) {
    std::vector<T> t((size_t)nth * KM * 4);
    for (int k = 0; k < nth; ++k)
        for (int m = 0; m < KM; ++m) {
            const double n = m + 2, a = n * k * (2 * PI / nth);
            T* e = t.data() + ((size_t)k * KM + m) * 4;
            e[0] = (T)std::cos(a);
            e[1] = (T)std::sin(a);
            e[2] = (T)(n * std::cos(a));
            e[3] = (T)(n * std::sin(a));
        }
    return t;
}

// Round a float to TF32 (10 mantissa bits), to nearest with ties away from
// zero: the rounding of cvt.rna.tf32.f32.
float tf32_round(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// Fragment table of the tensor-core contour contractions (the A operands of
// synth_mma and pullback_mma in fcc_kernels.cuh) for an nth-node contour:
// A[k][j] = 1, cos n phi_k, sin n phi_k for coefficient j in record order
// (a0, alpha_2, beta_2, ..., alpha_10, beta_10), phi_k = 2 pi k / nth
// (FourierBasis, src/basis.jl:35-63), zero beyond the contour and beyond
// the 19 coefficients.  Synthesis tiles (A, 48 x 24) then pullback tiles
// (A transposed, 32 x 40), each entry stored as a TF32 high part and the TF32
// rounding of the remainder, in the m16n8k8 A-fragment order: lane (g, t) =
// (lane / 4, lane % 4) holds rows g, g + 8, g, g + 8 and columns t, t, t + 4,
// t + 4 of the tile.
std::vector<float> mma_table(int nth) {
    auto basis = [&](int node, int j) -> double {
        if (node >= nth || j >= NCM) return 0.0;
        if (j == 0) return 1.0;
        const int m = (j - 1) / 2;
        const double a = (m + 2) * node * (2 * PI / nth);
        return (j & 1) ? std::cos(a) : std::sin(a);
    };
    std::vector<float> t((size_t)MMA_TABLE_FLOATS, 0.f);
    auto put = [&](int tile, int lane, int i, double v) {
        const float hi = tf32_round((float)v);
        const float lo = tf32_round((float)(v - (double)hi));
        t[((size_t)(tile * 2) * 32 + lane) * 4 + i] = hi;
        t[((size_t)(tile * 2 + 1) * 32 + lane) * 4 + i] = lo;
    };
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane / 4, tq = lane % 4;
        const int rows[4] = {g, g + 8, g, g + 8}, cols[4] = {tq, tq, tq + 4, tq + 4};
        for (int i = 0; i < 4; ++i) {
            for (int mt = 0; mt < 3; ++mt)
                for (int kt = 0; kt < 3; ++kt)  // synthesis: rows nodes, columns coefficients
                    put(mt * 3 + kt, lane, i, basis(16 * mt + rows[i], 8 * kt + cols[i]));
            for (int mt = 0; mt < 2; ++mt)
                for (int kt = 0; kt < 5; ++kt)  // pullback: rows coefficients, columns nodes
                    put(MMA_SYN_TILES + mt * 5 + kt, lane, i, basis(8 * kt + cols[i], 16 * mt + rows[i]));
        }
    }
    return t;
}

struct EngineBase {
    virtual ~EngineBase() = default;
    virtual fcc_status step(int64_t n, bool eager) = 0;
    virtual fcc_status run(fcc_sim* h, int64_t n, int64_t every, fcc_callback cb, void* user, bool graph) = 0;
    virtual fcc_status update_neighbors(bool force) = 0;
    virtual fcc_status compute_gradients() = 0;
    virtual fcc_status get_state(fcc_bodies_host* out, int64_t* clock, double* t, int64_t* stp) = 0;
    virtual fcc_status set_state(const fcc_bodies_host* in, int64_t clock) = 0;
    virtual fcc_status set_dt(double dt) = 0;
    virtual fcc_status get_gradients(const fcc_gradients_host* out) = 0;
    virtual fcc_status get_geometry(const fcc_geometry_host* out) = 0;
    virtual fcc_status neighbor_dims(int32_t*, int32_t*, int32_t*, int64_t*, int32_t*) = 0;
    virtual fcc_status get_neighbors(const fcc_neighbors_host* out) = 0;
    virtual fcc_status observable(int which, int32_t type, double* out, int64_t* count) = 0;
    virtual fcc_status body_energy(double* out) = 0;
    virtual fcc_status timing(double* ms, int64_t* launches, int64_t* steps) = 0;
    virtual fcc_status health(int32_t* nonfinite, int32_t* barrier_error) = 0;
};

template <class T>
struct Engine final : EngineBase {
    int device = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // configuration
    int64_t N = 0;
    int K = 0, nc = 0, nth = 0, cap = 32, ncx = 1, ncy = 1;
    bool has_contact = false, split = false;
    SimDesc<T> desc{};
    std::vector<int32_t> type_h, parent_h;
    std::vector<T> R0_h;
    // host mirror of run state
    long long clock_h = 0;
    long long gstep = 0;  // engine step counter: the current record buffer is rec[gstep & 1]
    T t_h = T(0);
    int64_t step_h = 0;
    int64_t builds_adjust = 0;
    double last_ms = 0;
    int64_t last_launches = 0, last_steps = 0;
    int step_grid = 0;
    // device buffers
    DBuf<SimDesc<T>> sims;
    DBuf<T> rec0, rec1, coef, R0, x0, y0, rmax0, cs, basis, gx, gy, gth, glab, E, P, GR, GD, GDD, gcoef;
    DBuf<float> mtab;  // FP32: tensor-core fragment table
    DBuf<int> imgx, imgy, sim_of, nb_idx, nb_count, cellid, slot, perm, cstart, cstop, ccount, cell_sim, ch_idx,
        ch_count, bd_idx, bd_count;
    // run state of the simulation, one device block so that one copy reads it
    // back (read_status) and one copy writes its head (load_state); builds
    // last, out of the written head
    struct Status {
        int flags, maxcount;
        long long clock;
        GridSync sync;
        long long builds;
    };
    DBuf<Status> dstat;
    int* flags_d = nullptr;
    int* maxcount_d = nullptr;
    long long* clock_d = nullptr;
    long long* builds_d = nullptr;
    GridSync* sync_d = nullptr;
    ObsArea obs;  // perimeters / areas / shape indices: reused device and pinned host buffers
    int ccap = 1, bcap = 1;
    Status* st_h = nullptr;  // pinned read-back of the run state
    Status* up_h = nullptr;  // pinned head written by load_state
    // state exchange with the host (set_state / get_state): the caller's
    // double arrays are copied as they are into one device area (x, y, theta,
    // coefficients in the reference's layout), and converted and repacked on
    // the device; allocated at create and reused, so no exchange allocates.
    // w_dev holds the (parent, type) record words, fixed since create.
    DBuf<double> xch_d;
    DBuf<int> w_dev;

    ~Engine() override {
        if (stream) cudaStreamSynchronize(stream);
        if (st_h) cudaFreeHost(st_h);
        if (up_h) cudaFreeHost(up_h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    DevPtrs<T> ptrs() const {
        DevPtrs<T> d{};
        d.sims = sims.p;
        d.nsims = 1;
        d.Ntot = (int)N;
        d.Ctot = ncx * ncy;
        d.nth = nth;
        d.cap = cap;
        d.sim_of = sim_of.p;
        d.rec0 = rec0.p;
        d.rec1 = rec1.p;
        d.coef = coef.p;
        d.imgx = imgx.p;
        d.imgy = imgy.p;
        d.R0 = R0.p;
        d.x0 = x0.p;
        d.y0 = y0.p;
        d.rmax0 = rmax0.p;
        d.nb_idx = nb_idx.p;
        d.nb_count = nb_count.p;
        d.cellid = cellid.p;
        d.slot = slot.p;
        d.perm = perm.p;
        d.cstart = cstart.p;
        d.cstop = cstop.p;
        d.ccount = ccount.p;
        d.cell_sim = cell_sim.p;
        d.ccap = ccap;
        d.ch_idx = ch_idx.p;
        d.ch_count = ch_count.p;
        d.bcap = bcap;
        d.bd_idx = bd_idx.p;
        d.bd_count = bd_count.p;
        d.flags = flags_d;
        d.clock = clock_d;
        d.builds = builds_d;
        d.maxcount = maxcount_d;
        d.sync = sync_d;
        d.cs = cs.p;
        d.basis = basis.p;
        d.mtab = mtab.p;
        d.gx = gx.p;
        d.gy = gy.p;
        d.gth = gth.p;
        d.glab = glab.p;
        d.E = E.p;
        d.P = P.p;
        d.GR = GR.p;
        d.GD = GD.p;
        d.GDD = GDD.p;
        d.gcoef = gcoef.p;
        return d;
    }

    // ------------------------------------------------------------ set-up --
    fcc_status init(const fcc_params* p, const fcc_bodies_host* b) {
        SimSpec<T> sp;
        FCC_TRY(make_spec(p, b, sp));
        // device and stream
        CUDA_TRY(cudaGetDevice(&device));
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        int coop = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        if (!coop) return fail(FCC_ERR_UNSUPPORTED, "device lacks cooperative launch");
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreate(&ev0));
        CUDA_TRY(cudaEventCreate(&ev1));
        CUDA_TRY(cudaMallocHost(&st_h, sizeof(Status)));
        CUDA_TRY(cudaMallocHost(&up_h, sizeof(Status)));

        N = sp.N;
        K = sp.K;
        nc = sp.nc;
        nth = sp.nth;
        ncx = sp.ncx;
        ncy = sp.ncy;
        has_contact = sp.has_contact;
        split = sp.split;
        desc = sp.desc;
        user = desc.nub + desc.nuc + desc.nubd > 0;
        type_h = std::move(sp.type);
        parent_h = std::move(sp.parent);
        R0_h = std::move(sp.R0);
        ccap = sp.ccap;
        bcap = sp.bcap;
        const std::vector<int>& chi = sp.chi;
        const std::vector<int>& chc = sp.chc;
        const std::vector<int>& bdi = sp.bdi;
        const std::vector<int>& bdc = sp.bdc;

        // device buffers
        cap = p->nl_capacity > 0 ? p->nl_capacity : 32;
        const size_t n = (size_t)N;
        FCC_TRY(sims.upload(std::vector<SimDesc<T>>{desc}, stream));
        FCC_TRY(rec0.alloc(n * RECW, stream));
        FCC_TRY(rec1.alloc(n * RECW, stream));
        FCC_TRY(coef.alloc(n * NCM, stream));
        FCC_TRY(R0.upload(R0_h, stream));
        FCC_TRY(x0.alloc(n, stream));
        FCC_TRY(y0.alloc(n, stream));
        FCC_TRY(rmax0.alloc(n, stream));
        FCC_TRY(gx.alloc(n, stream));
        FCC_TRY(gy.alloc(n, stream));
        FCC_TRY(gth.alloc(n, stream));
        FCC_TRY(E.alloc(n, stream));
        FCC_TRY(glab.alloc(n * NCM, stream));
        std::vector<T> csh(2 * (size_t)nth);
        for (int k = 0; k < nth; ++k) {  // FourierBasis.cs, src/basis.jl:50-52
            const double phi = k * (2 * PI / nth);
            csh[2 * k] = (T)std::cos(phi);
            csh[2 * k + 1] = (T)std::sin(phi);
        }
        FCC_TRY(cs.upload(csh, stream));
        FCC_TRY(basis.upload(mode_table<T>(nth), stream));
        if (sizeof(T) == 4 && nth <= BASIS_NODES) FCC_TRY(mtab.upload(mma_table(nth), stream));
        FCC_TRY(imgx.upload(std::vector<int>(b->imgx, b->imgx + N), stream));
        FCC_TRY(imgy.upload(std::vector<int>(b->imgy, b->imgy + N), stream));
        FCC_TRY(sim_of.alloc(n, stream));
        FCC_TRY(nb_idx.alloc(n * cap, stream));
        FCC_TRY(nb_count.alloc(n, stream));
        FCC_TRY(cellid.alloc(n, stream));
        FCC_TRY(slot.alloc(n, stream));
        FCC_TRY(perm.alloc(n, stream));
        FCC_TRY(cstart.alloc((size_t)ncx * ncy, stream));
        FCC_TRY(cstop.alloc((size_t)ncx * ncy, stream));
        FCC_TRY(ccount.alloc((size_t)ncx * ncy, stream));
        FCC_TRY(cell_sim.alloc((size_t)ncx * ncy, stream));
        FCC_TRY(ch_idx.upload(chi, stream));
        FCC_TRY(ch_count.upload(chc, stream));
        FCC_TRY(bd_idx.upload(bdi, stream));
        FCC_TRY(bd_count.upload(bdc, stream));
        FCC_TRY(dstat.alloc(1, stream));  // zeroed; load_state below writes the head
        flags_d = &dstat.p->flags;
        maxcount_d = &dstat.p->maxcount;
        clock_d = &dstat.p->clock;
        builds_d = &dstat.p->builds;
        sync_d = &dstat.p->sync;

        std::vector<int> w(n);
        for (size_t i = 0; i < n; ++i) w[i] = ((parent_h[i] - 1) << 3) | (type_h[i] - 1);
        FCC_TRY(w_dev.upload(w, stream));
        FCC_TRY(xch_d.alloc(n * (3 + (size_t)nc), stream));

        // launch configuration of the persistent kernel: all co-resident blocks
        FCC_TRY(configure());
        FCC_TRY(load_state(b, 0));
        return sync_stream();
    }

    int variant = 0;
    const Variant& var() const { return VARIANTS[variant]; }
    static constexpr size_t grad_stage_bytes() {
        return basis_table_bytes<T>() + (size_t)(256 / 32) * stage_bytes_per_warp<T, LANES>();
    }
    size_t stage_bytes() const {
        return basis_table_bytes<T>() + (size_t)(var().blk / 32) * (sizeof(T) == 4 ? var().stage32 : var().stage64);
    }
    // compiled user terms: the 8 x 5 / 256-thread kernels with the user-term code
    bool user = false;
    bool owners_set = false;  // sim_of and cell_sim written (by the first load_state)
    void* step_kernel() const {
        if (user)
            return split ? (void*)k_step<T, 8, 5, true, true, 256, (sizeof(T) == 4 ? 2 : 1), true>
                         : (void*)k_step<T, 8, 5, true, false, 256, (sizeof(T) == 4 ? 2 : 1), true>;
        return (sizeof(T) == 4 ? var().f32 : var().f64)(one_chunk(), split);
    }
    void* grad_kernel() const {
        if (user) return (void*)k_gradients<T, LANES, SLOTS, true, true>;
        return nth <= LANES * SLOTS ? (void*)k_gradients<T, LANES, SLOTS, true> : (void*)k_gradients<T, LANES, SLOTS, false>;
    }

    bool one_chunk() const { return nth <= var().L * var().S; }

    // Variant choice.  FCC_VARIANT overrides (FP64: only variants with an FP64
    // build).  Otherwise a one-chunk step without parent drag compares the
    // launch shapes of the default family (bit-identical results, FP32 and
    // FP64) by the rounds of warp groups a step takes at this N, weighted by
    // the measured time of one round.  224-thread blocks (14 warps per SM in
    // FP32, 7 in FP64) run a round in about 0.97 (FP32) or 0.945 (FP64) of the
    // time of 256-thread blocks but hold 12.5% fewer warps.  FP32 takes its
    // groups dynamically, so a step costs whole rounds: 224 wins where the
    // 256-thread grid leaves its last round part-empty (N = 1024: 9.57 vs
    // 10.03 µs; N = 16384: 23.44 vs 23.45 µs, 61.4 vs 65.4 µs with a rebuild
    // every step) and loses where both fill it (N = 65536: 88.1 vs 78.6 µs).
    // FP64 splits them statically, so a step costs the mean rounds per warp
    // (at least one): 224 wins only while one round holds all groups (N =
    // 1024: 16.4 vs 16.6 µs; N = 16384: 63.1 vs 60.3 µs).  (Deformed states
    // after 300 warm-up steps, flat step barrier.)
    fcc_status choose_variant() {
        variant = 0;
        if (user) {  // one kernel family carries the user-term code
            if (!one_chunk()) return fail(FCC_ERR_UNSUPPORTED, "user terms need ntheta <= 40 (one contour chunk)");
            return FCC_OK;
        }
        if (const char* e = std::getenv("FCC_VARIANT")) {
            const int v = std::atoi(e);
            if (v >= 0 && v < NVARIANTS && (sizeof(T) == 4 || VARIANTS[v].f64)) variant = v;
            return FCC_OK;
        }
        if (N <= 0 || !one_chunk() || split) return FCC_OK;
        struct Candidate {
            int v;
            double round_time;
        };
        const Candidate cands[] = {{0, 1.0}, {5, sizeof(T) == 4 ? 0.97 : 0.945}};
        double best = 1e300;
        int pick = 0;
        for (const Candidate& c : cands) {
            variant = c.v;
            const int smem = (int)stage_bytes();
            CUDA_TRY(cudaFuncSetAttribute(step_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            int per_sm = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel(), var().blk, smem));
            if (per_sm < 1) continue;
            const int64_t bpw = 32 / var().L, wpb = var().blk / 32;
            const int64_t groups = (N + bpw - 1) / bpw;
            const int64_t blocks = std::min<int64_t>((groups + wpb - 1) / wpb, (int64_t)per_sm * nsm);
            const double rounds = sizeof(T) == 4 ? (double)((groups + blocks * wpb - 1) / (blocks * wpb))
                                                 : std::max(1.0, (double)groups / (double)(blocks * wpb));
            const double cost = rounds * c.round_time;
            if (cost < best) {
                best = cost;
                pick = c.v;
            }
        }
        variant = pick;
        return FCC_OK;
    }

    fcc_status configure() {
        FCC_TRY(choose_variant());
        const int smem = (int)stage_bytes();
        CUDA_TRY(cudaFuncSetAttribute(step_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CUDA_TRY(cudaFuncSetAttribute(grad_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_stage_bytes()));
        int per_sm = 0;
        const int blk = var().blk;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel(), blk, smem));
        if (per_sm < 1) return fail(FCC_ERR_UNSUPPORTED, "step kernel does not fit on an SM");
        const int maxblocks = per_sm * nsm;
        const int bpw = 32 / var().L;
        const int64_t groups = (N + bpw - 1) / bpw;
        const int64_t want = std::max<int64_t>(1, (groups + blk / 32 - 1) / (blk / 32));
        step_grid = (int)std::min<int64_t>(want, maxblocks);
        return FCC_OK;
    }

    // Copy a host body state in and rebuild the derived geometry (k_init),
    // which rounds the caller's doubles to T and repacks the coefficients on
    // the device.  Page-locked host arrays are read by k_init in place (one
    // launch, no copy call); other arrays go to the device as they are, one
    // copy each (the driver stages pageable memory).  The call returns once
    // the inputs are no longer needed: the caller may reuse its buffers.
    fcc_status load_state(const fcc_bodies_host* b, int64_t clk) {
        const size_t n = (size_t)N;
        if (clk >= 0) clock_h = clk;
        const double *px = nullptr, *py = nullptr, *pth = nullptr, *pc = nullptr;
        const int *pix = nullptr, *piy = nullptr;
        if (n) {
            px = mapped_view(b->x);
            py = mapped_view(b->y);
            pth = mapped_view(b->theta);
            pc = mapped_view(b->coef);
            pix = mapped_view(b->imgx);
            piy = mapped_view(b->imgy);
            const bool in_place = px && py && pth && pc && (!b->imgx || pix) && (!b->imgy || piy);
            if (!in_place) {
                double* dx = xch_d.p;
                px = dx;
                py = dx + n;
                pth = dx + 2 * n;
                pc = dx + 3 * n;
                pix = piy = nullptr;
                CUDA_TRY(cudaMemcpyAsync(dx, b->x, n * sizeof(double), cudaMemcpyHostToDevice, stream));
                CUDA_TRY(cudaMemcpyAsync(dx + n, b->y, n * sizeof(double), cudaMemcpyHostToDevice, stream));
                CUDA_TRY(cudaMemcpyAsync(dx + 2 * n, b->theta, n * sizeof(double), cudaMemcpyHostToDevice, stream));
                CUDA_TRY(cudaMemcpyAsync(dx + 3 * n, b->coef, n * nc * sizeof(double), cudaMemcpyHostToDevice, stream));
                if (b->imgx) CUDA_TRY(cudaMemcpyAsync(imgx.p, b->imgx, n * sizeof(int), cudaMemcpyHostToDevice, stream));
                if (b->imgy) CUDA_TRY(cudaMemcpyAsync(imgy.p, b->imgy, n * sizeof(int), cudaMemcpyHostToDevice, stream));
            }
        }
        if (!owners_set) {  // every body and cell belongs to simulation 0; set once, at create
            if (n) CUDA_TRY(cudaMemsetAsync(sim_of.p, 0, n * sizeof(int), stream));
            CUDA_TRY(cudaMemsetAsync(cell_sim.p, 0, (size_t)ncx * ncy * sizeof(int), stream));
            owners_set = true;
        }
        const DevPtrs<T> d = ptrs();
        if (N > 0) {
            const int grid = (int)((N + INIT_BLOCK - 1) / INIT_BLOCK);
            k_init<T><<<grid, INIT_BLOCK, init_smem_bytes(nc), stream>>>(d, par(), 0, (int)N, px, py, pth, pc, nc, K,
                                                                        w_dev.p, pix, piy);
            CUDA_TRY(cudaGetLastError());
        }
        // clock, and the list invalid: the next step (or update_neighbors!)
        // rebuilds; one copy of the status head from pinned memory
        up_h->flags = F_ACTIVE | (has_contact ? (F_CONTACT | F_NEED) : 0);
        up_h->maxcount = 0;
        up_h->clock = clock_h;
        up_h->sync = GridSync{0, 0, 0, has_contact ? 1 : 0, 0};
        CUDA_TRY(cudaMemcpyAsync(dstat.p, up_h, offsetof(Status, builds), cudaMemcpyHostToDevice, stream));
        return sync_stream();  // the caller's arrays (and up_h) are free for reuse on return
    }

    int par() const { return (int)(gstep & 1); }

    fcc_status sync_stream() {
        CUDA_TRY(cudaStreamSynchronize(stream));
        return FCC_OK;
    }

    fcc_status read_status() {
        CUDA_TRY(cudaMemcpyAsync(st_h, dstat.p, sizeof(Status), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (st_h->sync.error) return fail(FCC_ERR_DEVICE, "a grid barrier wait timed out in the step kernel");
        return FCC_OK;
    }

    // Account executed steps (t accumulates in T, as sim.t += sim.dt does).
    void account(long long newclock) {
        const long long executed = newclock - clock_h;
        for (long long q = 0; q < executed; ++q) t_h += desc.dt;
        step_h += executed;
        clock_h = newclock;
    }

    // Neighbour-list overflow: grow the capacity to twice the largest count
    // (src/neighbors.jl:226-233) and rebuild at the next step.
    fcc_status regrow() {
        const int newcap = std::max(2 * st_h->maxcount, cap + 1);
        FCC_TRY(nb_idx.alloc((size_t)N * newcap, stream));
        cap = newcap;
        builds_adjust -= 1;  // the overflowed build is repeated
        const int f = (st_h->flags & ~(F_FROZEN | F_VALID | F_REBUILD)) | F_NEED;
        CUDA_TRY(cudaMemcpyAsync(flags_d, &f, sizeof(int), cudaMemcpyHostToDevice, stream));
        const int one = 1;
        CUDA_TRY(cudaMemcpyAsync(&sync_d->any_need, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
        return sync_stream();
    }

    fcc_status launch_steps(int nsteps) {
        DevPtrs<T> d = ptrs();
        int p0 = par();
        void* args[] = {&d, &nsteps, &p0};
        CUDA_TRY(cudaLaunchCooperativeKernel(step_kernel(), dim3(step_grid), dim3(var().blk), args, stage_bytes(), stream));
        gstep += nsteps;
        ++last_launches;
        return FCC_OK;
    }

    // Run n steps as launches of `per` steps each.  A neighbour-list overflow
    // freezes the simulation on the device (the remaining launched steps do
    // nothing); the host then regrows the list and launches the missing steps.
    fcc_status advance(int64_t n, int per) {
        Range range("fcc advance");
        int64_t done = 0;
        while (done < n) {
            const long long start = clock_h;
            const int64_t requested = n - done;
            for (int64_t remaining = requested; remaining > 0;) {
                const int k = (int)std::min<int64_t>(per, remaining);
                FCC_TRY(launch_steps(k));
                remaining -= k;
            }
            FCC_TRY(read_status());
            account(st_h->clock);
            const int64_t executed = st_h->clock - start;
            done += executed;
            if (st_h->flags & F_FROZEN) FCC_TRY(regrow());
            else if (executed < requested) return fail(FCC_ERR_DEVICE, "step kernel did not advance the clock");
        }
        return FCC_OK;
    }

    fcc_status step(int64_t n, bool eager) override {
        if (n <= 0 || N == 0) {
            if (n > 0) {  // no bodies: only the clock and time advance
                for (int64_t q = 0; q < n; ++q) t_h += desc.dt;
                step_h += n;
                clock_h += n;
                CUDA_TRY(cudaMemcpyAsync(clock_d, &clock_h, sizeof(long long), cudaMemcpyHostToDevice, stream));
                return sync_stream();
            }
            return FCC_OK;
        }
        last_launches = 0;
        const long long c0 = clock_h;
        CUDA_TRY(cudaEventRecord(ev0, stream));
        FCC_TRY(advance(n, eager ? 1 : 512));
        CUDA_TRY(cudaEventRecord(ev1, stream));
        CUDA_TRY(cudaEventSynchronize(ev1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        last_steps = clock_h - c0;
        return FCC_OK;
    }

    fcc_status run(fcc_sim* h, int64_t n, int64_t every, fcc_callback cb, void* user, bool graph) override {
        if (!cb || every <= 0) return step(n, !graph);
        int64_t done = 0;
        while (done < n) {
            const int64_t k = std::min(every, n - done);
            FCC_TRY(step(k, !graph));
            done += k;
            cb(h, user);
        }
        return FCC_OK;
    }

    fcc_status update_neighbors(bool force) override {
        Range range("fcc update_neighbors");
        if (!has_contact || N == 0) return FCC_OK;
        const DevPtrs<T> d = ptrs();
        const int grid = (int)((N + 255) / 256);
        for (int attempt = 0; attempt < 8; ++attempt) {
            DevPtrs<T> dd = ptrs();
            if (!force && attempt == 0) {
                k_skin_check<T><<<grid, 256, 0, stream>>>(dd, par());
                CUDA_TRY(cudaGetLastError());
            }
            k_prepare_rebuild<T><<<1, 256, 0, stream>>>(dd, (force || attempt > 0) ? 1 : 0);
            k_phase_count<T><<<grid, 256, 0, stream>>>(dd, par());
            k_phase_scan<T><<<1, 1024, 0, stream>>>(dd);
            k_phase_scatter<T><<<grid, 256, 0, stream>>>(dd);
            k_phase_sort<T><<<(ncx * ncy + 255) / 256, 256, 0, stream>>>(dd);
            k_phase_neighbors<T><<<neighbor_grid(N), 256, 0, stream>>>(dd, par());
            k_finish_rebuild<T><<<1, 256, 0, stream>>>(dd);
            CUDA_TRY(cudaGetLastError());
            FCC_TRY(read_status());
            if (!(st_h->flags & F_FROZEN)) return FCC_OK;
            FCC_TRY(regrow());
        }
        (void)d;
        return fail(FCC_ERR_DEVICE, "neighbour list did not fit after regrowth");
    }

    fcc_status ensure_diag() {
        if (P.p) return FCC_OK;
        const size_t n = (size_t)N * nth;
        FCC_TRY(P.alloc(n, stream));
        FCC_TRY(GR.alloc(n, stream));
        FCC_TRY(GD.alloc(n, stream));
        FCC_TRY(GDD.alloc(n, stream));
        FCC_TRY(gcoef.alloc((size_t)N * NCM, stream));
        return FCC_OK;
    }

    fcc_status compute_gradients() override {
        Range range("fcc compute_gradients");
        if (N == 0) return FCC_OK;
        FCC_TRY(ensure_diag());
        const DevPtrs<T> d = ptrs();
        const int64_t groups = (N + (32 / LANES) - 1) / (32 / LANES);
        const int grid = (int)((groups + 256 / 32 - 1) / (256 / 32));
        if (user)
            k_gradients<T, LANES, SLOTS, true, true><<<grid, 256, grad_stage_bytes(), stream>>>(d, par());
        else if (nth <= LANES * SLOTS)
            k_gradients<T, LANES, SLOTS, true><<<grid, 256, grad_stage_bytes(), stream>>>(d, par());
        else
            k_gradients<T, LANES, SLOTS, false><<<grid, 256, grad_stage_bytes(), stream>>>(d, par());
        CUDA_TRY(cudaGetLastError());
        return sync_stream();
    }

    // engine coefficient layout [a0; a_2..a_10; b_2..b_10] -> reference rows [a0; a_2..a_M; b_2..b_M]
    void coef_out(const T* src, double* dst) const {
        for (int64_t i = 0; i < N; ++i) {
            dst[(size_t)i * nc] = (double)src[(size_t)i * NCM];
            for (int m = 0; m < K; ++m) {
                dst[(size_t)i * nc + 1 + m] = (double)src[(size_t)i * NCM + 1 + m];
                dst[(size_t)i * nc + 1 + K + m] = (double)src[(size_t)i * NCM + 1 + KM + m];
            }
        }
    }

    template <class V>
    fcc_status fetch(const V* src, size_t n, std::vector<V>& out) {
        out.resize(n);
        if (n) CUDA_TRY(cudaMemcpyAsync(out.data(), src, n * sizeof(V), cudaMemcpyDeviceToHost, stream));
        return FCC_OK;
    }

    // sim.bodies: k_store_host widens x, y, theta and the coefficients to
    // double in the reference's layout on the device and writes them, with
    // the image counters, into the caller's page-locked arrays in place (one
    // launch), or into the exchange area for one copy per array into other
    // memory.  R0, type and parent are fixed since create and come from the
    // host mirror.
    fcc_status get_state(fcc_bodies_host* o, int64_t* clk, double* t, int64_t* stp) override {
        if (o) {
            if (o->n != N || o->ncoef != nc) return fail(FCC_ERR_DIMENSION, "state buffers do not match the simulation");
            const size_t n = (size_t)N;
            if (n) {
                double *vx = mapped_view(o->x), *vy = mapped_view(o->y), *vth = mapped_view(o->theta),
                       *vc = mapped_view(o->coef);
                int *vix = mapped_view(o->imgx), *viy = mapped_view(o->imgy);
                const bool in_place = (!o->x || vx) && (!o->y || vy) && (!o->theta || vth) && (!o->coef || vc) &&
                                      (!o->imgx || vix) && (!o->imgy || viy);
                const int grid = (int)std::min<int64_t>((N * nc + 255) / 256, (int64_t)nsm * 8);
                if (in_place) {
                    k_store_host<T><<<grid, 256, 0, stream>>>(ptrs(), par(), 0, (int)N, vx, vy, vth, vc, nc, K, vix, viy);
                    CUDA_TRY(cudaGetLastError());
                } else {
                    double* dx = xch_d.p;
                    k_store_host<T><<<grid, 256, 0, stream>>>(ptrs(), par(), 0, (int)N, dx, dx + n, dx + 2 * n, dx + 3 * n,
                                                              nc, K, nullptr, nullptr);
                    CUDA_TRY(cudaGetLastError());
                    if (o->x) CUDA_TRY(cudaMemcpyAsync(o->x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                    if (o->y) CUDA_TRY(cudaMemcpyAsync(o->y, dx + n, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                    if (o->theta)
                        CUDA_TRY(cudaMemcpyAsync(o->theta, dx + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
                    if (o->coef)
                        CUDA_TRY(cudaMemcpyAsync(o->coef, dx + 3 * n, n * nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
                    if (o->imgx) CUDA_TRY(cudaMemcpyAsync(o->imgx, imgx.p, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
                    if (o->imgy) CUDA_TRY(cudaMemcpyAsync(o->imgy, imgy.p, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
                }
            }
            // the fixed fields while the device works
            for (size_t i = 0; i < n; ++i) {
                if (o->R0) o->R0[i] = (double)R0_h[i];
                if (o->type) o->type[i] = type_h[i];
                if (o->parent) o->parent[i] = parent_h[i];
            }
            FCC_TRY(sync_stream());
        }
        if (clk) *clk = clock_h;
        if (t) *t = (double)t_h;
        if (stp) *stp = step_h;
        return FCC_OK;
    }

    fcc_status set_state(const fcc_bodies_host* in, int64_t clk) override {
        if (!in || in->n != N || in->ncoef != nc) return fail(FCC_ERR_DIMENSION, "state buffers do not match the simulation");
        if (!in->x || !in->y || !in->theta || !in->coef) return fail(FCC_ERR_ARGUMENT, "set_state needs x, y, theta and coef");
        return load_state(in, clk);
    }

    fcc_status set_dt(double dt) override {
        desc.dt = (T)dt;
        set_noise_amplitudes(desc);
        CUDA_TRY(cudaMemcpyAsync(sims.p, &desc, sizeof(SimDesc<T>), cudaMemcpyHostToDevice, stream));
        return sync_stream();
    }

    fcc_status get_gradients(const fcc_gradients_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        if (!P.p) FCC_TRY(ensure_diag());
        const size_t n = (size_t)N;
        std::vector<T> a;
        auto copy_nodes = [&](DBuf<T>& src, double* dst) -> fcc_status {
            if (!dst) return FCC_OK;
            FCC_TRY(fetch(src.p, n * nth, a));
            FCC_TRY(sync_stream());
            for (size_t q = 0; q < n * nth; ++q) dst[q] = (double)a[q];
            return FCC_OK;
        };
        auto copy_vec = [&](DBuf<T>& src, double* dst) -> fcc_status {
            if (!dst) return FCC_OK;
            FCC_TRY(fetch(src.p, n, a));
            FCC_TRY(sync_stream());
            for (size_t q = 0; q < n; ++q) dst[q] = (double)a[q];
            return FCC_OK;
        };
        auto copy_coef = [&](DBuf<T>& src, double* dst) -> fcc_status {
            if (!dst) return FCC_OK;
            FCC_TRY(fetch(src.p, n * NCM, a));
            FCC_TRY(sync_stream());
            coef_out(a.data(), dst);
            return FCC_OK;
        };
        FCC_TRY(copy_nodes(GR, o->GR));
        FCC_TRY(copy_nodes(GD, o->GD));
        FCC_TRY(copy_nodes(GDD, o->GDD));
        FCC_TRY(copy_nodes(P, o->P));
        FCC_TRY(copy_vec(gx, o->gx));
        FCC_TRY(copy_vec(gy, o->gy));
        FCC_TRY(copy_vec(gth, o->gtheta));
        FCC_TRY(copy_coef(glab, o->glab));
        FCC_TRY(copy_coef(gcoef, o->gcoef));
        FCC_TRY(copy_vec(E, o->Ebody));
        return FCC_OK;
    }

    fcc_status get_geometry(const fcc_geometry_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        if (N == 0) return FCC_OK;
        const size_t n = (size_t)N;
        DBuf<T> lab, labR0, R, dR, ddR, rmax;
        FCC_TRY(lab.alloc(n * NCM, stream));
        FCC_TRY(labR0.alloc(n * NCM, stream));
        FCC_TRY(R.alloc(n * nth, stream));
        FCC_TRY(dR.alloc(n * nth, stream));
        FCC_TRY(ddR.alloc(n * nth, stream));
        FCC_TRY(rmax.alloc(n, stream));
        k_geometry<T><<<(int)((N + 127) / 128), 128, 0, stream>>>(ptrs(), par(), lab.p, labR0.p, R.p, dR.p, ddR.p, rmax.p);
        CUDA_TRY(cudaGetLastError());
        std::vector<T> a;
        auto nodes = [&](DBuf<T>& src, double* dst) -> fcc_status {
            if (!dst) return FCC_OK;
            FCC_TRY(fetch(src.p, n * nth, a));
            FCC_TRY(sync_stream());
            for (size_t q = 0; q < n * nth; ++q) dst[q] = (double)a[q];
            return FCC_OK;
        };
        auto coefs = [&](DBuf<T>& src, double* dst) -> fcc_status {
            if (!dst) return FCC_OK;
            FCC_TRY(fetch(src.p, n * NCM, a));
            FCC_TRY(sync_stream());
            coef_out(a.data(), dst);
            return FCC_OK;
        };
        FCC_TRY(coefs(lab, o->lab));
        FCC_TRY(coefs(labR0, o->labR0));
        FCC_TRY(nodes(R, o->R));
        FCC_TRY(nodes(dR, o->dR));
        FCC_TRY(nodes(ddR, o->ddR));
        if (o->rmax) {
            FCC_TRY(fetch(rmax.p, n, a));
            FCC_TRY(sync_stream());
            for (size_t q = 0; q < n; ++q) o->rmax[q] = (double)a[q];
        }
        return sync_stream();
    }

    fcc_status neighbor_dims(int32_t* cx, int32_t* cy, int32_t* cp, int64_t* b, int32_t* v) override {
        FCC_TRY(read_status());
        if (cx) *cx = ncx;
        if (cy) *cy = ncy;
        if (cp) *cp = cap;
        if (b) *b = st_h->builds + builds_adjust;
        if (v) *v = (st_h->flags & F_VALID) ? 1 : 0;
        return FCC_OK;
    }

    fcc_status get_neighbors(const fcc_neighbors_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        const size_t n = (size_t)N, nce = (size_t)ncx * ncy;
        std::vector<int> a, b2;
        if (o->cellid) {
            FCC_TRY(fetch(cellid.p, n, a));
            FCC_TRY(sync_stream());
            for (size_t i = 0; i < n; ++i) o->cellid[i] = a[i] + 1;
        }
        if (o->perm) {
            FCC_TRY(fetch(perm.p, n, a));
            FCC_TRY(sync_stream());
            for (size_t i = 0; i < n; ++i) o->perm[i] = a[i] + 1;
        }
        if (o->start || o->stop) {
            FCC_TRY(fetch(cstart.p, nce, a));
            FCC_TRY(fetch(cstop.p, nce, b2));
            FCC_TRY(sync_stream());
            for (size_t c = 0; c < nce; ++c) {
                const bool empty = b2[c] <= a[c];
                if (o->start) o->start[c] = empty ? 1 : a[c] + 1;
                if (o->stop) o->stop[c] = empty ? 0 : b2[c];
            }
        }
        std::vector<int> cnt;
        FCC_TRY(fetch(nb_count.p, n, cnt));
        FCC_TRY(sync_stream());
        if (o->count) std::copy(cnt.begin(), cnt.end(), o->count);
        if (o->idx) {
            FCC_TRY(fetch(nb_idx.p, n * cap, a));
            FCC_TRY(sync_stream());
            for (size_t i = 0; i < n; ++i)
                for (int q = 0; q < cap; ++q) o->idx[i * cap + q] = q < cnt[i] ? a[i * cap + q] + 1 : 0;
        }
        return FCC_OK;
    }

    fcc_status observable(int which, int32_t typ, double* out, int64_t* count) override {
        const double* v = nullptr;
        if (N > 0) {
            FCC_TRY(obs.reserve(3 * (size_t)N, stream));
            k_observables<T><<<(int)((N + 127) / 128), 128, 0, stream>>>(ptrs(), par(), 0, (int)N, obs.dev.p);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaMemcpyAsync(obs.host, obs.dev.p, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, stream));
            FCC_TRY(sync_stream());
            v = obs.host;
        }
        int64_t w = 0;
        for (int64_t i = 0; i < N; ++i) {
            if (typ != 0 && type_h[i] != typ) continue;
            if (out) out[w] = v[3 * i + which];
            ++w;
        }
        if (count) *count = w;
        return FCC_OK;
    }

    fcc_status health(int32_t* nonfinite, int32_t* barrier_error) override {
        int f = 0;
        GridSync g{};
        CUDA_TRY(cudaMemcpyAsync(&f, flags_d, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(&g, sync_d, sizeof(GridSync), cudaMemcpyDeviceToHost, stream));
        FCC_TRY(sync_stream());
        if (nonfinite) *nonfinite = (f & F_NONFINITE) ? 1 : 0;
        if (barrier_error) *barrier_error = g.error ? 1 : 0;
        return FCC_OK;
    }

    fcc_status body_energy(double* out) override {
        std::vector<T> e;
        FCC_TRY(fetch(E.p, (size_t)N, e));
        FCC_TRY(sync_stream());
        double acc = 0;
        for (T v : e) acc += (double)v;
        *out = acc;
        return FCC_OK;
    }

    fcc_status timing(double* ms, int64_t* launches, int64_t* steps) override {
        if (ms) *ms = last_ms;
        if (launches) *launches = last_launches;
        if (steps) *steps = last_steps;
        return FCC_OK;
    }
};

// ------------------------------------------------- stateless entry points
template <class T>
fcc_status build_neighbors_t(int64_t n, const double* x, const double* y, const double* rmax, double Lx, double Ly,
                             double cutoff, double range, int32_t cap, int32_t* cellid_o, int32_t* perm_o,
                             int32_t* start_o, int32_t* stop_o, int32_t* idx_o, int32_t* count_o) {
    if (n < 0 || cap < 1) return fail(FCC_ERR_ARGUMENT, "n must be >= 0 and cap >= 1");
    if (n == 0) return FCC_OK;
    if (n > (1 << 27)) return fail(FCC_ERR_UNSUPPORTED, "at most 2^27 bodies");
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    } guard{st};
    SimDesc<T> s{};
    s.Lx = (T)Lx;
    s.Ly = (T)Ly;
    int64_t gx = 0, gy = 0;
    FCC_TRY(cell_grid_dims((double)s.Lx, (double)s.Ly, cutoff, &gx, &gy));
    if (gx * gy > (1 << 28)) return fail(FCC_ERR_UNSUPPORTED, "cell grid too large");
    const int ncx = (int)gx, ncy = (int)gy;
    s.wx = s.Lx / (T)ncx;
    s.wy = s.Ly / (T)ncy;
    s.ncx = ncx;
    s.ncy = ncy;
    s.ncells = ncx * ncy;
    s.n = (int)n;
    s.nbrange = (T)range;
    s.skin = T(0);
    const size_t N = (size_t)n, C = (size_t)ncx * ncy;
    DBuf<SimDesc<T>> sims;
    DBuf<T> rec, xd, yd, rd;
    DBuf<int> sim_of, cellid, slot, perm, cstart, cstop, ccount, cell_sim, nb_idx, nb_count, flags, maxcount;
    DBuf<long long> clock, builds;
    DBuf<GridSync> sync;
    FCC_TRY(sims.upload(std::vector<SimDesc<T>>{s}, st));
    std::vector<T> hx(N), hy(N), hr(N);
    for (size_t i = 0; i < N; ++i) hx[i] = (T)x[i], hy[i] = (T)y[i], hr[i] = (T)rmax[i];
    FCC_TRY(xd.upload(hx, st));
    FCC_TRY(yd.upload(hy, st));
    FCC_TRY(rd.upload(hr, st));
    FCC_TRY(rec.alloc(N * RECW, st));
    FCC_TRY(sim_of.alloc(N, st));
    FCC_TRY(cellid.alloc(N, st));
    FCC_TRY(slot.alloc(N, st));
    FCC_TRY(perm.alloc(N, st));
    FCC_TRY(cstart.alloc(C, st));
    FCC_TRY(cstop.alloc(C, st));
    FCC_TRY(ccount.alloc(C, st));
    FCC_TRY(cell_sim.alloc(C, st));
    FCC_TRY(nb_idx.alloc(N * cap, st));
    FCC_TRY(nb_count.alloc(N, st));
    FCC_TRY(flags.upload(std::vector<int>{F_ACTIVE | F_CONTACT | F_NEED}, st));
    FCC_TRY(maxcount.alloc(1, st));
    FCC_TRY(clock.alloc(1, st));
    FCC_TRY(builds.alloc(1, st));
    FCC_TRY(sync.upload(std::vector<GridSync>{GridSync{0, 0, 0, 1}}, st));
    DevPtrs<T> d{};
    d.sims = sims.p;
    d.nsims = 1;
    d.Ntot = (int)N;
    d.Ctot = (int)C;
    d.cap = cap;
    d.sim_of = sim_of.p;
    d.rec0 = rec.p;
    d.rec1 = rec.p;
    d.cellid = cellid.p;
    d.slot = slot.p;
    d.perm = perm.p;
    d.cstart = cstart.p;
    d.cstop = cstop.p;
    d.ccount = ccount.p;
    d.cell_sim = cell_sim.p;
    d.nb_idx = nb_idx.p;
    d.nb_count = nb_count.p;
    d.flags = flags.p;
    d.maxcount = maxcount.p;
    d.clock = clock.p;
    d.builds = builds.p;
    d.sync = sync.p;
    const int grid = (int)((N + 255) / 256);
    k_pack_head<T><<<grid, 256, 0, st>>>(rec.p, xd.p, yd.p, rd.p, (int)N);
    k_phase_count<T><<<grid, 256, 0, st>>>(d, 0);
    k_phase_scan<T><<<1, 1024, 0, st>>>(d);
    k_phase_scatter<T><<<grid, 256, 0, st>>>(d);
    k_phase_sort<T><<<(int)((C + 255) / 256), 256, 0, st>>>(d);
    k_phase_neighbors<T><<<neighbor_grid(N), 256, 0, st>>>(d, 0);
    CUDA_TRY(cudaGetLastError());
    std::vector<int> a, b, cnt;
    a.resize(N);
    CUDA_TRY(cudaMemcpyAsync(a.data(), cellid.p, N * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < N; ++i) cellid_o[i] = a[i] + 1;
    CUDA_TRY(cudaMemcpyAsync(a.data(), perm.p, N * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < N; ++i) perm_o[i] = a[i] + 1;
    a.resize(C);
    b.resize(C);
    CUDA_TRY(cudaMemcpyAsync(a.data(), cstart.p, C * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(b.data(), cstop.p, C * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t c = 0; c < C; ++c) {
        const bool empty = b[c] <= a[c];
        start_o[c] = empty ? 1 : a[c] + 1;
        stop_o[c] = empty ? 0 : b[c];
    }
    cnt.resize(N);
    a.resize(N * cap);
    CUDA_TRY(cudaMemcpyAsync(cnt.data(), nb_count.p, N * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(a.data(), nb_idx.p, N * cap * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < N; ++i) {
        count_o[i] = cnt[i];
        for (int q = 0; q < cap; ++q) idx_o[i * cap + q] = q < cnt[i] ? a[i * cap + q] + 1 : 0;
    }
    return FCC_OK;
}

}  // namespace

#include "fcc_noalloc.cu"
#include "fcc_pool.cu"

struct fcc_sim {
    std::unique_ptr<EngineBase> impl;
    int device = 0;
};

extern "C" {

fcc_status fcc_create(const fcc_params* params, const fcc_bodies_host* bodies, fcc_sim** out) {
    if (!out) return fail(FCC_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!params) return fail(FCC_ERR_ARGUMENT, "null params");
    std::unique_ptr<fcc_sim> h(new fcc_sim);
    fcc_status st;
    if (params->precision == 64) {
        auto e = std::make_unique<Engine<double>>();
        st = e->init(params, bodies);
        h->impl = std::move(e);
    } else if (params->precision == 32) {
        auto e = std::make_unique<Engine<float>>();
        st = e->init(params, bodies);
        h->impl = std::move(e);
    } else {
        return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    }
    if (st != FCC_OK) return st;
    cudaGetDevice(&h->device);
    *out = h.release();
    return FCC_OK;
}

fcc_status fcc_destroy(fcc_sim* sim) {
    if (sim) cudaSetDevice(sim->device);
    delete sim;
    return FCC_OK;
}

#define SIM_CALL(expr)                                                   \
    do {                                                                 \
        if (!sim) return fail(FCC_ERR_ARGUMENT, "null simulation");      \
        cudaError_t e_ = cudaSetDevice(sim->device);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, "cudaSetDevice");    \
        return sim->impl->expr;                                          \
    } while (0)

fcc_status fcc_step(fcc_sim* sim, int64_t n) { SIM_CALL(step(n, true)); }
fcc_status fcc_run(fcc_sim* sim, int64_t n, int64_t every, fcc_callback cb, void* user, int32_t graph) {
    SIM_CALL(run(sim, n, every, cb, user, graph != 0));
}
fcc_status fcc_update_neighbors(fcc_sim* sim, int32_t force) { SIM_CALL(update_neighbors(force != 0)); }
fcc_status fcc_compute_gradients(fcc_sim* sim) { SIM_CALL(compute_gradients()); }
fcc_status fcc_get_state(fcc_sim* sim, fcc_bodies_host* out, int64_t* clock, double* t, int64_t* step) {
    SIM_CALL(get_state(out, clock, t, step));
}
fcc_status fcc_set_state(fcc_sim* sim, const fcc_bodies_host* in, int64_t clock) { SIM_CALL(set_state(in, clock)); }
fcc_status fcc_set_dt(fcc_sim* sim, double dt) { SIM_CALL(set_dt(dt)); }
fcc_status fcc_host_alloc(int64_t bytes, void** out) {
    if (!out || bytes < 0) return fail(FCC_ERR_ARGUMENT, "fcc_host_alloc: bad argument");
    *out = nullptr;
    if (bytes == 0) return FCC_OK;
    CUDA_TRY(cudaMallocHost(out, (size_t)bytes));
    return FCC_OK;
}
fcc_status fcc_host_free(void* ptr) {
    if (ptr) CUDA_TRY(cudaFreeHost(ptr));
    return FCC_OK;
}
fcc_status fcc_get_gradients(fcc_sim* sim, const fcc_gradients_host* out) { SIM_CALL(get_gradients(out)); }
fcc_status fcc_get_geometry(fcc_sim* sim, const fcc_geometry_host* out) { SIM_CALL(get_geometry(out)); }
fcc_status fcc_neighbor_dims(fcc_sim* sim, int32_t* ncx, int32_t* ncy, int32_t* cap, int64_t* builds, int32_t* valid) {
    SIM_CALL(neighbor_dims(ncx, ncy, cap, builds, valid));
}
fcc_status fcc_get_neighbors(fcc_sim* sim, const fcc_neighbors_host* out) { SIM_CALL(get_neighbors(out)); }
fcc_status fcc_perimeters(fcc_sim* sim, int32_t type, double* out, int64_t* count) { SIM_CALL(observable(0, type, out, count)); }
fcc_status fcc_areas(fcc_sim* sim, int32_t type, double* out, int64_t* count) { SIM_CALL(observable(1, type, out, count)); }
fcc_status fcc_shape_index(fcc_sim* sim, int32_t type, double* out, int64_t* count) { SIM_CALL(observable(2, type, out, count)); }
fcc_status fcc_body_energy(fcc_sim* sim, double* out) { SIM_CALL(body_energy(out)); }
fcc_status fcc_last_timing(fcc_sim* sim, double* ms, int64_t* launches, int64_t* steps) {
    SIM_CALL(timing(ms, launches, steps));
}
fcc_status fcc_health(fcc_sim* sim, int32_t* nonfinite, int32_t* barrier_error) {
    SIM_CALL(health(nonfinite, barrier_error));
}

fcc_status fcc_barrier_selftest(int32_t blocks, int32_t* error, double* ms) {
    if (blocks < 1 || blocks > 148) return fail(FCC_ERR_ARGUMENT, "blocks must be 1..148");
    if (!error) return fail(FCC_ERR_ARGUMENT, "null argument");
    GridSync* gs = nullptr;  // [0]: generation-word barrier, [1]: flat barrier
    CUDA_TRY(cudaMalloc(&gs, 2 * sizeof(GridSync)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMemset(gs, 0, 2 * sizeof(GridSync));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
    if (e == cudaSuccess) {
        void* args[] = {&gs};
        e = cudaLaunchCooperativeKernel((void*)k_barrier_selftest, dim3(blocks), dim3(64), args, 0, 0);
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    GridSync g[2]{};
    if (e == cudaSuccess) e = cudaMemcpy(g, gs, 2 * sizeof(GridSync), cudaMemcpyDeviceToHost);
    float t = 0.f;
    if (e == cudaSuccess && ms) e = cudaEventElapsedTime(&t, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(gs);
    CUDA_TRY(e);
    // 1: both waits ran out; 0: neither did; 2: only one of them did
    *error = g[0].error && g[1].error ? 1 : (g[0].error || g[1].error ? 2 : 0);
    if (ms) *ms = t;
    return FCC_OK;
}

fcc_status fcc_philox_noise(uint64_t seed, uint64_t draw, int64_t nbodies, int32_t precision, double* out) {
    if (precision != 32 && precision != 64) return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    if (nbodies <= 0) return FCC_OK;
    if (nbodies > (1ll << 30)) return fail(FCC_ERR_UNSUPPORTED, "at most 2^30 bodies");
    const uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
    const size_t n3 = 3 * (size_t)nbodies;
    const int grid = (int)((nbodies + 255) / 256);
    if (precision == 64) {
        double* d = nullptr;
        CUDA_TRY(cudaMalloc(&d, n3 * sizeof(double)));
        k_noise<double><<<grid, 256>>>(k0, k1, draw, (int)nbodies, d);
        cudaError_t e = cudaMemcpy(out, d, n3 * sizeof(double), cudaMemcpyDeviceToHost);
        cudaFree(d);
        CUDA_TRY(e);
    } else {
        float* d = nullptr;
        CUDA_TRY(cudaMalloc(&d, n3 * sizeof(float)));
        k_noise<float><<<grid, 256>>>(k0, k1, draw, (int)nbodies, d);
        std::vector<float> h(n3);
        cudaError_t e = cudaMemcpy(h.data(), d, n3 * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d);
        CUDA_TRY(e);
        for (size_t q = 0; q < n3; ++q) out[q] = (double)h[q];
    }
    return FCC_OK;
}

fcc_status fcc_build_neighbors(int32_t precision, int64_t n, const double* x, const double* y, const double* rmax,
                               double Lx, double Ly, double cutoff, double range, int32_t cap, int32_t* cellid,
                               int32_t* perm, int32_t* start, int32_t* stop, int32_t* idx, int32_t* count) {
    if (precision == 64)
        return build_neighbors_t<double>(n, x, y, rmax, Lx, Ly, cutoff, range, cap, cellid, perm, start, stop, idx, count);
    if (precision == 32)
        return build_neighbors_t<float>(n, x, y, rmax, Lx, Ly, cutoff, range, cap, cellid, perm, start, stop, idx, count);
    return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
}

const char* fcc_last_error(void) { return g_err.c_str(); }

const char* fcc_version(void) {
    return "libfcc_b200 sm_100a: persistent cooperative step kernel (lanes x nodes per body: 8x5, 4x10, 16x3)";
}

}  // extern "C"
