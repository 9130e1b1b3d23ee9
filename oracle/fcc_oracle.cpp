// fcc_oracle.cpp — CPU oracle of the FourierContourCells.jl time step.
//
// TEST INFRASTRUCTURE ONLY: the parity reference of tests/ and the timed CPU
// baseline of bench.py.  The product library never links or calls it.
//
// A plain restatement of the reference's CPU path, function by function, in
// the reference's operation order (no FMA contraction: built with
// -ffp-contract=off, like Julia, which never fuses a*b+c by itself).  Each
// function cites the reference file:line it follows.  Templated on the
// floating-point type T (double = the Float64 oracle, float = Float32).
// Bodies are data-parallel (OpenMP), as the KernelAbstractions CPU backend is.

#include "fcc_oracle.h"
#include "../include/fcc_user_terms.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <set>
#include <string>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

fcc_status fail(fcc_status code, const std::string& msg) {
    g_err = msg;
    return code;
}

// ---------------------------------------------------------------- Philox --
// src/random.jl:10-36: Philox4x32 with 10 rounds.
void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// src/random.jl:42-44
inline float uniform_open(float*, uint32_t a, uint32_t) { return ((float)(a >> 9) + 0.5f) * 0x1p-23f; }
inline double uniform_open(double*, uint32_t a, uint32_t b) {
    return ((double)(((((uint64_t)a) << 32) | b) >> 12) + 0.5) * 0x1p-52;
}

inline float t_log(float x) { return std::log(x); }
inline double t_log(double x) { return std::log(x); }

// src/random.jl:47-51: Box-Muller.
template <class T> void box_muller(T u1, T u2, T& z1, T& z2) {
    T r = std::sqrt(T(-2) * t_log(u1));
    T arg = (T(2) * T(M_PI)) * u2;
    T s = std::sin(arg), c = std::cos(arg);
    z1 = r * c;
    z2 = r * s;
}

// src/random.jl:75-78: two normals of body i (1-based) in draw n from block b.
template <class T> void philox_pair(uint32_t k0, uint32_t k1, uint64_t i, uint64_t n, uint32_t block, T& z1, T& z2) {
    uint32_t c[4] = {(uint32_t)i, (uint32_t)n, (uint32_t)(n >> 32), block};
    philox(c, k0, k1);
    T* tag = nullptr;
    box_muller<T>(uniform_open(tag, c[0], c[1]), uniform_open(tag, c[2], c[3]), z1, z2);
}

// ---------------------------------------------------------------- box ------
// src/box.jl:14
template <class T> inline T minimum_image(T d, T L) { return d - L * std::rint(d / L); }

// src/box.jl:21-30
template <class T> inline T wrap(T x, T L, int32_t& shift) {
    T s = std::floor(x / L);
    T xp = x - s * L;
    if (xp >= L) {
        xp = T(0);
        s += T(1);
    }
    shift = (int32_t)s;
    return xp;
}

// src/neighbors.jl:40-42
template <class T> inline void grid_coords(int32_t ncx, int32_t ncy, T wx, T wy, T x, T y, int32_t& cx, int32_t& cy) {
    // clamped into the grid (inputs outside [0, L) would index outside it)
    cx = std::max<int32_t>(0, std::min((int32_t)(x / wx), ncx - 1));
    cy = std::max<int32_t>(0, std::min((int32_t)(y / wy), ncy - 1));
}

inline int32_t jmod(int32_t a, int32_t n) {
    int32_t r = a % n;
    return r < 0 ? r + n : r;
}

const double SHAPE_BOUND = std::sqrt(2.0 / 3.0);  // src/dynamics.jl:26

// ---------------------------------------------------------------- terms ----
template <class T> struct Term {
    int kind = 0;
    int user = 0;  // FCC_USER_*: index in the compiled table (include/fcc_user_terms.h)
    std::vector<int32_t> types_on;  // OnTypes; empty = all types
    T a = 0, b = 0;
    int nJ = 1;
    std::vector<T> J, Jrel;  // column-major nJ x nJ
    bool applies(int32_t type) const {  // src/energies/interface.jl:150, 284
        if (types_on.empty()) return true;
        return std::find(types_on.begin(), types_on.end(), type) != types_on.end();
    }
};

template <class T> struct BodyTypeT {
    T v0, Dr, Dt, mur, muth, muab;
    bool parent_drag;
    int maxmode;  // 0: every mode; else modes n > maxmode are held at zero (no reference counterpart)
};

struct SimBase {
    virtual ~SimBase() = default;
    virtual fcc_status step(int64_t n) = 0;
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
    virtual fcc_status counters(int64_t* tests, int64_t* hits, double* mind) = 0;
};

template <class T> struct Sim final : SimBase {
    // basis (src/basis.jl:35-63): nθ x nc column-major C, D, DD; cs 2 x nθ
    int64_t N = 0;
    int K = 0, nc = 0, nth = 0;
    T dphi = 0;
    std::vector<T> C, D, DD, cs;
    T Lx = 0, Ly = 0;
    // bodies (src/bodies.jl:62-72); type/parent kept 1-based
    std::vector<T> x, y, th, coef, R0;
    std::vector<int32_t> imgx, imgy, type, parent;
    // geometry (src/geometry.jl:13-32)
    std::vector<T> lab, labR0, R, dR, ddR, rmax;
    // gradients (src/gradients.jl:15-38)
    std::vector<T> GR, GD, GDD, P, gx, gy, gth, glab, gcoef, Ebody;
    // cell list (src/neighbors.jl:16-33), 1-based contents
    int32_t ncx = 1, ncy = 1;
    T wx = 0, wy = 0;
    std::vector<int32_t> cellid, perm, start, stop;
    // neighbour list (src/neighbors.jl:110-127)
    int32_t cap = 32;
    std::vector<int32_t> idx, count;
    T skin = 0;
    std::vector<T> x0, y0, rmax0;
    bool valid = false;
    int64_t builds = 0;
    // children and bonds (src/bodies.jl:116-135, src/energies/bonds.jl:47-71)
    int32_t ccap = 1, bcap = 1;
    std::vector<int32_t> cidx, ccount, bidx, bcount;
    // terms and types
    std::vector<BodyTypeT<T>> types;
    std::vector<Term<T>> body_terms, contact_terms, bond_terms;
    uint32_t k0 = 0, k1 = 0;
    std::vector<T> disp;
    int32_t status[3] = {0, 0, 0};
    int64_t clock = 0;
    T dt = 0, t = 0;
    int64_t stepno = 0;
    // work counters of the last contact evaluation
    int64_t n_tests = 0, n_hits = 0;
    std::vector<double> mind;

    static void to_T(std::vector<T>& v, const double* src, size_t n) {
        v.resize(n);
        for (size_t i = 0; i < n; ++i) v[i] = (T)src[i];
    }

    // ----------------------------------------------------------- setup --
    fcc_status init(const fcc_params* p, const fcc_bodies_host* b) {
        // src/simulation.jl:66-105 in order
        if (!p || !b) return fail(FCC_ERR_ARGUMENT, "null argument");
        if (p->ntypes < 1 || p->ntypes > FCC_MAX_TYPES || !p->types)
            return fail(FCC_ERR_ARGUMENT, "types must hold 1..8 BodyType entries");
        for (int t = 0; t < p->ntypes; ++t) {
            const fcc_body_type& bt = p->types[t];
            if (bt.parent_drag != 0 && bt.parent_drag != 1)
                return fail(FCC_ERR_ARGUMENT, "drag must be :substrate or :parent");
            if (bt.maxmode < 0) return fail(FCC_ERR_ARGUMENT, "a body type's maxmode must be >= 0");
            types.push_back({(T)bt.v0, (T)bt.Dr, (T)bt.Dt, (T)bt.mu_r, (T)bt.mu_theta, (T)bt.mu_ab, bt.parent_drag == 1,
                             bt.maxmode});
        }
        if (p->nterms < 0 || p->nterms > FCC_MAX_TERMS || (p->nterms > 0 && !p->terms))
            return fail(FCC_ERR_ARGUMENT, "energy terms must be BodyTerms, ContactTerms or BondTerms");
        for (int q = 0; q < p->nterms; ++q) {
            const fcc_term& ft = p->terms[q];
            Term<T> tm;
            tm.kind = ft.kind;
            if (ft.kind < FCC_TENSION || ft.kind > FCC_USER_BOND)
                return fail(FCC_ERR_ARGUMENT, "energy terms must be BodyTerms, ContactTerms or BondTerms");
            tm.user = ft.user;
            const int nuser = ft.kind == FCC_USER_BODY ? fcc_user::n_body
                              : ft.kind == FCC_USER_CONTACT ? fcc_user::n_contact
                              : ft.kind == FCC_USER_BOND ? fcc_user::n_bond : 1;
            if (ft.kind >= FCC_USER_BODY && (ft.user < 0 || ft.user >= nuser))
                return fail(FCC_ERR_ARGUMENT, "no compiled user term with this index");
            if (ft.ntypes_on < 0 || ft.ntypes_on > FCC_MAX_TYPES) return fail(FCC_ERR_ARGUMENT, "OnTypes: bad type list");
            for (int u = 0; u < ft.ntypes_on; ++u) tm.types_on.push_back(ft.types_on[u]);
            tm.a = (T)ft.a;
            tm.b = (T)ft.b;
            if (ft.kind == FCC_OVERLAP) {
                if (ft.nJ < 1 || ft.nJ > FCC_MAX_TYPES) return fail(FCC_ERR_DIMENSION, "coupling tables must be square and equal-sized");
                tm.nJ = ft.nJ;
                to_T(tm.J, ft.J, (size_t)ft.nJ * ft.nJ);
                to_T(tm.Jrel, ft.Jrel, (size_t)ft.nJ * ft.nJ);
            }
            if (ft.kind == FCC_TENSION || ft.kind == FCC_PERIMETER_ELASTICITY || ft.kind == FCC_USER_BODY)
                body_terms.push_back(tm);
            else if (ft.kind == FCC_OVERLAP || ft.kind == FCC_LINEAR_REPULSION || ft.kind == FCC_USER_CONTACT)
                contact_terms.push_back(tm);
            else bond_terms.push_back(tm);
        }
        N = b->n;
        if (N < 0) return fail(FCC_ERR_DIMENSION, "inconsistent body array lengths");
        int32_t maxtype = 0;
        for (int64_t i = 0; i < N; ++i) maxtype = std::max(maxtype, b->type[i]);
        for (const Term<T>& tm : contact_terms)
            if (tm.kind == FCC_OVERLAP && tm.nJ > 1 && tm.nJ < maxtype)
                return fail(FCC_ERR_DIMENSION, "Overlap coupling table smaller than the number of body types");
        for (int64_t i = 0; i < N; ++i)
            if (b->type[i] > p->ntypes) return fail(FCC_ERR_ARGUMENT, "body type without BodyType entry");
        for (int64_t i = 0; i < N; ++i)
            if (b->type[i] < 1) return fail(FCC_ERR_ARGUMENT, "body type ids are 1-based");
        // check_parents (src/simulation.jl:108-118)
        for (int64_t i = 0; i < N; ++i) {
            int64_t pp = b->parent[i];
            if (pp < 1 || pp > N)
                return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has parent " + std::to_string(pp) + " outside 1:" + std::to_string(N));
            if (!types[b->type[i] - 1].parent_drag) continue;
            if (pp == i + 1)
                return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has drag = :parent but is its own parent");
            if (types[b->type[pp - 1] - 1].parent_drag)
                return fail(FCC_ERR_ARGUMENT, "body " + std::to_string(i + 1) + " has drag = :parent, but so has its parent " + std::to_string(pp) + " (one level only)");
        }
        // basis (src/basis.jl:35-63)
        K = b->ncoef / 2;
        int maxmode = K + 1;
        nth = p->ntheta;
        if (maxmode < 2) return fail(FCC_ERR_ARGUMENT, "maxmode must be ≥ 2");
        if (!(nth > 2 * maxmode)) return fail(FCC_ERR_ARGUMENT, "nθ must exceed 2·maxmode");
        for (const BodyTypeT<T>& bt : types)
            if (bt.maxmode > maxmode) return fail(FCC_ERR_ARGUMENT, "a body type's maxmode exceeds the simulation's");
        nc = 2 * K + 1;
        if (b->ncoef != nc) return fail(FCC_ERR_DIMENSION, "coefficient rows must be odd: [a₀; aₙ; bₙ]");
        double dphi64 = 2 * M_PI / nth;
        dphi = (T)dphi64;
        C.assign((size_t)nth * nc, 0); D.assign((size_t)nth * nc, 0); DD.assign((size_t)nth * nc, 0); cs.assign(2 * (size_t)nth, 0);
        for (int k = 0; k < nth; ++k) {
            double phi = k * dphi64;
            cs[2 * k] = (T)std::cos(phi);
            cs[2 * k + 1] = (T)std::sin(phi);
            C[k] = 1;
            for (int m = 1; m <= K; ++m) {
                int n = m + 1;
                double s = std::sin(n * phi), c = std::cos(n * phi);
                C[k + (size_t)nth * m] = (T)c;
                C[k + (size_t)nth * (K + m)] = (T)s;
                D[k + (size_t)nth * m] = (T)(-n * s);
                D[k + (size_t)nth * (K + m)] = (T)(n * c);
                DD[k + (size_t)nth * m] = (T)(-(n * n) * c);
                DD[k + (size_t)nth * (K + m)] = (T)(-(n * n) * s);
            }
        }
        Lx = (T)p->Lx;
        Ly = (T)p->Ly;
        to_T(x, b->x, N); to_T(y, b->y, N); to_T(th, b->theta, N);
        to_T(coef, b->coef, (size_t)nc * N); to_T(R0, b->R0, N);
        imgx.assign(b->imgx, b->imgx + N); imgy.assign(b->imgy, b->imgy + N);
        type.assign(b->type, b->type + N); parent.assign(b->parent, b->parent + N);
        // cutoff and CellList (src/simulation.jl:90-91, src/neighbors.jl:27-33), in Float64 as Julia promotes
        double maxR0 = 0;
        for (int64_t i = 0; i < N; ++i) maxR0 = std::max(maxR0, (double)R0[i]);
        // contact_range (src/energies/contact.jl:54): the largest interaction
        // range of the contact terms (0 for the built-in ones), in T
        double range64 = 0;
        for (const Term<T>& tm : contact_terms)
            if (tm.kind == FCC_USER_CONTACT)
                range64 = std::max(range64, (double)fcc_user::contact_range<T>(tm.user, tm.a, tm.b));
        double cutoff = 2 * maxR0 * (1 + SHAPE_BOUND) + range64 + p->skin;
        auto ncells = [&](T L) { int64_t n = (int64_t)std::floor((double)L / cutoff); return (int32_t)(n >= 3 ? n : 1); };
        ncx = ncells(Lx);
        ncy = ncells(Ly);
        wx = Lx / (T)ncx;
        wy = Ly / (T)ncy;
        cellid.assign(N, 0); perm.assign(N, 0);
        start.assign((size_t)ncx * ncy, 0); stop.assign((size_t)ncx * ncy, 0);
        disp.assign(3 * (size_t)N, 0);
        // NeighborList (src/neighbors.jl:121-127)
        if (!(p->skin >= 0)) return fail(FCC_ERR_ARGUMENT, "skin must be non-negative");
        skin = (T)p->skin;
        cap = p->nl_capacity > 0 ? p->nl_capacity : 32;
        idx.assign((size_t)cap * N, 0); count.assign(N, 0);
        x0.assign(N, 0); y0.assign(N, 0); rmax0.assign(N, 0);
        // ChildList (src/bodies.jl:121-135)
        ccount.assign(N, 0);
        for (int64_t k = 0; k < N; ++k) if (parent[k] != k + 1) ccount[parent[k] - 1] += 1;
        ccap = 1;
        for (int64_t k = 0; k < N; ++k) ccap = std::max(ccap, ccount[k]);
        cidx.assign((size_t)ccap * N, 0);
        std::fill(ccount.begin(), ccount.end(), 0);
        for (int64_t k = 0; k < N; ++k) {
            int32_t pp = parent[k];
            if (pp == k + 1) continue;
            ccount[pp - 1] += 1;
            cidx[(size_t)(ccount[pp - 1] - 1) + (size_t)ccap * (pp - 1)] = (int32_t)(k + 1);
        }
        // BondList (src/energies/bonds.jl:52-71)
        bcount.assign(N, 0);
        std::set<std::pair<int64_t, int64_t>> seen;
        for (int64_t q = 0; q < p->nbonds; ++q) {
            int64_t i = p->bonds[2 * q], j = p->bonds[2 * q + 1];
            if (!(1 <= i && i <= N && 1 <= j && j <= N))
                return fail(FCC_ERR_ARGUMENT, "bond (" + std::to_string(i) + ", " + std::to_string(j) + ") refers to a body outside 1:" + std::to_string(N));
            if (i == j) return fail(FCC_ERR_ARGUMENT, "bond (" + std::to_string(i) + ", " + std::to_string(j) + ") connects a body to itself");
            auto key = std::make_pair(std::min(i, j), std::max(i, j));
            if (seen.count(key)) return fail(FCC_ERR_ARGUMENT, "duplicate bond (" + std::to_string(i) + ", " + std::to_string(j) + ")");
            seen.insert(key);
            bcount[i - 1] += 1;
            bcount[j - 1] += 1;
        }
        bcap = 1;
        for (int64_t k = 0; k < N; ++k) bcap = std::max(bcap, bcount[k]);
        bidx.assign((size_t)bcap * N, 0);
        std::fill(bcount.begin(), bcount.end(), 0);
        for (int64_t q = 0; q < p->nbonds; ++q) {
            int64_t i = p->bonds[2 * q], j = p->bonds[2 * q + 1];
            int64_t ab[2][2] = {{i, j}, {j, i}};
            for (auto& e : ab) {
                bcount[e[0] - 1] += 1;
                bidx[(size_t)(bcount[e[0] - 1] - 1) + (size_t)bcap * (e[0] - 1)] = (int32_t)e[1];
            }
        }
        // philox_key (src/random.jl:103)
        k0 = (uint32_t)(p->seed & 0xffffffffu);
        k1 = (uint32_t)(p->seed >> 32);
        dt = (T)p->dt;
        // geometry and gradient buffers
        lab.assign((size_t)nc * N, 0); labR0.assign((size_t)nc * N, 0);
        R.assign((size_t)nth * N, 0); dR.assign((size_t)nth * N, 0); ddR.assign((size_t)nth * N, 0); rmax.assign(N, 0);
        GR.assign((size_t)nth * N, 0); GD.assign((size_t)nth * N, 0); GDD.assign((size_t)nth * N, 0); P.assign((size_t)nth * N, 0);
        gx.assign(N, 0); gy.assign(N, 0); gth.assign(N, 0);
        glab.assign((size_t)nc * N, 0); gcoef.assign((size_t)nc * N, 0); Ebody.assign(N, 0);
        mind.assign(N, INFINITY);
        range_T = (T)range64 + skin;
        contact_range_T = (T)range64;
        // enforce_shape! and update_geometry! (src/simulation.jl:102-103)
        enforce_all();
        update_geometry();
        return FCC_OK;
    }
    T range_T = 0, contact_range_T = 0;

    // ---------------------------------------------------- shape & geometry --
    // Modes above the body type's maxmode held at zero (a per-type limit the
    // reference does not have; maxmode = 0 leaves every mode free).
    void mask_modes(int64_t i) {
        const int mm = types[type[i] - 1].maxmode;
        if (mm <= 0) return;
        T* c = &coef[(size_t)nc * i];
        for (int m = std::max(mm - 1, 0) + 1; m <= K; ++m) c[m] = c[K + m] = T(0);
    }

    // src/dynamics.jl:44-64
    void enforce_shape(int64_t i) {
        mask_modes(i);
        T* c = &coef[(size_t)nc * i];
        T s = 0;
        for (int m = 1; m <= K; ++m) s += std::sqrt(c[m] * c[m] + c[K + m] * c[K + m]);
        T bound = (T)SHAPE_BOUND;
        if (s > bound) {
            T f = bound / s;
            for (int m = 1; m <= K; ++m) {
                c[m] *= f;
                c[K + m] *= f;
            }
        }
        T q = 0;
        for (int m = 1; m <= K; ++m) q += c[m] * c[m] + c[K + m] * c[K + m];
        c[0] = std::sqrt(T(1) - q / T(2));
    }
    void enforce_all() {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) enforce_shape(i);
    }

    // src/geometry.jl:208-227
    void lab_frame(int64_t i, T thi, T r0) {
        const T* c = &coef[(size_t)nc * i];
        T* l = &lab[(size_t)nc * i];
        T* lr = &labR0[(size_t)nc * i];
        l[0] = c[0];
        lr[0] = r0 * c[0];
        T bound = c[0];
        for (int m = 1; m <= K; ++m) {
            int n = m + 1;
            T a = c[m], b = c[K + m];
            T arg = (T)n * thi;
            T s = std::sin(arg), co = std::cos(arg);
            T al = a * co - b * s;
            T be = a * s + b * co;
            l[m] = al;
            l[K + m] = be;
            lr[m] = r0 * al;
            lr[K + m] = r0 * be;
            bound += std::sqrt(a * a + b * b);
        }
        rmax[i] = r0 * bound;
    }

    // src/geometry.jl:248-257 (CPU: three products into the row blocks)
    void synthesize_body(int64_t i) {
        const T* lr = &labR0[(size_t)nc * i];
        for (int k = 0; k < nth; ++k) {
            T r = 0, r1 = 0, r2 = 0;
            for (int c = 0; c < nc; ++c) {
                r += C[k + (size_t)nth * c] * lr[c];
                r1 += D[k + (size_t)nth * c] * lr[c];
                r2 += DD[k + (size_t)nth * c] * lr[c];
            }
            R[k + (size_t)nth * i] = r;
            dR[k + (size_t)nth * i] = r1;
            ddR[k + (size_t)nth * i] = r2;
        }
    }
    void synthesize() {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) synthesize_body(i);
    }
    // src/geometry.jl:240-245
    void update_geometry() {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            lab_frame(i, th[i], R0[i]);
            synthesize_body(i);
        }
    }

    // src/geometry.jl:282-291
    T contour_radius_dir(int64_t j, T c1, T s1) const {
        const T* l = &lab[(size_t)nc * j];
        T c = c1, s = s1;
        T r = l[0];
        for (int m = 1; m <= K; ++m) {
            T cn = c * c1 - s * s1;
            T sn = s * c1 + c * s1;
            c = cn;
            s = sn;
            r += l[m] * c + l[K + m] * s;
        }
        return R0[j] * r;
    }

    // ---------------------------------------------------- neighbours ------
    // src/neighbors.jl:81-92: cell index, stable sortperm, cell bounds
    void update_celllist() {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            int32_t cx, cy;
            grid_coords(ncx, ncy, wx, wy, x[i], y[i], cx, cy);
            cellid[i] = cx + ncx * cy + 1;
        }
        for (int64_t i = 0; i < N; ++i) perm[i] = (int32_t)(i + 1);
        std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return cellid[a - 1] < cellid[b - 1]; });
        std::fill(start.begin(), start.end(), 1);
        std::fill(stop.begin(), stop.end(), 0);
        for (int64_t s = 0; s < N; ++s) {
            int32_t c = cellid[perm[s] - 1];
            if (s == 0 || cellid[perm[s - 1] - 1] != c) start[c - 1] = (int32_t)(s + 1);
            if (s == N - 1 || cellid[perm[s + 1] - 1] != c) stop[c - 1] = (int32_t)(s + 1);
        }
    }

    // src/neighbors.jl:148-174 (one body)
    int32_t neighbor_body(int64_t i, int32_t* out, int32_t capv) const {
        T xi = x[i], yi = y[i];
        T ri = rmax[i] + range_T;
        int32_t cx, cy;
        grid_coords(ncx, ncy, wx, wy, xi, yi, cx, cy);
        int32_t rx = ncx >= 3 ? 1 : 0, ry = ncy >= 3 ? 1 : 0;
        int32_t n = 0;
        for (int32_t oy = -ry; oy <= ry; ++oy)
            for (int32_t ox = -rx; ox <= rx; ++ox) {
                int32_t cell = jmod(cx + ox, ncx) + ncx * jmod(cy + oy, ncy);
                for (int32_t q = start[cell]; q <= stop[cell]; ++q) {
                    int32_t j = perm[q - 1] - 1;
                    if (j == i) continue;
                    T dx = minimum_image(xi - x[j], Lx);
                    T dy = minimum_image(yi - y[j], Ly);
                    T lim = ri + rmax[j];
                    if (dx * dx + dy * dy <= lim * lim) {
                        n += 1;
                        if (n <= capv) out[n - 1] = j + 1;
                    }
                }
            }
        return n;
    }

    // src/neighbors.jl:223-242
    void rebuild_neighbors() {
        while (true) {
            int32_t nmax = 0;
#pragma omp parallel for schedule(static) reduction(max : nmax)
            for (int64_t i = 0; i < N; ++i) {
                count[i] = neighbor_body(i, &idx[(size_t)cap * i], cap);
                nmax = std::max(nmax, count[i]);
            }
            if (nmax <= cap) break;
            cap = 2 * nmax;
            idx.assign((size_t)cap * N, 0);
        }
        if (skin > 0) {
            x0 = x;
            y0 = y;
            rmax0 = rmax;
        }
        valid = true;
        builds += 1;
    }

    // src/neighbors.jl:198-205
    bool skin_exceeded(int64_t i) const {
        T dx = minimum_image(x[i] - x0[i], Lx);
        T dy = minimum_image(y[i] - y0[i], Ly);
        T delta = std::sqrt(dx * dx + dy * dy) + std::max(T(0), rmax[i] - rmax0[i]);
        return T(2) * delta > skin;
    }

    // src/simulation.jl:132-142
    fcc_status update_neighbors(bool force) override {
        if (!force && valid && skin > 0) {
            bool flag = status[0] != 0;
            for (int64_t i = 0; i < N && !flag; ++i) flag = skin_exceeded(i);
            if (flag) status[0] = 1;
            if (status[0] == 0) return FCC_OK;
        }
        update_celllist();
        rebuild_neighbors();
        status[0] = status[1] = status[2] = 0;
        return FCC_OK;
    }

    // ---------------------------------------------------- gradients -------
    // src/gradients.jl:47-64 (reset!) when there are no body terms
    void reset_body(int64_t i) {
        for (int k = 0; k < nth; ++k) {
            GR[k + (size_t)nth * i] = 0;
            GD[k + (size_t)nth * i] = 0;
            GDD[k + (size_t)nth * i] = 0;
        }
        gx[i] = gy[i] = gth[i] = 0;
        Ebody[i] = 0;
    }

    // src/gradients.jl:70-98, 113-128 with Tension / PerimeterElasticity
    // (src/energies/body_terms.jl:8-34): q = sqrt(R^2 + R'^2), J = (R/q, R'/q, 0)
    void body_terms_body(int64_t i) {
        reset_body(i);
        if (body_terms.empty()) return;
        const T* r = &R[(size_t)nth * i];
        const T* r1 = &dR[(size_t)nth * i];
        T* gr = &GR[(size_t)nth * i];
        T* gd = &GD[(size_t)nth * i];
        T* gdd = &GDD[(size_t)nth * i];
        std::vector<T> energies(body_terms.size(), T(0));
        const T* r2 = &ddR[(size_t)nth * i];
        for (size_t q = 0; q < body_terms.size(); ++q) {
            const Term<T>& tm = body_terms[q];
            if (!tm.applies(type[i])) continue;
            if (tm.kind == FCC_USER_BODY) {  // src/gradients.jl:70-98 with the term's own q, F
                const int M = fcc_user::body_M(tm.user);
                T Q[fcc_user::MAX_M] = {}, qk[fcc_user::MAX_M], dF[fcc_user::MAX_M], dq[fcc_user::MAX_M][3];
                for (int k = 0; k < nth; ++k) {
                    fcc_user::body_q<T>(tm.user, r[k], r1[k], r2[k], tm.a, tm.b, qk);
                    for (int j = 0; j < M; ++j) Q[j] += qk[j];
                }
                for (int j = 0; j < M; ++j) Q[j] *= dphi;
                fcc_user::body_dF<T>(tm.user, Q, R0[i], type[i], tm.a, tm.b, dF);
                for (int k = 0; k < nth; ++k) {
                    fcc_user::body_dq<T>(tm.user, r[k], r1[k], r2[k], tm.a, tm.b, dq);
                    for (int j = 0; j < M; ++j) {
                        const T w = dF[j] * dphi;
                        gr[k] += dq[j][0] * w;
                        gd[k] += dq[j][1] * w;
                        gdd[k] += dq[j][2] * w;
                    }
                }
                energies[q] = fcc_user::body_F<T>(tm.user, Q, R0[i], type[i], tm.a, tm.b);
                continue;
            }
            T Q = std::sqrt(r[0] * r[0] + r1[0] * r1[0]);
            for (int k = 1; k < nth; ++k) Q += std::sqrt(r[k] * r[k] + r1[k] * r1[k]);
            Q *= dphi;
            T dF, E;
            if (tm.kind == FCC_TENSION) {
                dF = tm.a;
                E = tm.a * Q;
            } else {  // PerimeterElasticity: E = λ (Q - p0 √π R0)^2
                T l0 = (tm.b * std::sqrt(T(M_PI))) * R0[i];
                dF = tm.a * (T(2) * (Q - l0));
                E = tm.a * ((Q - l0) * (Q - l0));
            }
            T w = dF * dphi;
            for (int k = 0; k < nth; ++k) {
                T s = std::sqrt(r[k] * r[k] + r1[k] * r1[k]);
                gr[k] += (r[k] / s) * w;
                gd[k] += (r1[k] / s) * w;
                gdd[k] += T(0) * w;
            }
            energies[q] = E;
        }
        T acc = 0;  // e1 + (e2 + (... + 0))
        for (size_t q = body_terms.size(); q-- > 0;) acc = energies[q] + acc;
        Ebody[i] = acc;
    }

    // src/energies/contact.jl:267-293
    T pressure_sum(T d, int32_t ti, int32_t tj, bool rel) const {
        T acc = 0;
        for (size_t q = contact_terms.size(); q-- > 0;) {
            const Term<T>& tm = contact_terms[q];
            T g = 0;
            if (tm.applies(ti)) {
                if (tm.kind == FCC_OVERLAP) {
                    // a 1 x 1 table (scalar coupling) applies to every type pair
                    int nJ = tm.nJ;
                    size_t ij = nJ == 1 ? 0 : (size_t)(ti - 1) + (size_t)nJ * (tj - 1);
                    T J = rel ? tm.Jrel[ij] : tm.J[ij];
                    g = d >= 0 ? J : T(0);
                } else if (tm.kind == FCC_USER_CONTACT) {
                    g = fcc_user::contact_g<T>(tm.user, d, ti, tj, rel, tm.a, tm.b);
                } else {
                    g = d > 0 ? tm.a * d : T(0);
                }
            }
            acc = g + acc;
        }
        return acc;
    }

    // src/energies/contact.jl:300-324 and the fused node kernel :391-429
    void contact_body(int64_t i, int64_t& tests, int64_t& hits) {
        T fx = 0, fy = 0, tt = 0;
        const T* r = &R[(size_t)nth * i];
        const T* r1 = &dR[(size_t)nth * i];
        int32_t ti = type[i], pi_ = parent[i];
        double md = INFINITY;
        for (int k = 0; k < nth; ++k) {
            T c = cs[2 * k], s = cs[2 * k + 1];
            T ux = x[i] + r[k] * c;
            T uy = y[i] + r[k] * s;
            T p = 0;
            for (int32_t q = 0; q < count[i]; ++q) {
                int64_t j = idx[(size_t)q + (size_t)cap * i] - 1;
                T dx = minimum_image(ux - x[j], Lx);
                T dy = minimum_image(uy - y[j], Ly);
                T dist2 = dx * dx + dy * dy;
                T lim = rmax[j] + contact_range_T;
                ++tests;
                if (dist2 > lim * lim) continue;
                ++hits;
                T dist = std::sqrt(dist2);
                T cps = dist > 0 ? dx / dist : T(1);
                T sps = dist > 0 ? dy / dist : T(0);
                T d = contour_radius_dir(j, cps, sps) - dist;
                md = std::min(md, std::fabs((double)d));
                p += pressure_sum(d, ti, type[j], pi_ == parent[j]);
            }
            P[k + (size_t)nth * i] = p;
            T pw = p * dphi;
            GR[k + (size_t)nth * i] += pw * r[k];
            // node k's force/torque terms are summed in node order, as the
            // fused node kernel's final loop over fbuf does (contact.jl:416-424)
            fx += pw * (r[k] * c + r1[k] * s);
            fy += pw * (r[k] * s - r1[k] * c);
            tt += (-pw * r[k]) * r1[k];
        }
        gx[i] += fx;
        gy[i] += fy;
        gth[i] += tt;
        mind[i] = md;
    }

    // src/energies/bonds.jl:18-29, 77-111
    void bond_body(int64_t i) {
        T g0 = 0, g1 = 0;
        for (int32_t q = 0; q < bcount[i]; ++q) {
            int64_t j = bidx[(size_t)q + (size_t)bcap * i] - 1;
            T d0 = minimum_image(x[i] - x[j], Lx);
            T d1 = minimum_image(y[i] - y[j], Ly);
            T a0 = 0, a1 = 0;  // g1 + (g2 + (... + 0))
            for (size_t u = bond_terms.size(); u-- > 0;) {
                const Term<T>& tm = bond_terms[u];
                T h0 = 0, h1 = 0;
                if (tm.applies(type[i]) && tm.applies(type[j])) {
                    if (tm.kind == FCC_USER_BOND) {
                        fcc_user::bond_grad<T>(tm.user, d0, d1, type[i], type[j], tm.a, tm.b, h0, h1);
                    } else {
                        T rr = std::sqrt(d0 * d0 + d1 * d1);
                        T f = rr > 0 ? tm.a * (T(1) - tm.b / rr) : (tm.b == 0 ? tm.a : T(0));
                        h0 = f * d0;
                        h1 = f * d1;
                    }
                }
                a0 = h0 + a0;
                a1 = h1 + a1;
            }
            g0 += a0;
            g1 += a1;
        }
        gx[i] += g0;
        gy[i] += g1;
    }

    // src/gradients.jl:347-362
    void body_frame(int64_t i, T thi, T r0) {
        const T* gl = &glab[(size_t)nc * i];
        const T* c = &coef[(size_t)nc * i];
        T* gc = &gcoef[(size_t)nc * i];
        T ga0 = r0 * gl[0];
        T a0 = c[0];
        for (int m = 1; m <= K; ++m) {
            int n = m + 1;
            T ga = r0 * gl[m];
            T gb = r0 * gl[K + m];
            T arg = (T)n * thi;
            T s = std::sin(arg), co = std::cos(arg);
            T a = c[m], b = c[K + m];
            gc[m] = ga * co + gb * s - ga0 * a / (T(2) * a0);
            gc[K + m] = -ga * s + gb * co - ga0 * b / (T(2) * a0);
        }
        gc[0] = ga0;
    }

    // src/gradients.jl:374-386 (CPU: three products, glab = C'GR + D'GD + DD'GDD)
    void pullback_body(int64_t i) {
        const T* gr = &GR[(size_t)nth * i];
        const T* gd = &GD[(size_t)nth * i];
        const T* gdd = &GDD[(size_t)nth * i];
        T* gl = &glab[(size_t)nc * i];
        for (int c = 0; c < nc; ++c) {
            T a = 0, b = 0, e = 0;
            for (int k = 0; k < nth; ++k) a += C[k + (size_t)nth * c] * gr[k];
            for (int k = 0; k < nth; ++k) b += D[k + (size_t)nth * c] * gd[k];
            for (int k = 0; k < nth; ++k) e += DD[k + (size_t)nth * c] * gdd[k];
            gl[c] = (a + b) + e;
        }
    }

    // src/simulation.jl:150-158
    void gradients(bool frame) {
        int64_t tests = 0, hits = 0;
        bool contacts = !contact_terms.empty();
        bool bonds = !bond_terms.empty() && N > 0;
#pragma omp parallel for schedule(static) reduction(+ : tests, hits)
        for (int64_t i = 0; i < N; ++i) {
            body_terms_body(i);
        }
        if (contacts) {
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tests, hits)
            for (int64_t i = 0; i < N; ++i) contact_body(i, tests, hits);
        }
        if (bonds) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) bond_body(i);
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            pullback_body(i);
            if (frame) body_frame(i, th[i], R0[i]);
        }
        n_tests = tests;
        n_hits = hits;
    }

    fcc_status compute_gradients() override {
        gradients(true);
        return FCC_OK;
    }

    // ---------------------------------------------------- dynamics --------
    // src/dynamics.jl:84-99
    void substrate_displacement(int64_t i, T& ox, T& oy) const {
        const BodyTypeT<T>& p = types[type[i] - 1];
        T fx = gx[i], fy = gy[i];
        for (int32_t q = 0; q < ccount[i]; ++q) {
            int64_t k = cidx[(size_t)q + (size_t)ccap * i] - 1;
            if (types[type[k] - 1].parent_drag) {
                fx += gx[k];
                fy += gy[k];
            }
        }
        T s = std::sin(th[i]), c = std::cos(th[i]);
        T st = std::sqrt(T(2) * p.Dt * dt);
        T xi1, xi2;
        philox_pair<T>(k0, k1, (uint64_t)(i + 1), (uint64_t)clock, 0, xi1, xi2);
        ox = dt * (p.v0 * c - p.mur * fx) + st * xi1;
        oy = dt * (p.v0 * s - p.mur * fy) + st * xi2;
    }

    // src/dynamics.jl:128-147
    void displacement_body(int64_t i) {
        const BodyTypeT<T>& p = types[type[i] - 1];
        T* dp = &disp[3 * (size_t)i];
        if (p.parent_drag) {
            int64_t c = parent[i] - 1;
            T ux, uy;
            substrate_displacement(c, ux, uy);
            T s = std::sin(th[i]), co = std::cos(th[i]);
            T st = std::sqrt(T(2) * p.Dt * dt);
            T xi1, xi2;
            philox_pair<T>(k0, k1, (uint64_t)(i + 1), (uint64_t)clock, 0, xi1, xi2);
            dp[0] = ux + dt * (p.v0 * co - p.mur * gx[i]) + st * xi1;
            dp[1] = uy + dt * (p.v0 * s - p.mur * gy[i]) + st * xi2;
        } else {
            substrate_displacement(i, dp[0], dp[1]);
        }
        T z1, z2;
        philox_pair<T>(k0, k1, (uint64_t)(i + 1), (uint64_t)clock, 1, z1, z2);
        dp[2] = std::sqrt(T(2) * p.Dr * dt) * z1;
    }

    // src/dynamics.jl:180-203 (frame = true, lab = geom, skin check)
    void update_body(int64_t i, bool check_skin, int& flag) {
        const BodyTypeT<T>& p = types[type[i] - 1];
        body_frame(i, th[i], R0[i]);
        T thn = th[i] - (dt * p.muth) * gth[i] + disp[3 * (size_t)i + 2];
        th[i] = thn;
        T* c = &coef[(size_t)nc * i];
        const T* gc = &gcoef[(size_t)nc * i];
        for (int r = 1; r < nc; ++r) c[r] -= (dt * p.muab) * gc[r];
        enforce_shape(i);
        int32_t sx, sy;
        T xw = wrap(x[i] + disp[3 * (size_t)i], Lx, sx);
        T yw = wrap(y[i] + disp[3 * (size_t)i + 1], Ly, sy);
        x[i] = xw;
        y[i] = yw;
        imgx[i] += sx;
        imgy[i] += sy;
        lab_frame(i, thn, R0[i]);
        if (check_skin && skin_exceeded(i)) flag = 1;
    }

    // src/simulation.jl:181-191 (advance!) and :165-173 (step!)
    fcc_status step(int64_t n) override {
        for (int64_t s = 0; s < n; ++s) {
            bool contacts = !contact_terms.empty();
            if (contacts) update_neighbors(false);
            gradients(false);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) displacement_body(i);
            bool check = contacts && valid && skin > 0;
            int flag = 0;
#pragma omp parallel for schedule(static) reduction(max : flag)
            for (int64_t i = 0; i < N; ++i) update_body(i, check, flag);
            if (flag) status[0] = 1;
            clock += 1;
            synthesize();
            t += dt;
            stepno += 1;
        }
        return FCC_OK;
    }

    // ---------------------------------------------------- accessors -------
    fcc_status get_state(fcc_bodies_host* o, int64_t* clk, double* tt, int64_t* stp) override {
        if (o) {
            if (o->n != N || o->ncoef != nc) return fail(FCC_ERR_DIMENSION, "state buffers do not match the simulation");
            for (int64_t i = 0; i < N; ++i) {
                if (o->x) o->x[i] = x[i];
                if (o->y) o->y[i] = y[i];
                if (o->theta) o->theta[i] = th[i];
                if (o->imgx) o->imgx[i] = imgx[i];
                if (o->imgy) o->imgy[i] = imgy[i];
                if (o->R0) o->R0[i] = R0[i];
                if (o->type) o->type[i] = type[i];
                if (o->parent) o->parent[i] = parent[i];
            }
            if (o->coef) for (size_t q = 0; q < (size_t)nc * N; ++q) o->coef[q] = coef[q];
        }
        if (clk) *clk = clock;
        if (tt) *tt = (double)t;
        if (stp) *stp = stepno;
        return FCC_OK;
    }

    fcc_status set_state(const fcc_bodies_host* in, int64_t clk) override {
        if (!in || in->n != N || in->ncoef != nc) return fail(FCC_ERR_DIMENSION, "state buffers do not match the simulation");
        for (int64_t i = 0; i < N; ++i) {
            if (in->x) x[i] = (T)in->x[i];
            if (in->y) y[i] = (T)in->y[i];
            if (in->theta) th[i] = (T)in->theta[i];
            if (in->imgx) imgx[i] = in->imgx[i];
            if (in->imgy) imgy[i] = in->imgy[i];
        }
        if (in->coef) for (size_t q = 0; q < (size_t)nc * N; ++q) coef[q] = (T)in->coef[q];
        if (clk >= 0) clock = clk;
        enforce_all();
        update_geometry();
        valid = false;
        status[0] = status[1] = status[2] = 0;
        return FCC_OK;
    }

    fcc_status set_dt(double v) override {
        dt = (T)v;
        return FCC_OK;
    }

    template <class V> static void put(double* dst, const V& src) {
        if (!dst) return;
        for (size_t q = 0; q < src.size(); ++q) dst[q] = (double)src[q];
    }

    fcc_status get_gradients(const fcc_gradients_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        put(o->GR, GR); put(o->GD, GD); put(o->GDD, GDD); put(o->P, P);
        put(o->gx, gx); put(o->gy, gy); put(o->gtheta, gth);
        put(o->glab, glab); put(o->gcoef, gcoef); put(o->Ebody, Ebody);
        return FCC_OK;
    }

    fcc_status get_geometry(const fcc_geometry_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        put(o->lab, lab); put(o->labR0, labR0); put(o->R, R); put(o->dR, dR); put(o->ddR, ddR); put(o->rmax, rmax);
        return FCC_OK;
    }

    fcc_status neighbor_dims(int32_t* cx, int32_t* cy, int32_t* cp, int64_t* b, int32_t* v) override {
        if (cx) *cx = ncx;
        if (cy) *cy = ncy;
        if (cp) *cp = cap;
        if (b) *b = builds;
        if (v) *v = valid ? 1 : 0;
        return FCC_OK;
    }

    fcc_status get_neighbors(const fcc_neighbors_host* o) override {
        if (!o) return fail(FCC_ERR_ARGUMENT, "null argument");
        if (o->cellid) std::copy(cellid.begin(), cellid.end(), o->cellid);
        if (o->perm) std::copy(perm.begin(), perm.end(), o->perm);
        if (o->start) std::copy(start.begin(), start.end(), o->start);
        if (o->stop) std::copy(stop.begin(), stop.end(), o->stop);
        if (o->idx) std::copy(idx.begin(), idx.end(), o->idx);
        if (o->count) std::copy(count.begin(), count.end(), o->count);
        return FCC_OK;
    }

    // src/observables.jl:7-18; which: 0 perimeters, 1 areas, 2 shape index, 3 protrusion
    fcc_status observable(int which, int32_t typ, double* out, int64_t* cnt) override {
        int64_t w = 0;
        for (int64_t i = 0; i < N; ++i) {
            if (typ != 0 && type[i] != typ) continue;
            const T* r = &R[(size_t)nth * i];
            const T* r1 = &dR[(size_t)nth * i];
            double v;
            if (which == 3) {
                v = protrusion_body(i);
            } else {
                T per = 0, ar = 0;
                for (int k = 0; k < nth; ++k) {
                    per += std::sqrt(r[k] * r[k] + r1[k] * r1[k]);
                    ar += r[k] * r[k];
                }
                per *= dphi;
                ar *= dphi / T(2);
                v = which == 0 ? (double)per : which == 1 ? (double)ar : (double)(per / std::sqrt(ar));
            }
            if (out) out[w] = v;
            ++w;
        }
        if (cnt) *cnt = w;
        return FCC_OK;
    }

    // src/observables.jl:232-252 (one body)
    double protrusion_body(int64_t i) const {
        int64_t c = parent[i] - 1;
        if (c == i) return NAN;
        T p = -INFINITY;
        for (int k = 0; k < nth; ++k) {
            T phi = (T)k * dphi;
            T s = std::sin(phi), co = std::cos(phi);
            T dx = minimum_image(x[i] + R[k + (size_t)nth * i] * co - x[c], Lx);
            T dy = minimum_image(y[i] + R[k + (size_t)nth * i] * s - y[c], Ly);
            T psi = std::atan2(dy, dx);
            T rc = contour_radius_dir(c, std::cos(psi), std::sin(psi));
            p = std::max(p, std::hypot(dx, dy) - rc);
        }
        return (double)p;
    }

    fcc_status body_energy(double* out) override {
        T acc = 0;
        for (int64_t i = 0; i < N; ++i) acc += Ebody[i];
        *out = (double)acc;
        return FCC_OK;
    }

    fcc_status counters(int64_t* tests, int64_t* hits, double* md) override {
        if (tests) *tests = n_tests;
        if (hits) *hits = n_hits;
        if (md) std::copy(mind.begin(), mind.end(), md);
        return FCC_OK;
    }
};

// Standalone cell-list + neighbour build on caller arrays.
template <class T>
fcc_status build_neighbors_t(int64_t n, const double* xd, const double* yd, const double* rd, double Lx64, double Ly64,
                             double cutoff, double range64, int32_t cap, int32_t* cellid, int32_t* perm,
                             int32_t* start, int32_t* stop, int32_t* idx, int32_t* count) {
    Sim<T> s;
    s.N = n;
    s.Lx = (T)Lx64;
    s.Ly = (T)Ly64;
    auto ncells = [&](T L) { int64_t m = (int64_t)std::floor((double)L / cutoff); return (int32_t)(m >= 3 ? m : 1); };
    s.ncx = ncells(s.Lx);
    s.ncy = ncells(s.Ly);
    s.wx = s.Lx / (T)s.ncx;
    s.wy = s.Ly / (T)s.ncy;
    Sim<T>::to_T(s.x, xd, n);
    Sim<T>::to_T(s.y, yd, n);
    Sim<T>::to_T(s.rmax, rd, n);
    s.cellid.assign(n, 0);
    s.perm.assign(n, 0);
    s.start.assign((size_t)s.ncx * s.ncy, 0);
    s.stop.assign((size_t)s.ncx * s.ncy, 0);
    s.range_T = (T)range64;
    s.update_celllist();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) count[i] = s.neighbor_body(i, &idx[(size_t)cap * i], cap);
    std::copy(s.cellid.begin(), s.cellid.end(), cellid);
    std::copy(s.perm.begin(), s.perm.end(), perm);
    std::copy(s.start.begin(), s.start.end(), start);
    std::copy(s.stop.begin(), s.stop.end(), stop);
    return FCC_OK;
}

}  // namespace

struct fcco_sim {
    std::unique_ptr<SimBase> impl;
};

extern "C" {

fcc_status fcco_create(const fcc_params* params, const fcc_bodies_host* bodies, fcco_sim** out) {
    if (!out) return fail(FCC_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!params) return fail(FCC_ERR_ARGUMENT, "null params");
    std::unique_ptr<fcco_sim> h(new fcco_sim);
    fcc_status st;
    if (params->precision == 64) {
        auto s = std::make_unique<Sim<double>>();
        st = s->init(params, bodies);
        h->impl = std::move(s);
    } else if (params->precision == 32) {
        auto s = std::make_unique<Sim<float>>();
        st = s->init(params, bodies);
        h->impl = std::move(s);
    } else {
        return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
    }
    if (st != FCC_OK) return st;
    *out = h.release();
    return FCC_OK;
}

fcc_status fcco_destroy(fcco_sim* sim) {
    delete sim;
    return FCC_OK;
}

#define ORACLE_CALL(expr)                                              \
    do {                                                               \
        if (!sim) return fail(FCC_ERR_ARGUMENT, "null simulation");    \
        return sim->impl->expr;                                        \
    } while (0)

fcc_status fcco_step(fcco_sim* sim, int64_t n) { ORACLE_CALL(step(n)); }
fcc_status fcco_update_neighbors(fcco_sim* sim, int32_t force) { ORACLE_CALL(update_neighbors(force != 0)); }
fcc_status fcco_compute_gradients(fcco_sim* sim) { ORACLE_CALL(compute_gradients()); }
fcc_status fcco_get_state(fcco_sim* sim, fcc_bodies_host* out, int64_t* clock, double* t, int64_t* step) { ORACLE_CALL(get_state(out, clock, t, step)); }
fcc_status fcco_set_state(fcco_sim* sim, const fcc_bodies_host* in, int64_t clock) { ORACLE_CALL(set_state(in, clock)); }
fcc_status fcco_set_dt(fcco_sim* sim, double dt) { ORACLE_CALL(set_dt(dt)); }
fcc_status fcco_get_gradients(fcco_sim* sim, const fcc_gradients_host* out) { ORACLE_CALL(get_gradients(out)); }
fcc_status fcco_get_geometry(fcco_sim* sim, const fcc_geometry_host* out) { ORACLE_CALL(get_geometry(out)); }
fcc_status fcco_neighbor_dims(fcco_sim* sim, int32_t* ncx, int32_t* ncy, int32_t* cap, int64_t* builds, int32_t* valid) { ORACLE_CALL(neighbor_dims(ncx, ncy, cap, builds, valid)); }
fcc_status fcco_get_neighbors(fcco_sim* sim, const fcc_neighbors_host* out) { ORACLE_CALL(get_neighbors(out)); }
fcc_status fcco_perimeters(fcco_sim* sim, int32_t type, double* out, int64_t* count) { ORACLE_CALL(observable(0, type, out, count)); }
fcc_status fcco_areas(fcco_sim* sim, int32_t type, double* out, int64_t* count) { ORACLE_CALL(observable(1, type, out, count)); }
fcc_status fcco_shape_index(fcco_sim* sim, int32_t type, double* out, int64_t* count) { ORACLE_CALL(observable(2, type, out, count)); }
fcc_status fcco_protrusion(fcco_sim* sim, int32_t type, double* out, int64_t* count) { ORACLE_CALL(observable(3, type, out, count)); }
fcc_status fcco_body_energy(fcco_sim* sim, double* out) { ORACLE_CALL(body_energy(out)); }
fcc_status fcco_contact_counters(fcco_sim* sim, int64_t* tests, int64_t* hits, double* mind) { ORACLE_CALL(counters(tests, hits, mind)); }

void fcco_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox(c, key[0], key[1]);
    for (int q = 0; q < 4; ++q) out[q] = c[q];
}

// src/random.jl:59-67, 113-121 (first three normals of philox_normals)
fcc_status fcco_philox_noise(uint64_t seed, uint64_t draw, int64_t nbodies, int32_t precision, double* out) {
    uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
    if (precision != 32 && precision != 64) return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nbodies; ++i) {
        if (precision == 64) {
            double z1, z2, z3, z4;
            philox_pair<double>(k0, k1, (uint64_t)(i + 1), draw, 0, z1, z2);
            philox_pair<double>(k0, k1, (uint64_t)(i + 1), draw, 1, z3, z4);
            out[3 * i] = z1; out[3 * i + 1] = z2; out[3 * i + 2] = z3;
        } else {
            float z1, z2, z3, z4;
            philox_pair<float>(k0, k1, (uint64_t)(i + 1), draw, 0, z1, z2);
            philox_pair<float>(k0, k1, (uint64_t)(i + 1), draw, 1, z3, z4);
            out[3 * i] = z1; out[3 * i + 1] = z2; out[3 * i + 2] = z3;
        }
    }
    return FCC_OK;
}

fcc_status fcco_build_neighbors(int32_t precision, int64_t n, const double* x, const double* y, const double* rmax,
                                double Lx, double Ly, double cutoff, double range, int32_t cap, int32_t* cellid,
                                int32_t* perm, int32_t* start, int32_t* stop, int32_t* idx, int32_t* count) {
    if (precision == 64)
        return build_neighbors_t<double>(n, x, y, rmax, Lx, Ly, cutoff, range, cap, cellid, perm, start, stop, idx, count);
    if (precision == 32)
        return build_neighbors_t<float>(n, x, y, rmax, Lx, Ly, cutoff, range, cap, cellid, perm, start, stop, idx, count);
    return fail(FCC_ERR_ARGUMENT, "precision must be 32 or 64");
}

int32_t fcco_set_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    else omp_set_num_threads(omp_get_num_procs());
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

const char* fcco_last_error(void) { return g_err.c_str(); }

}  // extern "C"
