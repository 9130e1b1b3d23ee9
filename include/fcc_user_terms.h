/*
 * fcc_user_terms.h — user-defined energy terms, compiled into the library.
 *
 * The reference lets users add energy terms by defining Julia methods for a
 * new struct (src/energies/interface.jl:27-106, README.md:103-160):
 *   BodyTerm     contour_integrands(term, R, R', R'') -> q_j,
 *                energy(term, Q, body) -> F(Q)   (default sum(Q)),
 *                derivatives by automatic differentiation or by hand;
 *   ContactTerm  pressure(term, d, t_i, t_j, related) -> g(d),
 *                interaction_range(term);
 *   BondTerm     bond_energy(term, Delta, t_i, t_j) (+ bond_gradient).
 * Julia closures cannot cross a C ABI, so here a user term is a C++ functor
 * with the same methods (derivatives written out) compiled into the library
 * and into the CPU oracle: add a struct below, list it in its table at the
 * end of the file, rebuild, and select it with fcc_term.kind =
 * FCC_USER_BODY / FCC_USER_CONTACT / FCC_USER_BOND, fcc_term.user = its
 * index and parameters fcc_term.a, fcc_term.b (converted to the simulation
 * precision like every parameter).  OnTypes (fcc_term.ntypes_on) applies.
 *
 * Every method is a template on the float type T and must be
 * allocation-free: it runs inside the CUDA kernels (and the oracle).
 *
 * Body terms:   static constexpr int M;             integrals, 1 <= M <= 2
 *   q (R, dR, ddR, a, b, out[M])                    integrands q_j
 *   dq(R, dR, ddR, a, b, out[M][3])                 dq_j / d(R, R', R'')
 *   F (Q[M], R0, type, a, b) -> E                   energy of the integrals
 *   dF(Q[M], R0, type, a, b, out[M])                dF / dQ_j
 * Contact terms:
 *   g(d, ti, tj, related, a, b) -> energy density at penetration depth d
 *                                  (d > 0 inside the neighbour; types 1-based)
 *   range(a, b)                 -> largest |d|, d < 0, at which g != 0
 * Bond terms:
 *   grad(dx, dy, ti, tj, a, b, gx, gy): dE/dDelta, Delta = r_i - r_j
 *   (E symmetric under Delta -> -Delta with swapped types).
 */
#ifndef FCC_USER_TERMS_H
#define FCC_USER_TERMS_H

#include <math.h>

#if defined(__CUDACC__)
#define FCC_HD __host__ __device__ __forceinline__
#else
#define FCC_HD inline
#endif

namespace fcc_user {

/* Bending energy kappa * contour integral of c^2 ds, kappa = a: the
 * reference README's example of an integrand-only body term
 * (README.md:118-121); it needs R''. */
struct Bending {
    static constexpr int M = 1;
    template <class T>
    FCC_HD static void q(T R, T dR, T ddR, T a, T, T* out) {
        const T S = R * R + dR * dR, N = R * R + T(2) * dR * dR - R * ddR;
        out[0] = a * N * N / (S * S * sqrt(S));
    }
    template <class T>
    FCC_HD static void dq(T R, T dR, T ddR, T a, T, T (*out)[3]) {
        // q = a N^2 S^(-5/2):  dq/dx = a N S^(-7/2) (2 S dN/dx - 5/2 N dS/dx)
        const T S = R * R + dR * dR, N = R * R + T(2) * dR * dR - R * ddR;
        const T f = a * N / (S * S * S * sqrt(S));
        out[0][0] = f * (T(2) * S * (T(2) * R - ddR) - T(5) * N * R);
        out[0][1] = f * (T(8) * S * dR - T(5) * N * dR);
        out[0][2] = f * (-T(2) * S * R);
    }
    template <class T>
    FCC_HD static T F(const T* Q, T, int, T, T) { return Q[0]; }
    template <class T>
    FCC_HD static void dF(const T*, T, int, T, T, T* out) { out[0] = T(1); }
};

/* Shape-index elasticity k (P / sqrt(A) - p0)^2 with k = a, p0 = b: a
 * nonlinear energy of two integrals, the perimeter P = contour integral of
 * sqrt(R^2 + R'^2) dphi and the area A = contour integral of R^2 / 2 dphi
 * (the integrands of src/energies/interface.jl:38-42; P / sqrt(A) is the
 * shape index of src/observables.jl:18). */
struct ShapeIndexElasticity {
    static constexpr int M = 2;
    template <class T>
    FCC_HD static void q(T R, T dR, T, T, T, T* out) {
        out[0] = sqrt(R * R + dR * dR);
        out[1] = R * R / T(2);
    }
    template <class T>
    FCC_HD static void dq(T R, T dR, T, T, T, T (*out)[3]) {
        const T s = sqrt(R * R + dR * dR);
        out[0][0] = R / s;
        out[0][1] = dR / s;
        out[0][2] = T(0);
        out[1][0] = R;
        out[1][1] = T(0);
        out[1][2] = T(0);
    }
    template <class T>
    FCC_HD static T F(const T* Q, T, int, T a, T b) {
        const T e = Q[0] / sqrt(Q[1]) - b;
        return a * e * e;
    }
    template <class T>
    FCC_HD static void dF(const T* Q, T, int, T a, T b, T* out) {
        const T sa = sqrt(Q[1]);
        const T e = Q[0] / sa - b;
        out[0] = a * (T(2) * e) / sa;
        out[1] = -a * (T(2) * e) * Q[0] / (T(2) * Q[1] * sa);
    }
};

/* Short-range adhesion: energy density -eps in a band of width w outside the
 * neighbour's contour (-w < d < 0), zero elsewhere; eps = a, w = b.  Its
 * interaction range w widens the neighbour lists (interaction_range,
 * src/energies/interface.jl:96). */
struct Adhesion {
    template <class T>
    FCC_HD static T g(T d, int, int, bool, T a, T b) { return (d < T(0) && d > -b) ? -a : T(0); }
    template <class T>
    FCC_HD static T range(T, T b) { return b; }
};

/* Quartic bond E = k |Delta|^4 / 4, k = a. */
struct QuarticBond {
    template <class T>
    FCC_HD static void grad(T dx, T dy, int, int, T a, T, T& gx, T& gy) {
        const T r2 = dx * dx + dy * dy;
        gx = a * r2 * dx;
        gy = a * r2 * dy;
    }
};

/* ----------------------------------------------------------- the tables --
 * X(index, struct): fcc_term.user selects the entry of the term's kind. */
#define FCC_USER_BODY_TERMS(X) X(0, Bending) X(1, ShapeIndexElasticity)
#define FCC_USER_CONTACT_TERMS(X) X(0, Adhesion)
#define FCC_USER_BOND_TERMS(X) X(0, QuarticBond)

/* Dispatch by index (generated from the tables). */
#define FCC_UT_COUNT(i, S) +1
constexpr int n_body = 0 FCC_USER_BODY_TERMS(FCC_UT_COUNT);
constexpr int n_contact = 0 FCC_USER_CONTACT_TERMS(FCC_UT_COUNT);
constexpr int n_bond = 0 FCC_USER_BOND_TERMS(FCC_UT_COUNT);
#undef FCC_UT_COUNT
constexpr int MAX_M = 2;  /* integrals per body term */

FCC_HD int body_M(int id) {
#define FCC_UT_CASE(i, S) \
    case i:               \
        return S::M;
    switch (id) { FCC_USER_BODY_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
    return 0;
}
template <class T>
FCC_HD void body_q(int id, T R, T dR, T ddR, T a, T b, T* out) {
#define FCC_UT_CASE(i, S)             \
    case i:                           \
        S::q(R, dR, ddR, a, b, out); \
        return;
    switch (id) { FCC_USER_BODY_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
}
template <class T>
FCC_HD void body_dq(int id, T R, T dR, T ddR, T a, T b, T (*out)[3]) {
#define FCC_UT_CASE(i, S)              \
    case i:                            \
        S::dq(R, dR, ddR, a, b, out); \
        return;
    switch (id) { FCC_USER_BODY_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
}
template <class T>
FCC_HD T body_F(int id, const T* Q, T R0, int type, T a, T b) {
#define FCC_UT_CASE(i, S) \
    case i:               \
        return S::F(Q, R0, type, a, b);
    switch (id) { FCC_USER_BODY_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
    return T(0);
}
template <class T>
FCC_HD void body_dF(int id, const T* Q, T R0, int type, T a, T b, T* out) {
#define FCC_UT_CASE(i, S)                 \
    case i:                               \
        S::dF(Q, R0, type, a, b, out);   \
        return;
    switch (id) { FCC_USER_BODY_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
}
template <class T>
FCC_HD T contact_g(int id, T d, int ti, int tj, bool related, T a, T b) {
#define FCC_UT_CASE(i, S) \
    case i:               \
        return S::g(d, ti, tj, related, a, b);
    switch (id) { FCC_USER_CONTACT_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
    return T(0);
}
template <class T>
FCC_HD T contact_range(int id, T a, T b) {
#define FCC_UT_CASE(i, S) \
    case i:               \
        return S::range(a, b);
    switch (id) { FCC_USER_CONTACT_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
    return T(0);
}
template <class T>
FCC_HD void bond_grad(int id, T dx, T dy, int ti, int tj, T a, T b, T& gx, T& gy) {
    gx = gy = T(0);
#define FCC_UT_CASE(i, S)                          \
    case i:                                        \
        S::grad(dx, dy, ti, tj, a, b, gx, gy);    \
        return;
    switch (id) { FCC_USER_BOND_TERMS(FCC_UT_CASE) }
#undef FCC_UT_CASE
}

}  // namespace fcc_user

#endif /* FCC_USER_TERMS_H */
