// fcc_kernels.cuh — sm_100a kernels of the Fourier contour cell time step.
//
// One persistent cooperative kernel runs whole steps (k_step):
//   [rebuild prologue, only when a simulation needs it: counting-sort cell
//    list + neighbour list, five phases separated by grid barriers]
//   forces + Euler-Maruyama update fused per body (no parent drag), or
//   forces | barrier | displacement + update (parent drag: a body's motion
//   needs its children's forces)
//   grid barrier that ticks the clocks and decides the next rebuild (the
//   device-side form of update_neighbors!'s skin check): for a lone
//   simulation every block decides from the same arrival counter (flat
//   barrier), for a pool the last block to arrive decides and releases.
//
// Work mapping of the force evaluation: L lanes per body (L = 8 for nθ = 40),
// 32/L bodies per warp; lane l owns contour nodes k = l + L*s, s < S, so a
// body's nθ nodes are spread evenly and node quadratures are L-lane shuffle
// reductions.  Warp groups are the work units of a grid-stride loop.

#pragma once

#include <climits>

#include "fcc_device.cuh"
#include "../../include/fcc_user_terms.h"

namespace fcc {

// ---------------------------------------------------------- record access
__device__ __forceinline__ void load_rec(const float* p, float (&r)[RECW]) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int u = 0; u < RECW / 4; ++u) {
        float4 v = ldcg(q + u);
        r[4 * u] = v.x;
        r[4 * u + 1] = v.y;
        r[4 * u + 2] = v.z;
        r[4 * u + 3] = v.w;
    }
}
__device__ __forceinline__ void load_rec(const double* p, double (&r)[RECW]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int u = 0; u < RECW / 2; ++u) {
        double2 v = ldcg(q + u);
        r[2 * u] = v.x;
        r[2 * u + 1] = v.y;
    }
}
// x, y, rmax, w of a record
__device__ __forceinline__ void load_head(const float* p, float& x, float& y, float& rm, float& w) {
    float4 v = ldcg(reinterpret_cast<const float4*>(p));
    x = v.x, y = v.y, rm = v.z, w = v.w;
}
__device__ __forceinline__ void load_head(const double* p, double& x, double& y, double& rm, double& w) {
    double2 a = ldcg(reinterpret_cast<const double2*>(p));
    double2 b = ldcg(reinterpret_cast<const double2*>(p) + 1);
    x = a.x, y = a.y, rm = b.x, w = b.y;
}
// R0-scaled lab coefficients of a record (slots 4..22; slot 23 comes along)
__device__ __forceinline__ void load_lab(const float* p, float (&c)[20]) {
    const float4* q = reinterpret_cast<const float4*>(p + R_A0);
#pragma unroll
    for (int u = 0; u < 5; ++u) {
        float4 v = ldcg(q + u);
        c[4 * u] = v.x;
        c[4 * u + 1] = v.y;
        c[4 * u + 2] = v.z;
        c[4 * u + 3] = v.w;
    }
}
__device__ __forceinline__ void load_lab(const double* p, double (&c)[20]) {
    const double2* q = reinterpret_cast<const double2*>(p + R_A0);
#pragma unroll
    for (int u = 0; u < 10; ++u) {
        double2 v = ldcg(q + u);
        c[2 * u] = v.x;
        c[2 * u + 1] = v.y;
    }
}

// The current record buffer is rec[par], par = parity of the engine's step
// counter (all simulations of an engine advance together; a frozen one
// copies its records forward).
template <class T>
__device__ __forceinline__ const T* rec_cur(const DevPtrs<T>& d, int par) {
    return par ? d.rec1 : d.rec0;
}
template <class T>
__device__ __forceinline__ T* rec_next(const DevPtrs<T>& d, int par) {
    return par ? d.rec0 : d.rec1;
}
template <class T>
__device__ __forceinline__ T* rec_cur_mut(const DevPtrs<T>& d, int par) {
    return par ? d.rec1 : d.rec0;
}

// shared-memory vector loads of staged records
#ifndef FCC_LDS_ASM
#define FCC_LDS_ASM 0  // 1: explicit ld.shared (volatile asm); 0: plain vector load the compiler may schedule (measured 1.5% faster)
#endif
__device__ __forceinline__ float4 lds4(const float* p) {
#if FCC_LDS_ASM
    float4 v;
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
#else
    return *reinterpret_cast<const float4*>(p);
#endif
}
struct Double4 {
    double x, y, z, w;
};
__device__ __forceinline__ Double4 lds4(const double* p) { return Double4{p[0], p[1], p[2], p[3]}; }
__device__ __forceinline__ void lds_head(const float* p, float& x, float& y, float& rm, float& w) {
    const float4 v = lds4(p);
    x = v.x, y = v.y, rm = v.z, w = v.w;
}
__device__ __forceinline__ void lds_head(const double* p, double& x, double& y, double& rm, double& w) {
    x = p[R_X], y = p[R_Y], rm = p[R_RMAX], w = p[R_W];
}
__device__ __forceinline__ void lds_lab(const float* p, float (&c)[20]) {
#pragma unroll
    for (int u = 0; u < 5; ++u) {
        const float4 v = lds4(p + R_A0 + 4 * u);
        c[4 * u] = v.x, c[4 * u + 1] = v.y, c[4 * u + 2] = v.z, c[4 * u + 3] = v.w;
    }
}
__device__ __forceinline__ void lds_lab(const double* p, double (&c)[20]) {
#pragma unroll
    for (int u = 0; u < 20; ++u) c[u] = p[R_A0 + u];
}

// R_j(psi) = R0 [a0 + sum_n alpha_n cos n psi + beta_n sin n psi] of a staged
// record at direction (cp, sp) = (cos psi, sin psi).
// FP32: with z = e^{i psi}, c_n = alpha_n - i beta_n and w = z^2,
// sum_{n=2..10} Re(c_n z^n) = Re(w (E(w) + z O(w))), E and O the even and odd
// coefficient polynomials in w, each by complex Horner (two independent
// chains of 4 and 3 steps): 37 FMA-class operations per evaluation against
// 56 for angle addition, with the same dependency depth.
#ifndef FCC_RADIUS_HORNER
#define FCC_RADIUS_HORNER 1
#endif
__device__ __forceinline__ float radius_at(const float* p, float cp, float sp) {
#if FCC_RADIUS_HORNER
    const float wr = cp * cp - sp * sp, wi = 2.f * cp * sp;  // z^2
    const float4 v0 = lds4(p + R_A0);       // a0, al2, be2, al3
    const float4 v1 = lds4(p + R_A0 + 4);   // be3, al4, be4, al5
    const float4 v2 = lds4(p + R_A0 + 8);   // be5, al6, be6, al7
    const float4 v3 = lds4(p + R_A0 + 12);  // be7, al8, be8, al9
    const float4 v4 = lds4(p + R_A0 + 16);  // be9, al10, be10, theta
    // (er, ei) <- (er, ei) w + (al, -be)
    auto step = [&](float& r, float& im, float al, float be) {
        const float t = fmaf(r, wr, fmaf(-im, wi, al));
        im = fmaf(r, wi, fmaf(im, wr, -be));
        r = t;
    };
    float er = v4.y, ei = -v4.z;  // c10
    float orr = v3.w, oi = -v4.x;  // c9
    step(er, ei, v3.y, v3.z);   // c8
    step(orr, oi, v2.w, v3.x);  // c7
    step(er, ei, v2.y, v2.z);   // c6
    step(orr, oi, v1.w, v2.x);  // c5
    step(er, ei, v1.y, v1.z);   // c4
    step(orr, oi, v0.w, v1.x);  // c3
    step(er, ei, v0.y, v0.z);   // c2
    // q = E + z O, R = a0 + Re(w q)
    const float qr = fmaf(orr, cp, fmaf(-oi, sp, er));
    const float qi = fmaf(orr, sp, fmaf(oi, cp, ei));
    return fmaf(wr, qr, fmaf(-wi, qi, v0.x));
#else
    // angle addition (src/geometry.jl:282-291) as two chains, even and odd n,
    // both stepping by 2 psi; coefficients loaded as they are consumed
    const float c2 = cp * cp - sp * sp, s2 = 2.f * cp * sp;  // 2 psi
    const float c3 = c2 * cp - s2 * sp, s3 = s2 * cp + c2 * sp;  // 3 psi
    float4 v = lds4(p + R_A0);  // a0, al2, be2, al3
    float re = v.y * c2 + v.z * s2;
    float ro = v.w * c3;
    float ce = c2, se = s2, co = c3, so = s3;
    const float a0 = v.x;
    v = lds4(p + R_A0 + 4);  // be3, al4, be4, al5
    ro += v.x * s3;
    float t = ce * c2 - se * s2;
    se = se * c2 + ce * s2, ce = t;  // 4 psi
    re += v.y * ce + v.z * se;
    t = co * c2 - so * s2;
    so = so * c2 + co * s2, co = t;  // 5 psi
    ro += v.w * co;
    v = lds4(p + R_A0 + 8);  // be5, al6, be6, al7
    ro += v.x * so;
    t = ce * c2 - se * s2;
    se = se * c2 + ce * s2, ce = t;  // 6 psi
    re += v.y * ce + v.z * se;
    t = co * c2 - so * s2;
    so = so * c2 + co * s2, co = t;  // 7 psi
    ro += v.w * co;
    v = lds4(p + R_A0 + 12);  // be7, al8, be8, al9
    ro += v.x * so;
    t = ce * c2 - se * s2;
    se = se * c2 + ce * s2, ce = t;  // 8 psi
    re += v.y * ce + v.z * se;
    t = co * c2 - so * s2;
    so = so * c2 + co * s2, co = t;  // 9 psi
    ro += v.w * co;
    v = lds4(p + R_A0 + 16);  // be9, al10, be10, theta
    ro += v.x * so;
    t = ce * c2 - se * s2;
    se = se * c2 + ce * s2, ce = t;  // 10 psi
    re += v.y * ce + v.z * se;
    return a0 + (re + ro);
#endif
}
__device__ __forceinline__ double radius_at(const double* p, double cp, double sp) {
    double c = cp, sn = sp, r = p[R_A0];
#pragma unroll
    for (int m = 0; m < KM; ++m) {
        const double cn = c * cp - sn * sp;
        sn = sn * cp + c * sp;
        c = cn;
        r += p[r_al(m)] * c + p[r_be(m)] * sn;
    }
    return r;
}

// |u| and 1/|u| of a contour node distance (FP32: one rsqrt)
__device__ __forceinline__ void norm_inv(float x2, float& n, float& inv) {
    inv = rsqrtf(x2);
    n = x2 * inv;
}
__device__ __forceinline__ void norm_inv(double x2, double& n, double& inv) {
    n = sqrt(x2);
    inv = 1.0 / n;
}

__device__ __forceinline__ int jmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// grid coordinates, src/neighbors.jl:40-42 (clamped to the grid)
template <class T>
__device__ __forceinline__ void grid_coords(const SimDesc<T>& P, T x, T y, int& cx, int& cy) {
    cx = max(0, min((int)div_rn(x, P.wx), P.ncx - 1));
    cy = max(0, min((int)div_rn(y, P.wy), P.ncy - 1));
}

// ======================================================= rebuild phases ==
// update_celllist! + update_neighbors! (src/neighbors.jl:81-92, 148-174,
// 223-242) as a stable integer counting sort.  Each phase is a grid-stride
// loop over the bodies or cells of the simulations flagged F_NEED.

// Rebuild work list of a pool: the flagged simulations in slot order, with
// the running sums of their real bodies and of their cells.  Every block
// builds its own copy in shared memory when a rebuild starts (the flags do
// not change until it ends), so the phases visit the bodies and cells of the
// rebuilding simulations only, instead of testing every body of the arena.
struct WorkList {
    const int* sim;   // [m]     simulation slot
    const int* body;  // [m + 1] real bodies before entry t
    const int* cell;  // [m + 1] cells before entry t
    const int* boff;  // [m]     first body of the simulation
    const int* coff;  // [m]     first cell of the simulation
    int m;            // entries; -1: no list (the shared area is too small)
};
constexpr int WL_ARRAYS = 5;

// entry t holding item i of a running-sum array pre (pre[0] = 0 <= i < pre[m]):
// the largest t < m with pre[t] <= i
__device__ __forceinline__ int wl_find(const int* pre, int m, int i) {
    int lo = 0, hi = m - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Build the list in `area` (cap ints of shared memory no warp is using);
// called by every thread of the block.
template <class T>
__device__ WorkList build_worklist(const DevPtrs<T>& d, int* area, int cap) {
    __shared__ int s_scan[3][32];
    __shared__ int s_run[3];
    WorkList w{};
    w.m = -1;
    const int stride = d.nsims + 1;
    if (WL_ARRAYS * stride > cap) return w;  // uniform over the block
    int* ws = area;
    int* wb = ws + stride;
    int* wc = wb + stride;
    int* wo = wc + stride;
    int* wco = wo + stride;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (threadIdx.x == 0) s_run[0] = s_run[1] = s_run[2] = 0;
    __syncthreads();
    for (int base = 0; base < d.nsims; base += blockDim.x) {
        const int s = base + threadIdx.x;
        int need = 0, n = 0, nc = 0, bo = 0, co = 0;
        if (s < d.nsims && (ldcg(d.flags + s) & F_NEED)) {
            const SimDesc<T>& P = d.sims[s];
            need = 1;
            n = P.n;
            nc = P.ncells;
            bo = P.body_off;
            co = P.cell_off;
        }
        int a = need, b = n, c = nc;  // inclusive over the warp
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int oa = __shfl_up_sync(0xffffffffu, a, off);
            const int ob = __shfl_up_sync(0xffffffffu, b, off);
            const int oc = __shfl_up_sync(0xffffffffu, c, off);
            if (lane >= off) a += oa, b += ob, c += oc;
        }
        if (lane == 31) s_scan[0][wid] = a, s_scan[1][wid] = b, s_scan[2][wid] = c;
        __syncthreads();
        if (wid == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                int t = lane < nw ? s_scan[k][lane] : 0;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int o = __shfl_up_sync(0xffffffffu, t, off);
                    if (lane >= off) t += o;
                }
                s_scan[k][lane] = t;  // inclusive over warps
            }
        }
        __syncthreads();
        if (need) {
            const int e = s_run[0] + (wid ? s_scan[0][wid - 1] : 0) + a - 1;
            ws[e] = s;
            wb[e] = s_run[1] + (wid ? s_scan[1][wid - 1] : 0) + b - n;
            wc[e] = s_run[2] + (wid ? s_scan[2][wid - 1] : 0) + c - nc;
            wo[e] = bo;
            wco[e] = co;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_run[0] += s_scan[0][nw - 1];
            s_run[1] += s_scan[1][nw - 1];
            s_run[2] += s_scan[2][nw - 1];
        }
        __syncthreads();
    }
    w.m = s_run[0];
    if (threadIdx.x == 0) {
        wb[w.m] = s_run[1];
        wc[w.m] = s_run[2];
    }
    __syncthreads();
    w.sim = ws;
    w.body = wb;
    w.cell = wc;
    w.boff = wo;
    w.coff = wco;
    return w;
}

template <class T>
__device__ __forceinline__ void count_body(const DevPtrs<T>& d, const SimDesc<T>& P, int par, int g) {
    const T* r = rec_cur(d, par) + (size_t)g * RECW;
    int cx, cy;
    grid_coords(P, ldcg(r + R_X), ldcg(r + R_Y), cx, cy);
    const int cell = P.cell_off + cx + P.ncx * cy;
    d.cellid[g] = cell;
    d.slot[g] = atomicAdd(&d.ccount[cell], 1);
}

// `lone_need`: a single simulation's rebuild decision as the block knows it
// (the global flags may still be in flight from the last barrier), or -1:
// read each simulation's flags.
template <class T>
__device__ void phase_count(const DevPtrs<T>& d, int par, int tid, int nthr, const WorkList* wl, int lone_need = -1) {
    if (wl) {
        for (int i = tid; i < wl->body[wl->m]; i += nthr) {
            const int t = wl_find(wl->body, wl->m, i);
            count_body(d, d.sims[wl->sim[t]], par, wl->boff[t] + (i - wl->body[t]));
        }
        return;
    }
    if (lone_need == 0) return;
    for (int g = tid; g < d.Ntot; g += nthr) {
        const int s = __ldg(d.sim_of + g);
        if (s < 0 || !(lone_need > 0 || (ldcg(d.flags + s) & F_NEED))) continue;
        count_body(d, d.sims[s], par, g);
    }
}

// exclusive scan of the cell counts of each flagged simulation (one block per
// simulation); cell c holds perm[cstart[c] .. cstop[c]).  The cells go in
// chunks of SCAN_PER per thread: a thread loads its run of counts into
// registers (independent loads), one block-wide scan of the run totals gives
// the run's first slot, and the thread writes its run from the registers.
constexpr int SCAN_PER = 16;
template <class T>
__device__ void phase_scan(const DevPtrs<T>& d, const WorkList* wl) {
    __shared__ int s_warp[32];
    const int nw = (blockDim.x + 31) / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nk = wl ? wl->m : d.nsims;
    for (int k = blockIdx.x; k < nk; k += gridDim.x) {
        const int s = wl ? wl->sim[k] : k;
        if (!wl && !(ldcg(d.flags + s) & F_NEED)) continue;
        const SimDesc<T>& P = d.sims[s];
        int carry = P.body_off;
        for (int base = 0; base < P.ncells; base += blockDim.x * SCAN_PER) {
            const int u0 = base + threadIdx.x * SCAN_PER;
            const int c0 = P.cell_off + u0;
            int v[SCAN_PER];
            int sum = 0;
#pragma unroll
            for (int i = 0; i < SCAN_PER; ++i) {
                v[i] = u0 + i < P.ncells ? ldcg(d.ccount + c0 + i) : 0;
                sum += v[i];
            }
            int incl = sum;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int o = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += o;
            }
            if (lane == 31) s_warp[w] = incl;
            __syncthreads();
            if (threadIdx.x < 32) {
                int t = threadIdx.x < nw ? s_warp[threadIdx.x] : 0;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int o = __shfl_up_sync(0xffffffffu, t, off);
                    if ((int)threadIdx.x >= off) t += o;
                }
                s_warp[threadIdx.x] = t;  // inclusive over warps
            }
            __syncthreads();
            int st = carry + (w ? s_warp[w - 1] : 0) + incl - sum;
#pragma unroll
            for (int i = 0; i < SCAN_PER; ++i) {
                if (u0 + i < P.ncells) {
                    d.cstart[c0 + i] = st;
                    st += v[i];
                    d.cstop[c0 + i] = st;
                    d.ccount[c0 + i] = 0;
                }
            }
            carry += s_warp[nw - 1];
            __syncthreads();  // s_warp is rewritten by the next chunk
        }
        if (threadIdx.x == 0) {
            d.builds[s] += 1;
            d.maxcount[s] = 0;
            atomicOr(&d.flags[s], F_VALID);
        }
        __syncthreads();
    }
}

template <class T>
__device__ void phase_scatter(const DevPtrs<T>& d, int tid, int nthr, const WorkList* wl) {
    if (wl) {
        for (int i = tid; i < wl->body[wl->m]; i += nthr) {
            const int t = wl_find(wl->body, wl->m, i);
            const int g = wl->boff[t] + (i - wl->body[t]);
            d.perm[ldcg(d.cstart + ldcg(d.cellid + g)) + ldcg(d.slot + g)] = g;
        }
        return;
    }
    for (int g = tid; g < d.Ntot; g += nthr) {
        const int s = __ldg(d.sim_of + g);
        if (s < 0 || !(ldcg(d.flags + s) & F_NEED)) continue;
        d.perm[ldcg(d.cstart + ldcg(d.cellid + g)) + ldcg(d.slot + g)] = g;
    }
}

// ties of the stable sortperm! (src/neighbors.jl:86) are ordered by body
// index: sort each cell's few bodies ascending.  A cell of at most SORT_REG
// bodies is loaded into registers at once and each body is written to its
// rank (the ids are distinct); a larger cell takes the insertion sort.
constexpr int SORT_REG = 16;
template <class T>
__device__ void phase_sort(const DevPtrs<T>& d, int tid, int nthr, const WorkList* wl) {
    const int nc = wl ? wl->cell[wl->m] : d.Ctot;
    for (int i = tid; i < nc; i += nthr) {
        int c = i;
        if (wl) {
            const int t = wl_find(wl->cell, wl->m, i);
            c = wl->coff[t] + (i - wl->cell[t]);
        } else {
            const int s = __ldg(d.cell_sim + c);
            if (!(ldcg(d.flags + s) & F_NEED)) continue;
        }
        const int a = ldcg(d.cstart + c), b = ldcg(d.cstop + c);
        const int n = b - a;
        if (n <= 1) continue;
        if (n <= SORT_REG) {
            int v[SORT_REG];
#pragma unroll
            for (int i = 0; i < SORT_REG; ++i) v[i] = i < n ? ldcg(d.perm + a + i) : INT_MAX;
#pragma unroll
            for (int i = 0; i < SORT_REG; ++i) {
                if (i < n) {
                    int r = 0;
#pragma unroll
                    for (int k = 0; k < SORT_REG; ++k) r += v[k] < v[i] ? 1 : 0;
                    d.perm[a + r] = v[i];
                }
            }
            continue;
        }
        for (int q = a + 1; q < b; ++q) {
            const int v = ldcg(d.perm + q);
            int r = q - 1;
            while (r >= a && ldcg(d.perm + r) > v) {
                d.perm[r + 1] = ldcg(d.perm + r);
                --r;
            }
            d.perm[r + 1] = v;
        }
    }
}

// neighbour list of one body: the 3x3 grid cells around it in the
// reference's order (oy outer, ox inner), candidates in perm order, kept if
// |ri - rj| <= rmax_i + rmax_j + range (exactly rounded like the oracle).
// NB_LANES lanes per body: lane h reads the ranges of cells h and 8, the
// candidates of the nine cells are numbered in list order and taken
// NB_LANES * NB_PER at a time, NB_PER per lane (their perm entries, then
// their records, each as independent loads), and ballot prefixes write the
// kept ones in list order.  A body costs four dependent L2 round trips (own
// record, cell ranges, perm, records) instead of one per candidate.  With a
// single simulation (sim0: its descriptor in shared memory) the per-body
// simulation and flag reads are skipped.  tid / nthr count threads; the grid
// is whole warps.
constexpr int NB_LANES = 8, NB_PER = 8;
template <class T>
__device__ void phase_neighbors(const DevPtrs<T>& d, int par, int tid, int nthr, const SimDesc<T>* sim0,
                                const WorkList* wl, int* overflow = nullptr) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int BPW = 32 / NB_LANES, ROUND = NB_LANES * NB_PER;
    constexpr unsigned SUBMASK = (1u << NB_LANES) - 1u;
    const int lane = tid & 31, h = lane % NB_LANES, sub = lane / NB_LANES;
    if (sim0 && !(ldcg(d.flags) & F_NEED)) return;  // uniform over the grid
    const T* rc = rec_cur(d, par);
    // the loop bound is uniform over the warp: every lane takes every shuffle
    const int nitems = wl ? wl->body[wl->m] : d.Ntot;
    for (int gw = BPW * (tid >> 5); gw < nitems; gw += BPW * (nthr >> 5)) {
        int g = gw + sub;
        int s = 0;
        bool act;
        const SimDesc<T>* P = sim0;
        if (sim0) {
            act = g < d.Ntot;
        } else if (wl) {
            act = g < nitems;
            if (act) {
                const int t = wl_find(wl->body, wl->m, g);
                s = wl->sim[t];
                g = wl->boff[t] + (g - wl->body[t]);
                P = d.sims + s;
            }
        } else {
            s = g < d.Ntot ? __ldg(d.sim_of + g) : -1;
            act = s >= 0 && (ldcg(d.flags + s) & F_NEED);
            P = act ? d.sims + s : nullptr;
        }
        T xi = T(0), yi = T(0), rmi = T(0), ri = T(0);
        int qa0 = 0, cnt0 = 0, qa8 = 0, cnt8 = 0;
        if (act) {
            xi = ldcg(rc + (size_t)g * RECW + R_X);
            yi = ldcg(rc + (size_t)g * RECW + R_Y);
            rmi = ldcg(rc + (size_t)g * RECW + R_RMAX);
            ri = add_rn(rmi, P->nbrange);
            int cx, cy;
            grid_coords(*P, xi, yi, cx, cy);
            const int rx = P->ncx >= 3 ? 1 : 0, ry = P->ncy >= 3 ? 1 : 0;
            const int wx = 2 * rx + 1, ncell = wx * (2 * ry + 1);
            if (h < ncell) {
                const int oy = h / wx - ry, ox = h % wx - rx;
                const int cell = P->cell_off + jmod(cx + ox, P->ncx) + P->ncx * jmod(cy + oy, P->ncy);
                qa0 = ldcg(d.cstart + cell);
                cnt0 = ldcg(d.cstop + cell) - qa0;
            }
            if (8 < ncell) {  // cell 8 (ox = oy = +1), read by every lane of the body
                const int cell = P->cell_off + jmod(cx + 1, P->ncx) + P->ncx * jmod(cy + 1, P->ncy);
                qa8 = ldcg(d.cstart + cell);
                cnt8 = ldcg(d.cstop + cell) - qa8;
            }
        }
        int incl = cnt0;
#pragma unroll
        for (int off = 1; off < NB_LANES; off <<= 1) {
            const int o = __shfl_up_sync(FULL, incl, off, NB_LANES);
            if (h >= off) incl += o;
        }
        const int first8 = __shfl_sync(FULL, incl, NB_LANES - 1, NB_LANES);  // cells 0..7
        const int total = first8 + cnt8;
        // candidate k lies in cell c with from_c <= k < from_c + cnt_c, at perm[k + shift_c]
        int from[9], shift[9];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            from[c] = __shfl_sync(FULL, incl - cnt0, c, NB_LANES);
            shift[c] = __shfl_sync(FULL, qa0, c, NB_LANES) - from[c];
        }
        from[8] = first8;
        shift[8] = qa8 - first8;
        int tmax = max(total, __shfl_xor_sync(FULL, total, 8));
        tmax = max(tmax, __shfl_xor_sync(FULL, tmax, 16));
        int* out = d.nb_idx + (size_t)(act ? g : 0) * d.cap;
        int n = 0;
        for (int k0 = 0; k0 < tmax; k0 += ROUND) {
            int j[NB_PER];
#pragma unroll
            for (int i = 0; i < NB_PER; ++i) {
                const int k = k0 + NB_LANES * i + h;
                j[i] = -1;
                if (k < total) {
                    int q = k + shift[0];
#pragma unroll
                    for (int c = 1; c < 9; ++c)
                        if (k >= from[c]) q = k + shift[c];
                    j[i] = ldcg(d.perm + q);
                }
            }
            unsigned keepbits = 0;
#pragma unroll
            for (int i = 0; i < NB_PER; ++i) {
                if (j[i] >= 0 && j[i] != g) {
                    const T* rj = rc + (size_t)j[i] * RECW;
                    const T xj = ldcg(rj + R_X), yj = ldcg(rj + R_Y), rmj = ldcg(rj + R_RMAX);
                    const T dx = minimum_image_exact(sub_rn(xi, xj), P->Lx);
                    const T dy = minimum_image_exact(sub_rn(yi, yj), P->Ly);
                    const T lim = add_rn(ri, rmj);
                    if (add_rn(mul_rn(dx, dx), mul_rn(dy, dy)) <= mul_rn(lim, lim)) keepbits |= 1u << i;
                }
            }
#pragma unroll
            for (int i = 0; i < NB_PER; ++i) {
                const bool keep = (keepbits >> i) & 1u;
                const unsigned m = (__ballot_sync(FULL, keep) >> (NB_LANES * sub)) & SUBMASK;
                const int pos = n + __popc(m & ((1u << h) - 1u));
                if (keep && pos < d.cap) out[pos] = j[i];
                n += __popc(m);
            }
        }
        if (act && h == 0) {
            d.nb_count[g] = n;
            if (n > d.cap) {
                atomicOr(&d.flags[s], F_FROZEN);
                if (overflow) *overflow = 1;  // the block's vote at the closing flat barrier
            }
            atomicMax(&d.maxcount[s], n);
            if (P->skin > T(0)) {
                d.x0[g] = xi;
                d.y0[g] = yi;
                d.rmax0[g] = rmi;
            }
        }
    }
}

// ============================================================= update ==
// Neighbour records staged in shared memory per body (the rest are read from
// L2 in the loop).  At packing 0.95 with the 0.3 skin a body lists 6-9.
constexpr int NBMAX = 12;

#ifndef FCC_DYN
#define FCC_DYN 1  // 1: FP32, one simulation: warps take their block's warp groups dynamically
#endif
#ifndef FCC_FLAT_BARRIER
#define FCC_FLAT_BARRIER 1  // 1: a lone simulation's step barrier polls its arrival counter (flat_barrier)
#endif

// FP32 single-chunk kernels read cos(n phi_k), sin(n phi_k) (and n times
// them) of their contour nodes from a shared-memory table instead of running
// the angle-addition recurrence: four floats per node and mode, a node's row
// 36 words apart (conflict-free float4 reads for the 8 nodes a warp reads).
constexpr int BASIS_NODES = 40;
#ifndef FCC_MODE_TABLE
#define FCC_MODE_TABLE 2  // 1: synthesis reads the table, 2: pullback (measured fastest), 3: both
#endif
// Fragments of the tensor-core contractions (below), staged after the mode
// table: 9 synthesis tiles and 10 pullback tiles, each a TF32 high part and
// a TF32 remainder, 32 lanes x 4 values.
constexpr int MMA_SYN_TILES = 9;   // 3 node tiles (48 rows) x 3 coefficient tiles (24 columns)
constexpr int MMA_PB_TILES = 10;   // 2 coefficient tiles (32 rows) x 5 node tiles (40 columns)
constexpr int MMA_TABLE_FLOATS = (MMA_SYN_TILES + MMA_PB_TILES) * 2 * 32 * 4;
template <class T>
__host__ __device__ constexpr size_t basis_table_bytes() {
    return sizeof(T) == 4 ? (size_t)BASIS_NODES * KM * 4 * sizeof(T) + (size_t)MMA_TABLE_FLOATS * sizeof(float) : 0;
}

// Per warp: the own records of its 32/L bodies, then NBMAX neighbour
// records per body.
// Per warp, last: a copy of the simulation descriptor its bodies belong to
// (pools; a single simulation's is shared by the block).
template <class T>
__host__ __device__ constexpr size_t desc_slot_bytes() {
    return (sizeof(SimDesc<T>) + 15) / 16 * 16;
}
#ifndef FCC_WALK_SMEM
#define FCC_WALK_SMEM 1  // 1: the hit walk reads its node (R, cos, sin) and adds its pressure in shared memory
#endif
// node slots per lane of a variant with L lanes per body (one 40-node chunk)
__host__ __device__ constexpr int slots_of(int L) { return (BASIS_NODES + L - 1) / L; }
template <class T, int L>
__host__ __device__ constexpr size_t walk_bytes_per_warp() {
    return FCC_WALK_SMEM ? (size_t)32 * slots_of(L) * 4 * sizeof(T) : 0;
}
template <class T, int L>
__host__ __device__ constexpr size_t stage_bytes_per_warp() {
    return (size_t)(32 / L) * (1 + NBMAX) * RECW * sizeof(T) + desc_slot_bytes<T>() + walk_bytes_per_warp<T, L>();
}

// ------------------------------------------------ tensor-core contractions
// FP32 kernels of 8 lanes x 5 node slots with one 40-node chunk run the
// dense contour contractions of a warp's 4 bodies on the tensor cores
// (mma.sync m16n8k8, TF32 inputs, FP32 accumulation):
//   pullback    [g_b | h_b] (coefficients x 8) = A^T (32 x 40) . [GR_b | GD_b]
//     (40 x 8, columns 2b and 2b + 1 of body b), and glab = g + D h with D
//     the derivative's coefficient map (alpha_m: -n h[beta_m], beta_m:
//     +n h[alpha_m]): S' Gall of src/gradients.jl:374-386 with the R'' rows
//     empty, summed over all the body's nodes at once (no lane reductions);
//   synthesis   [R_b | R'_b] (nodes x 8) = A (48 x 24) . [c_b | c'_b] (24 x 8)
//     (FCC_MMA_SYNTH = 1), c the R0-scaled lab coefficients of the record
//     and c' = (0, n beta, -n alpha) the derivative's, so R' = A . c'
//     (src/geometry.jl:113-122, 248-257).
// A[k][j] = 1, cos n phi_k, sin n phi_k for coefficient j in record order
// (a0, alpha_2, beta_2, ...).  Each operand is split into a TF32 high part
// and a TF32 remainder and the product taken as lo.hi + hi.lo + hi.hi in
// separate accumulators (the lo.lo term, ~2^-22 relative, dropped): FP32-level
// accuracy from TF32 units, with dependency chains one k-tile long per term.
// The tiles pass between the fragment layout and the lanes' node slots
// through the warp's walk-slot shared memory as (column 2b, 2b + 1) float2
// pairs, rows of 8 floats with the columns of rows 4..7 (mod 8) rotated by 4
// words: conflict-free both ways.
#ifndef FCC_MMA_SYNTH
#define FCC_MMA_SYNTH 0  // 1: contour synthesis on the tensor cores too (measured: slower, see DESIGN)
#endif

__device__ __forceinline__ uint32_t tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - __uint_as_float(hi));  // x - hi is exact in FP32
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint4& a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}
// A fragment of `tile` (split 0: high, 1: remainder) for this lane
__device__ __forceinline__ uint4 mma_frag(const float* mtab, int tile, int split, int lane) {
    return *reinterpret_cast<const uint4*>(mtab + ((size_t)(tile * 2 + split) * 32 + lane) * 4);
}
// word offset of the (column 2b, 2b + 1) pair of row r in the transposition buffer
__device__ __forceinline__ int mma_pair(int r, int b) { return r * 8 + ((2 * b + 4 * ((r >> 2) & 1)) & 7); }
// word offset of element (r, column c)
__device__ __forceinline__ int mma_elem(int r, int c) { return r * 8 + ((c + 4 * ((r >> 2) & 1)) & 7); }

// Contour synthesis of the warp's 4 bodies on the tensor cores: R, R' at the
// lane's 5 node slots (node l + 8 s of body lane / 8).  own: the 4 staged own
// records; buf: 48 x 8 floats of warp scratch.
__device__ __forceinline__ void synth_mma(const float* own, float* buf, const float* mtab, int lane, float (&R)[5],
                                          float (&R1)[5]) {
    const int gid = lane >> 2, tig = lane & 3;
    const float* rec = own + (gid >> 1) * RECW + R_A0;  // B column gid: body gid / 2, derivative if odd
    const bool deriv = gid & 1;
    uint32_t bh[3][2], bl[3][2];
#pragma unroll
    for (int kt = 0; kt < 3; ++kt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = kt * 8 + tig + 4 * h;
            float v = 0.f;
            if (j < NCM) {
                if (!deriv) {
                    v = rec[j];
                } else if (j > 0) {  // alpha_m at j = 1 + 2m, beta_m at j = 2 + 2m; n = m + 2
                    const float n = (float)(((j - 1) >> 1) + 2);
                    v = (j & 1) ? n * rec[j + 1] : -n * rec[j - 1];
                }
            }
            tf32_split(v, bh[kt][h], bl[kt][h]);
        }
    float big[3][4], small[3][4];
#pragma unroll
    for (int mt = 0; mt < 3; ++mt)
#pragma unroll
        for (int i = 0; i < 4; ++i) big[mt][i] = small[mt][i] = 0.f;
#pragma unroll
    for (int kt = 0; kt < 3; ++kt)
#pragma unroll
        for (int mt = 0; mt < 3; ++mt) {
            const int tile = mt * 3 + kt;
            const uint4 ah = mma_frag(mtab, tile, 0, lane), al = mma_frag(mtab, tile, 1, lane);
            mma_tf32(small[mt], al, bh[kt][0], bh[kt][1]);
            mma_tf32(small[mt], ah, bl[kt][0], bl[kt][1]);
            mma_tf32(big[mt], ah, bh[kt][0], bh[kt][1]);
        }
    __syncwarp();  // every lane is done with the buffer's previous contents
#pragma unroll
    for (int mt = 0; mt < 3; ++mt) {  // rows gid, gid + 8 of the tile; the (R, R') pair of body tig
        const int r0 = 16 * mt + gid;
        *reinterpret_cast<float2*>(buf + mma_pair(r0, tig)) =
            make_float2(small[mt][0] + big[mt][0], small[mt][1] + big[mt][1]);
        *reinterpret_cast<float2*>(buf + mma_pair(r0 + 8, tig)) =
            make_float2(small[mt][2] + big[mt][2], small[mt][3] + big[mt][3]);
    }
    __syncwarp();
    const int b = lane >> 3, l = lane & 7;
#pragma unroll
    for (int sl = 0; sl < 5; ++sl) {
        const float2 v = *reinterpret_cast<const float2*>(buf + mma_pair(l + 8 * sl, b));
        R[sl] = v.x;
        R1[sl] = v.y;
    }
    __syncwarp();  // the buffer is free again
}

// Pullback of the warp's 4 bodies on the tensor cores: from GR, GD at the
// lane's 5 node slots (0 at slots beyond the contour), leaves the (g, h)
// pairs in buf (32 x 8) for pullback_entry, readable by every lane.
__device__ __forceinline__ void pullback_mma(const float (&GR)[5], const float (&GD)[5], float* buf,
                                             const float* mtab, int lane) {
    const int b = lane >> 3, l = lane & 7;
    __syncwarp();
#pragma unroll
    for (int sl = 0; sl < 5; ++sl)
        *reinterpret_cast<float2*>(buf + mma_pair(l + 8 * sl, b)) = make_float2(GR[sl], GD[sl]);
    __syncwarp();
    const int gid = lane >> 2, tig = lane & 3;
    float big[2][4], small[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int i = 0; i < 4; ++i) big[mt][i] = small[mt][i] = 0.f;
#pragma unroll
    for (int kt = 0; kt < 5; ++kt) {  // B rows (nodes) 8 kt + tig and + 4, column gid
        uint32_t b0h, b0l, b1h, b1l;
        tf32_split(buf[mma_elem(8 * kt + tig, gid)], b0h, b0l);
        tf32_split(buf[mma_elem(8 * kt + tig + 4, gid)], b1h, b1l);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int tile = MMA_SYN_TILES + mt * 5 + kt;
            const uint4 ah = mma_frag(mtab, tile, 0, lane), al = mma_frag(mtab, tile, 1, lane);
            mma_tf32(small[mt], al, b0h, b1h);
            mma_tf32(small[mt], ah, b0l, b1l);
            mma_tf32(big[mt], ah, b0h, b1h);
        }
    }
    __syncwarp();  // every lane has read its B fragments
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {  // rows (coefficients) gid, gid + 8; the (g, h) pair of body tig
        const int r0 = 16 * mt + gid;
        *reinterpret_cast<float2*>(buf + mma_pair(r0, tig)) =
            make_float2(small[mt][0] + big[mt][0], small[mt][1] + big[mt][1]);
        *reinterpret_cast<float2*>(buf + mma_pair(r0 + 8, tig)) =
            make_float2(small[mt][2] + big[mt][2], small[mt][3] + big[mt][3]);
    }
    __syncwarp();
}
// glab entry r (engine order [a0; alpha_2..alpha_10; beta_2..beta_10]) of
// body b from the pullback buffer
__device__ __forceinline__ float pullback_entry(const float* buf, int b, int r) {
    if (r == 0) return buf[mma_pair(0, b)];
    const bool alpha = r <= KM;
    const int m = alpha ? r - 1 : r - 1 - KM;
    const float n = (float)(m + 2);
    const float2 pa = *reinterpret_cast<const float2*>(buf + mma_pair(1 + 2 * m, b));  // (g, h) of alpha_m
    const float2 pb = *reinterpret_cast<const float2*>(buf + mma_pair(2 + 2 * m, b));  // (g, h) of beta_m
    return alpha ? pa.x - n * pb.y : pb.x + n * pa.y;
}

// Operands of the update loaded early (their latency overlaps the force
// evaluation): the body's a0, its lane's shape modes and, on lane 0, the
// skin reference of the last neighbour-list build.
template <class T, int L>
struct UpdatePre {
    static constexpr int MPL = (KM + L - 1) / L;
    T a0, a[MPL], b[MPL], x0, y0, rmax0;
};

template <class T, int L>
__device__ __forceinline__ void load_update_pre(const DevPtrs<T>& d, int gg, int l, int K, UpdatePre<T, L>& u) {
    const T* cf = d.coef + (size_t)gg * NCM;
    u.a0 = ldcg(cf);
#pragma unroll
    for (int v = 0; v < UpdatePre<T, L>::MPL; ++v) {
        const int m = l + v * L;
        u.a[v] = m < K ? ldcg(cf + 1 + m) : T(0);
        u.b[v] = m < K ? ldcg(cf + 1 + KM + m) : T(0);
    }
    if (l == 0) {
        u.x0 = ldcg(d.x0 + gg);
        u.y0 = ldcg(d.y0 + gg);
        u.rmax0 = ldcg(d.rmax0 + gg);
    } else {
        u.x0 = u.y0 = u.rmax0 = T(0);
    }
}

// (cos n t, sin n t) from (cos t, sin t) by binary powering, n = 2..10 (a
// few complex products instead of one sincos per mode).
// Per-mode pieces of the end of a step, shared by the update and by k_init so
// that a state loaded with set_state continues exactly as the run that wrote
// it: |(a, b)| for rmax and the projection, its FP64 square for a0, and the
// rotation into the lab frame.
template <class T>
__device__ __forceinline__ T mode_norm(T a, T b) {
    return t_sqrt(a * a + b * b);
}
template <class T>
__device__ __forceinline__ double mode_sq(T a, T b) {
    return (double)a * (double)a + (double)b * (double)b;
}
template <class T>
__device__ __forceinline__ void to_lab(T a, T b, T co, T so, T& al, T& be) {
    al = a * co - b * so;
    be = a * so + b * co;
}

template <class T>
__device__ __forceinline__ void cis_pow(T c1, T s1, int n, T& cn, T& sn) {
    T rc = T(1), rs = T(0), bc = c1, bs = s1;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        if (n & (1 << b)) {
            const T t = rc * bc - rs * bs;
            rs = rc * bs + rs * bc;
            rc = t;
        }
        const T t = bc * bc - bs * bs;
        bs = T(2) * bc * bs;
        bc = t;
    }
    cn = rc;
    sn = rs;
}

// Translational displacement of a body with substrate drag, plus the forces
// of its children with parent drag (src/dynamics.jl:84-99).
template <class T>
__device__ __forceinline__ void substrate_displacement(const DevPtrs<T>& d, const SimDesc<T>& P, const T* rc, int c,
                                                       long long clk, T& ox, T& oy) {
    const int tc = unpack_w(ldcg(rc + (size_t)c * RECW + R_W)) & 7;
    T fx = ldcg(d.gx + c), fy = ldcg(d.gy + c);
    const int nch = __ldg(d.ch_count + c);
    for (int q = 0; q < nch; ++q) {
        const int k = __ldg(d.ch_idx + (size_t)c * d.ccap + q);
        const int tk = unpack_w(ldcg(rc + (size_t)k * RECW + R_W)) & 7;
        if (P.parent_drag[tk]) {
            fx += ldcg(d.gx + k);
            fy += ldcg(d.gy + k);
        }
    }
    T so, co;
    t_sincos(ldcg(rc + (size_t)c * RECW + R_TH), &so, &co);
    const T dt = P.dt;
    const T sig = P.sigt[tc];
    T x1 = T(0), x2 = T(0);
    if (sig != T(0)) philox_pair<T>(P.k0, P.k1, (uint32_t)(c - P.body_off + 1), (uint64_t)clk, 0u, x1, x2);
    ox = dt * (P.v0[tc] * co - P.mur[tc] * fx) + sig * x1;
    oy = dt * (P.v0[tc] * so - P.mur[tc] * fy) + sig * x2;
}

// The lab-frame gradients a lane's update needs: gA[u], gB[u] = dE/dalpha,
// dE/dbeta of its modes m = l + L u, from the full group-reduced glab row.
template <class T, int L>
__device__ __forceinline__ void lane_mode_grads(const T (&gl)[NCM], int l, T (&gA)[UpdatePre<T, L>::MPL],
                                                T (&gB)[UpdatePre<T, L>::MPL]) {
#pragma unroll
    for (int u = 0; u < UpdatePre<T, L>::MPL; ++u) {
        const int m = l + u * L;
        T ga = gl[1], gb = gl[1 + KM];
#pragma unroll
        for (int mm = 1; mm < KM; ++mm)
            if (mm == m) ga = gl[1 + mm], gb = gl[1 + KM + mm];
        gA[u] = ga;
        gB[u] = gb;
    }
}

// Euler-Maruyama update of body g by the L lanes of its group
// (src/dynamics.jl:128-203 with frame = true): body-frame gradient, theta and
// shape update, shape bound projection and a0 (FP64 accumulation), wrap,
// lab frame of the new state into rec[next], skin check.  fx, fy, tt and gl0
// (dE/da0 of the lab frame / R0) are uniform across the group; gA, gB are the
// lab-frame mode gradients of the lane's modes (lane_mode_grads).
template <class T, int L>
__device__ __forceinline__ void update_body(const DevPtrs<T>& d, const SimDesc<T>& P, bool act, int g, int s, int l,
                                            int par, long long clk, T xo, T yo, T wo, T tho, T r0, int ti, T fx, T fy,
                                            T tt, T gl0, const T (&gA)[UpdatePre<T, L>::MPL],
                                            const T (&gB)[UpdatePre<T, L>::MPL], const UpdatePre<T, L>& pre, int fl,
                                            const T (&nz)[2], bool split, int* rbp) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int MPL = UpdatePre<T, L>::MPL;
    const T dt = P.dt;
    const uint32_t li = (uint32_t)(g - P.body_off + 1);
    // standard normals of this body and step (src/random.jl:88-100): lane 0
    // holds block 1 (orientation), lane 1 block 0 (translation)
    const T z3 = __shfl_sync(FULL, nz[0], 0, L);
    const T xi1 = __shfl_sync(FULL, nz[0], 1, L);
    const T xi2 = __shfl_sync(FULL, nz[1], 1, L);
    const T sig_r = P.sigr[ti];
    const T thn = tho - (dt * P.muth[ti]) * tt + sig_r * z3;
    T so1, co1, sn1, cn1;
    t_sincos(tho, &so1, &co1);
    t_sincos(thn, &sn1, &cn1);

    T* cf = d.coef + (size_t)(act ? g : 0) * NCM;
    const T a0 = pre.a0;
    const T ga0 = r0 * gl0;
    const T h0 = ga0 / (T(2) * a0);  // dE/da0 * da0/da_n = -h0 a_n (area constraint)
    const T dtmu = dt * P.muab[ti];
    const int K = P.K;
    const int Kt = min(K, P.kmax[ti]);  // modes of this type; the rest stay zero
    T an[MPL], bn[MPL];
    double sp = 0.0;
#pragma unroll
    for (int u = 0; u < MPL; ++u) {
        const int m = l + u * L;
        an[u] = T(0);
        bn[u] = T(0);
        if (m < Kt) {
            const T ga = gA[u] * r0, gb = gB[u] * r0;
            T so, co;
            cis_pow(co1, so1, m + 2, co, so);
            const T a = pre.a[u], b = pre.b[u];
            const T gca = ga * co + gb * so - h0 * a;
            const T gcb = -ga * so + gb * co - h0 * b;
            an[u] = a - dtmu * gca;
            bn[u] = b - dtmu * gcb;
            sp += (double)mode_norm(an[u], bn[u]);
        }
    }
    // enforce_shape! (src/dynamics.jl:44-64) with FP64 sums
    const double ssum = group_sum<L>(sp);
    if (ssum > SHAPE_BOUND) {
        const double f = SHAPE_BOUND / ssum;
#pragma unroll
        for (int u = 0; u < MPL; ++u) {
            an[u] = T((double)an[u] * f);
            bn[u] = T((double)bn[u] * f);
        }
    }
    double qp = 0.0;
#pragma unroll
    for (int u = 0; u < MPL; ++u) qp += mode_sq(an[u], bn[u]);
    const double qs = group_sum<L>(qp);
    const T a0n = T(sqrt(1.0 - qs * 0.5));

    // lab frame of the new state (src/geometry.jl:208-227)
    T* rn = rec_next(d, par) + (size_t)(act ? g : 0) * RECW;
    T bp = T(0);
#pragma unroll
    for (int u = 0; u < MPL; ++u) {
        const int m = l + u * L;
        if (m < K) {
            T so, co, al, be;
            cis_pow(cn1, sn1, m + 2, co, so);
            to_lab(an[u], bn[u], co, so, al, be);
            bp += mode_norm(an[u], bn[u]);
            if (act) {
                rn[r_al(m)] = r0 * al;
                rn[r_be(m)] = r0 * be;
                cf[1 + m] = an[u];
                cf[1 + KM + m] = bn[u];
            }
        }
    }
    const T rmax = r0 * (a0n + group_sum<L>(bp));

    if (act && l == 0) {
        T dxp, dyp;
        if (split) {
            const T* rc = rec_cur(d, par);
            if (P.parent_drag[ti]) {
                const int c = unpack_w(wo) >> 3;
                T ux, uy;
                substrate_displacement(d, P, rc, c, clk, ux, uy);
                const T sig = P.sigt[ti];
                dxp = ux + dt * (P.v0[ti] * co1 - P.mur[ti] * fx) + sig * xi1;
                dyp = uy + dt * (P.v0[ti] * so1 - P.mur[ti] * fy) + sig * xi2;
            } else {
                substrate_displacement(d, P, rc, g, clk, dxp, dyp);
            }
        } else {
            const T sig = P.sigt[ti];
            dxp = dt * (P.v0[ti] * co1 - P.mur[ti] * fx) + sig * xi1;
            dyp = dt * (P.v0[ti] * so1 - P.mur[ti] * fy) + sig * xi2;
        }
        int sx, sy;
        const T xw = wrap_exact(add_rn(xo, dxp), P.Lx, sx);
        const T yw = wrap_exact(add_rn(yo, dyp), P.Ly, sy);
        if (sx) d.imgx[g] += sx;  // image counters change only on a wrap
        if (sy) d.imgy[g] += sy;
        rn[R_X] = xw;
        rn[R_Y] = yw;
        rn[R_RMAX] = rmax;
        rn[R_W] = wo;
        rn[R_A0] = r0 * a0n;
        rn[R_TH] = thn;
        cf[0] = a0n;
        // skin check of the new state (src/neighbors.jl:198-205); the flags of
        // this step (read at its start) already carry F_VALID of a rebuild
        if ((fl & F_CONTACT) && (fl & F_VALID) && P.skin > T(0)) {
            const T dx = minimum_image_exact(sub_rn(xw, pre.x0), P.Lx);
            const T dy = minimum_image_exact(sub_rn(yw, pre.y0), P.Ly);
            const T grow = sub_rn(rmax, pre.rmax0);
            const T delta = add_rn(t_sqrt(add_rn(mul_rn(dx, dx), mul_rn(dy, dy))), grow > T(0) ? grow : T(0));
            if (mul_rn(T(2), delta) > P.skin) {
                atomicOr(&d.flags[s], F_REBUILD);
                if (rbp) *rbp = 1;  // the block's arrival at the step barrier reports it
            }
        }
        if (!(isfinite(xw) && isfinite(yw) && isfinite(thn) && isfinite(rmax))) atomicOr(&d.flags[s], F_NONFINITE);
    }
}

// A simulation that does not step (frozen or an empty slot) keeps its state:
// its records are copied into the next buffer.
template <class T, int L>
__device__ __forceinline__ void carry_record(const DevPtrs<T>& d, int g, int l, int par, const T (&rv)[RECW]) {
    T* rn = rec_next(d, par) + (size_t)g * RECW;
#pragma unroll
    for (int u = 0; u < RECW; ++u)
        if ((u & (L - 1)) == l) rn[u] = rv[u];
}
// the same from the record staged in shared memory
template <class T, int L>
__device__ __forceinline__ void carry_record_staged(const DevPtrs<T>& d, int g, int l, int par, const T* own) {
    T* rn = rec_next(d, par) + (size_t)g * RECW;
    for (int u = l; u < RECW; u += L) rn[u] = own[u];
}

// ==================================================== force evaluation ==
enum : int { MODE_FUSED = 0, MODE_FORCES = 1, MODE_DIAG = 2 };

// Forces on the 32/L bodies of warp group `wg`, and in MODE_FUSED their
// update.  `stage` is this warp's shared-memory slot for neighbour records.
// Follows, per body i:
//   contour synthesis R, R' at the nodes        src/geometry.jl:248-257
//   body terms (Tension, PerimeterElasticity)   src/gradients.jl:70-98, 197-228
//   contact pressure at the nodes (Overlap,     src/energies/contact.jl:300-324,
//     LinearRepulsion) and its gradients          391-429; src/gradients.jl:265-307
//   bond forces                                 src/energies/bonds.jl:98-111
//   pullback glab = S' Gall                     src/gradients.jl:374-386
// USER: the simulation has compiled user terms (include/fcc_user_terms.h):
// R'' is synthesised, user integrals, node gradients (GDD included),
// pressures and bond gradients are added, and the pullback includes R''.
template <class T, int L, int S, bool ONE, int MODE, bool USER = false>
__device__ __forceinline__ void forces_warp(const DevPtrs<T>& d, int wg, T* stage, int par, const SimDesc<T>* sim0,
                                            const T* tab, int& cached, int* rbp, const BarrierLocal* lone) {
    constexpr int BPW = 32 / L;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int CH16 = RECW * (int)sizeof(T) / 16;  // 16-byte chunks per record
    constexpr int IDS = (NBMAX + L - 1) / L;           // staged neighbour ids per lane
    // the mode table is staged (stage_basis); synthesis and pullback may use it
    constexpr bool USE_TAB = ONE && sizeof(T) == 4;
    constexpr bool TAB_SYNTH = USE_TAB && (FCC_MODE_TABLE & 1);
    constexpr bool TAB_PULL = USE_TAB && (FCC_MODE_TABLE & 2);
    // FP32, 8 lanes x 5 node slots, one chunk: synthesis and pullback on the tensor cores
    constexpr bool MMA = ONE && sizeof(T) == 4 && L == 8 && S == 5 && !USER;
    constexpr bool MMA_S = MMA && FCC_MMA_SYNTH;
    constexpr int MPL = UpdatePre<T, L>::MPL;
    const int lane = threadIdx.x & 31;
    const int l = lane & (L - 1);
    const int g = wg * BPW + lane / L;
    // Several simulations: each one's bodies start at a multiple of 8 and its
    // padding follows them, so a warp group lies in one simulation and its
    // first body is real unless the whole group is padding.
    int s = 0;
    if (!sim0) {
        const int gf = wg * BPW;
        s = gf < d.Ntot ? __ldg(d.sim_of + gf) : -1;
        if (s < 0) return;
        if (s != cached) {  // the warp moved to another simulation: copy its descriptor
            SimDesc<T>* wd = reinterpret_cast<SimDesc<T>*>(stage + (size_t)BPW * (1 + NBMAX) * RECW);
            const unsigned* src = reinterpret_cast<const unsigned*>(d.sims + s);
            unsigned* dst = reinterpret_cast<unsigned*>(wd);
            __syncwarp();
            for (int u = lane; u < (int)(sizeof(SimDesc<T>) / 4); u += 32) dst[u] = __ldg(src + u);
            __syncwarp();
            cached = s;
        }
    }
    const SimDesc<T>& P =
        sim0 ? *sim0 : *reinterpret_cast<const SimDesc<T>*>(stage + (size_t)BPW * (1 + NBMAX) * RECW);
    const bool valid = sim0 ? g < d.Ntot : g < P.body_off + P.n;
    const int gg = valid ? g : (sim0 ? 0 : wg * BPW);
    const T* rc = rec_cur(d, par);
    // ---- independent loads first: own record (centre, tag, a0 and theta to
    // registers, the whole record to shared memory), neighbour count and ids,
    // simulation state, update operands
    T* own = stage + (size_t)(lane / L) * RECW;
    T* snb = stage + (size_t)BPW * RECW + (size_t)(lane / L) * NBMAX * RECW;
    const T* grec = rc + (size_t)gg * RECW;
    T xi, yi, rmi, wf;
    load_head(grec, xi, yi, rmi, wf);
    const T a0r = ldcg(grec + R_A0), th = ldcg(grec + R_TH);
    for (int c = l; c < CH16; c += L) cp_async16(own + c * (16 / sizeof(T)), grec + c * (16 / sizeof(T)));
    cp_async_commit();
    const T r0 = __ldg(d.R0 + gg);
    const int cnt_raw = ldcg(d.nb_count + gg);
    int ids[IDS];
#pragma unroll
    for (int u = 0; u < IDS; ++u) {
        const int q = l + u * L;
        ids[u] = q < min(d.cap, NBMAX) ? ldcg(d.nb_idx + (size_t)gg * d.cap + q) : gg;
    }
    // a lone simulation's flags and clock are known to the block (released with the barrier)
    const int fl = lone ? lone->flags : ldcg(d.flags + s);
    const long long clk = lone ? lone->clock : ldcg(d.clock + s);
    UpdatePre<T, L> pre;
    if (MODE == MODE_FUSED) load_update_pre(d, gg, l, P.K, pre);
    bool act = valid;
    if (MODE != MODE_DIAG) act = act && (fl & F_ACTIVE) && !(fl & (F_FROZEN | F_HOLD));
    const int nth = P.nth;
    const T dphi = P.dphi;

    // ---- Philox normals of this body and step, early so their latency hides
    // behind the loads: lane 1 draws block 0 (translation), the other lanes
    // block 1 (orientation) (src/random.jl:75-100)
    T nz[2] = {T(0), T(0)};
    if (MODE == MODE_FUSED && P.has_noise)
        philox_pair<T>(P.k0, P.k1, (uint32_t)(gg - P.body_off + 1), (uint64_t)clk, l == 1 ? 0u : 1u, nz[0], nz[1]);

    // ---- stage the neighbour records in shared memory (cp.async)
    const bool contact = act && (fl & F_CONTACT);
    const int cnt = contact ? min(cnt_raw, d.cap) : 0;
    auto stage_batch = [&](int base) {
        const int npre = min(cnt - base, NBMAX);
        __syncwarp();  // every lane is done with the previous contents
#pragma unroll
        for (int u = 0; u < IDS; ++u) {
            const int q = l + u * L;
            if (q < npre) {
                const int j = base == 0 ? ids[u] : ldcg(d.nb_idx + (size_t)gg * d.cap + base + q);
                const T* src = rc + (size_t)j * RECW;
#pragma unroll
                for (int c = 0; c < CH16; ++c) cp_async16(snb + q * RECW + c * (16 / sizeof(T)), src + c * (16 / sizeof(T)));
            }
        }
        cp_async_commit();
    };
    stage_batch(0);
    int staged_base = 0;

    const int wv = unpack_w(wf);
    const int ti = wv & 7;
    const int pi = wv >> 3;

    T R[S], R1[S], C1[S], S1[S];
    T R2[S];  // R'' (user terms only)
    unsigned vmask = 0;
    const int nch = ONE ? 1 : (nth + L * S - 1) / (L * S);

    // the warp's walk slots: also the transposition buffer of the tensor-core contractions
    T* wbase = stage + (size_t)BPW * (1 + NBMAX) * RECW + desc_slot_bytes<T>() / sizeof(T);
    const float* mtab = MMA ? reinterpret_cast<const float*>(tab) + BASIS_NODES * KM * 4 : nullptr;

    // own lab coefficients are read from the staged record (modes outer,
    // nodes inner; per node the same operations as one recurrence per node)
    auto synth = [&](int ch) {
        vmask = 0;
        if constexpr (MMA_S) {
#pragma unroll
            for (int sl = 0; sl < S; ++sl) {
                const int k = l + L * sl;
                const bool v = k < nth;
                C1[sl] = v ? __ldg(d.cs + 2 * k) : T(1);
                S1[sl] = v ? __ldg(d.cs + 2 * k + 1) : T(0);
                if (v) vmask |= 1u << sl;
            }
            synth_mma(reinterpret_cast<const float*>(stage), reinterpret_cast<float*>(wbase), mtab, lane,
                      reinterpret_cast<float(&)[5]>(R), reinterpret_cast<float(&)[5]>(R1));
#pragma unroll
            for (int sl = 0; sl < S; ++sl)
                if (!(vmask & (1u << sl))) R[sl] = R1[sl] = T(0);
            return;
        }
        T cc[S], ss[S];
#pragma unroll
        for (int sl = 0; sl < S; ++sl) {
            const int k = ch * L * S + l + L * sl;
            const bool v = k < nth;
            const T c1 = v ? __ldg(d.cs + 2 * k) : T(1);
            const T s1 = v ? __ldg(d.cs + 2 * k + 1) : T(0);
            C1[sl] = c1;
            S1[sl] = s1;
            cc[sl] = c1;
            ss[sl] = s1;
            R[sl] = a0r;
            R1[sl] = T(0);
            R2[sl] = T(0);
            if (v) vmask |= 1u << sl;
        }
#pragma unroll
        for (int m = 0; m < KM; ++m) {
            const T al = own[r_al(m)], be = own[r_be(m)];
            const T n = T(m + 2);
#pragma unroll
            for (int sl = 0; sl < S; ++sl) {
                if constexpr (TAB_SYNTH) {
                    const int k = l + L * sl;
                    const auto t = lds4(tab + ((vmask & (1u << sl)) ? k : 0) * KM * 4 + m * 4);
                    R[sl] += al * t.x + be * t.y;
                    R1[sl] += be * t.z - al * t.w;
                } else {
                    const T cn = cc[sl] * C1[sl] - ss[sl] * S1[sl];
                    ss[sl] = ss[sl] * C1[sl] + cc[sl] * S1[sl];
                    cc[sl] = cn;
                    R[sl] += al * cc[sl] + be * ss[sl];
                    R1[sl] += n * (be * cc[sl] - al * ss[sl]);
                    if constexpr (USER) R2[sl] -= (n * n) * (al * cc[sl] + be * ss[sl]);
                }
            }
        }
#pragma unroll
        for (int sl = 0; sl < S; ++sl)
            if (!(vmask & (1u << sl))) R[sl] = R1[sl] = R2[sl] = T(0);
    };

    cp_async_wait_group<1>();  // the own record (the neighbour copies may still fly)
    __syncwarp();
    // ---- pass 1: contour integral Q = sum_k sqrt(R^2 + R'^2) dphi
    T Qp = T(0);
    for (int ch = 0; ch < nch; ++ch) {
        synth(ch);
#pragma unroll
        for (int sl = 0; sl < S; ++sl)
            if (vmask & (1u << sl)) {
                T q, iq;
                norm_inv(R[sl] * R[sl] + R1[sl] * R1[sl], q, iq);
                Qp += q;
            }
    }
    const T Q = group_sum<L>(Qp) * dphi;
    // user body terms: integrals Q_j = sum over the nodes of q_j(R, R', R'') dphi
    T UQ[MUT][fcc_user::MAX_M];
    if constexpr (USER) {
        static_assert(ONE, "user terms run in single-chunk kernels");
#pragma unroll
        for (int u = 0; u < MUT; ++u) {
#pragma unroll
            for (int j = 0; j < fcc_user::MAX_M; ++j) UQ[u][j] = T(0);
            if (u >= P.nub || !((P.ub_mask[u] >> ti) & 1u)) continue;
#pragma unroll
            for (int sl = 0; sl < S; ++sl)
                if (vmask & (1u << sl)) {
                    T q[fcc_user::MAX_M] = {};
                    fcc_user::body_q<T>(P.ub_id[u], R[sl], R1[sl], R2[sl], P.ub_a[u], P.ub_b[u], q);
#pragma unroll
                    for (int j = 0; j < fcc_user::MAX_M; ++j) UQ[u][j] += q[j];
                }
#pragma unroll
            for (int j = 0; j < fcc_user::MAX_M; ++j) UQ[u][j] = group_sum<L>(UQ[u][j]) * dphi;
        }
    }

    // ---- body terms: W = sum_t dF_t/dQ * dphi, E = e_1 + (e_2 + ...)
    T W = T(0), E = T(0);
    {
        const int nbt = P.nbt;
        for (int q = 0; q < nbt; ++q) {
            if (!(P.bt_mask[q] & (1u << ti))) continue;
            const T a = P.bt_a[q];
            W += P.bt_kind[q] == BT_TENSION ? a : a * (T(2) * (Q - P.bt_b[q] * r0));
        }
        for (int q = nbt - 1; q >= 0; --q) {
            if (!(P.bt_mask[q] & (1u << ti))) continue;
            const T a = P.bt_a[q];
            const T dq = Q - P.bt_b[q] * r0;
            E = (P.bt_kind[q] == BT_TENSION ? a * Q : a * (dq * dq)) + E;
        }
        W *= dphi;
    }
    // user body terms: energies F_u(Q) and node weights UW = dF_u/dQ_j dphi
    T UW[MUT][fcc_user::MAX_M];
    if constexpr (USER) {
#pragma unroll
        for (int u = 0; u < MUT; ++u) {
#pragma unroll
            for (int j = 0; j < fcc_user::MAX_M; ++j) UW[u][j] = T(0);
            if (u >= P.nub || !((P.ub_mask[u] >> ti) & 1u)) continue;
            T dF[fcc_user::MAX_M] = {};
            fcc_user::body_dF<T>(P.ub_id[u], UQ[u], r0, ti + 1, P.ub_a[u], P.ub_b[u], dF);
#pragma unroll
            for (int j = 0; j < fcc_user::MAX_M; ++j) UW[u][j] = dF[j] * dphi;
            E += fcc_user::body_F<T>(P.ub_id[u], UQ[u], r0, ti + 1, P.ub_a[u], P.ub_b[u]);
        }
    }

    // ---- pass 2: contact pressure, contour gradients, force/torque and pullback partials
    T fx = T(0), fy = T(0), tt = T(0);
    T gl[NCM];  // pullback accumulators: live only from the gradient section on (one chunk)
    if (!ONE) {
#pragma unroll
        for (int r = 0; r < NCM; ++r) gl[r] = T(0);
    }

    cp_async_wait_all();
    __syncwarp();
    const int maxc = __reduce_max_sync(FULL, cnt);
    const T Lx = P.Lx, Ly = P.Ly, iLx = P.invLx, iLy = P.invLy, crange = P.crange;
    const bool rewrap = P.rewrap != 0;

    T GRs[S], GDs[S];  // node gradients of the tensor-core pullback (0 beyond the contour; one chunk)
    for (int ch = 0; ch < nch; ++ch) {
        if (!ONE) synth(ch);
        T p[S];
#pragma unroll
        for (int sl = 0; sl < S; ++sl) p[sl] = T(0);
        // per lane and node slot (R, cos, sin, pressure) for the hit walk
        T* wsl = stage + (size_t)BPW * (1 + NBMAX) * RECW + desc_slot_bytes<T>() / sizeof(T) + (size_t)lane * S * 4;
        if (FCC_WALK_SMEM && S <= slots_of(L) && maxc > 0) {
#pragma unroll
            for (int sl = 0; sl < S; ++sl) {
                wsl[sl * 4] = R[sl];
                wsl[sl * 4 + 1] = C1[sl];
                wsl[sl * 4 + 2] = S1[sl];
                wsl[sl * 4 + 3] = T(0);
            }
        }
        constexpr bool WS = FCC_WALK_SMEM && S <= slots_of(L);
        if (maxc > 0) {
            // neighbours in batches of the stage (one batch unless a list is long)
            constexpr int QB = 64 / S;  // neighbours per 64-bit hit mask
            for (int base = 0; base < maxc; base += NBMAX) {
                if (base != staged_base) {  // lists longer than the stage: restage
                    stage_batch(base);
                    cp_async_wait_all();
                    __syncwarp();
                    staged_base = base;
                }
                const int qn = min(maxc - base, NBMAX);
                for (int q0 = 0; q0 < qn; q0 += QB) {
                    // (1) bounding-circle test of every node against every staged
                    // neighbour: bit (q - q0) * S + slot of a 64-bit hit mask
                    unsigned long long hm = 0;
                    const int q1 = min(qn, q0 + QB);
                    for (int qq = q0; qq < q1; ++qq) {
                        if (base + qq < cnt) {
                            T xj, yj, rmj, wj;
                            lds_head(snb + qq * RECW, xj, yj, rmj, wj);
                            const T dxc = minimum_image_fast(xi - xj, Lx, iLx);
                            const T dyc = minimum_image_fast(yi - yj, Ly, iLy);
                            const T lim = rmj + crange;
                            const T lim2 = lim * lim;
                            unsigned m = 0;  // this neighbour's hits over the lane's node slots
#pragma unroll
                            for (int sl = 0; sl < S; ++sl) {
                                T dx = R[sl] * C1[sl] + dxc, dy = R[sl] * S1[sl] + dyc;
                                if (rewrap) {
                                    dx = minimum_image_fast(dx, Lx, iLx);
                                    dy = minimum_image_fast(dy, Ly, iLy);
                                }
                                m |= (dx * dx + dy * dy <= lim2) ? (1u << sl) : 0u;
                            }
                            hm |= (unsigned long long)(m & vmask) << ((qq - q0) * S);
                        }
                    }
                    // (2) every lane walks its own hits in (neighbour, node) order, so
                    // each node sums its neighbours' g(d) in list order
                    // (src/energies/contact.jl:309-322)
                    // g(d) of one hit (bit (q - q0) * S + slot of the mask)
                    auto hit_value = [&](int bit, int& sl) -> T {
                        const int qq = q0 + bit / S;
                        sl = bit - (bit / S) * S;
                        const T* nrec = snb + qq * RECW;
                        T xj, yj, rmj, wj;
                        lds_head(nrec, xj, yj, rmj, wj);
                        const T dxc = minimum_image_fast(xi - xj, Lx, iLx);
                        const T dyc = minimum_image_fast(yi - yj, Ly, iLy);
                        const int wjv = unpack_w(wj);
                        const T cAj = P.cA[(wjv >> 3) == pi ? 1 : 0][ti][wjv & 7];
                        T rr, rcs, rsn;
                        if constexpr (WS) {
                            const auto e = lds4(wsl + sl * 4);
                            rr = e.x, rcs = e.y, rsn = e.z;
                        } else {
                            rr = R[0], rcs = C1[0], rsn = S1[0];
#pragma unroll
                            for (int u = 1; u < S; ++u)
                                if (sl == u) rr = R[u], rcs = C1[u], rsn = S1[u];
                        }
                        T dx = rr * rcs + dxc;
                        T dy = rr * rsn + dyc;
                        if (rewrap) {
                            dx = minimum_image_fast(dx, Lx, iLx);
                            dy = minimum_image_fast(dy, Ly, iLy);
                        }
                        const T d2 = dx * dx + dy * dy;
                        T dist = T(0), cp = T(1), sp = T(0);
                        if (d2 > T(0)) {  // direction of u - r_j (psi = 0 at u = r_j, like atan(0, 0))
                            T inv;
                            norm_inv(d2, dist, inv);
                            cp = dx * inv;
                            sp = dy * inv;
                        }
                        const T dd = radius_at(nrec, cp, sp) - dist;
                        // pair coupling of the terms (src/energies/contact.jl:267-293)
                        T gv = dd >= T(0) ? cAj : T(0);
                        if (dd > T(0)) gv += P.cB[ti] * dd;
                        if constexpr (USER) {
#pragma unroll
                            for (int u = 0; u < MUT; ++u)
                                if (u < P.nuc && ((P.uc_mask[u] >> ti) & 1u))
                                    gv += fcc_user::contact_g<T>(P.uc_id[u], dd, ti + 1, (wjv & 7) + 1, (wjv >> 3) == pi,
                                                                P.uc_a[u], P.uc_b[u]);
                        }
                        return gv;
                    };
                    while (hm) {
                        const int bit = __ffsll((long long)hm) - 1;
                        hm &= hm - 1;
                        int sl;
                        const T gv = hit_value(bit, sl);
                        if constexpr (WS) {
                            wsl[sl * 4 + 3] += gv;
                        } else {
#pragma unroll
                            for (int u = 0; u < S; ++u)
                                if (sl == u) p[u] += gv;
                        }
                    }
                }
            }
            if constexpr (WS) {
#pragma unroll
                for (int sl = 0; sl < S; ++sl) p[sl] = wsl[sl * 4 + 3];
            }
        }
        if (ONE && !MMA) {
#pragma unroll
            for (int r = 0; r < NCM; ++r) gl[r] = T(0);
        }
        // contour gradients of node k: GR = W R/q + p dphi R, GD = W R'/q, GDD = 0
#pragma unroll
        for (int sl = 0; sl < S; ++sl) {
            GRs[sl] = GDs[sl] = T(0);
            if (!(vmask & (1u << sl))) continue;
            const T r = R[sl], r1 = R1[sl], c1 = C1[sl], s1 = S1[sl];
            T q, iq;
            norm_inv(r * r + r1 * r1, q, iq);
            const T pw = p[sl] * dphi;
            T GRk = W * r * iq + pw * r;
            T GDk = W * r1 * iq;
            T GDDk = T(0);
            if constexpr (USER) {
#pragma unroll
                for (int u = 0; u < MUT; ++u) {
                    if (u >= P.nub || !((P.ub_mask[u] >> ti) & 1u)) continue;
                    T dq[fcc_user::MAX_M][3] = {};
                    fcc_user::body_dq<T>(P.ub_id[u], r, r1, R2[sl], P.ub_a[u], P.ub_b[u], dq);
#pragma unroll
                    for (int j = 0; j < fcc_user::MAX_M; ++j) {
                        GRk += UW[u][j] * dq[j][0];
                        GDk += UW[u][j] * dq[j][1];
                        GDDk += UW[u][j] * dq[j][2];
                    }
                }
            }
            fx += pw * (r * c1 + r1 * s1);
            fy += pw * (r * s1 - r1 * c1);
            tt += (-pw * r) * r1;
            if constexpr (MMA) {
                GRs[sl] = GRk;
                GDs[sl] = GDk;
            } else {
            gl[0] += GRk;
            if constexpr (TAB_PULL) {
                const int k = l + L * sl;
#pragma unroll
                for (int m = 0; m < KM; ++m) {
                    const auto t = lds4(tab + (k * KM + m) * 4);
                    if constexpr (USER) {  // R'' rows: -n^2 cos, -n^2 sin
                        const T n = T(m + 2);
                        gl[1 + m] += t.x * GRk - t.w * GDk - (n * t.z) * GDDk;
                        gl[1 + KM + m] += t.y * GRk + t.z * GDk - (n * t.w) * GDDk;
                    } else {
                        gl[1 + m] += t.x * GRk - t.w * GDk;
                        gl[1 + KM + m] += t.y * GRk + t.z * GDk;
                    }
                }
            } else {
                T c = c1, sn = s1;
#pragma unroll
                for (int m = 0; m < KM; ++m) {
                    const T n = T(m + 2);
                    const T cn = c * c1 - sn * s1;
                    sn = sn * c1 + c * s1;
                    c = cn;
                    if constexpr (USER) {
                        gl[1 + m] += c * GRk - n * sn * GDk - (n * n) * c * GDDk;
                        gl[1 + KM + m] += sn * GRk + n * c * GDk - (n * n) * sn * GDDk;
                    } else {
                        gl[1 + m] += c * GRk - n * sn * GDk;
                        gl[1 + KM + m] += sn * GRk + n * c * GDk;
                    }
                }
            }
            }
            if (MODE == MODE_DIAG && act) {
                const int k = ch * L * S + l + L * sl;
                const size_t o = (size_t)g * nth + k;
                d.P[o] = p[sl];
                d.GR[o] = GRk;
                d.GD[o] = GDk;
                d.GDD[o] = GDDk;
            }
        }
    }

    if constexpr (MMA) {
        pullback_mma(reinterpret_cast<const float(&)[5]>(GRs), reinterpret_cast<const float(&)[5]>(GDs),
                     reinterpret_cast<float*>(wbase), mtab, lane);
    } else {
        (void)GRs;
        (void)GDs;
    }
    fx = group_sum<L>(fx);
    fy = group_sum<L>(fy);
    tt = group_sum<L>(tt);
    // dE/da0 and the lane's mode gradients of the lab frame (/ R0)
    T gl0, gA[MPL], gB[MPL];
    if constexpr (MMA) {
        const float* pb = reinterpret_cast<const float*>(wbase);
        const int b = lane / L;
        gl0 = pullback_entry(pb, b, 0);
#pragma unroll
        for (int u = 0; u < MPL; ++u) {
            const int m = l + u * L;
            gA[u] = m < KM ? pullback_entry(pb, b, 1 + m) : T(0);
            gB[u] = m < KM ? pullback_entry(pb, b, 1 + KM + m) : T(0);
        }
    } else {
#pragma unroll
        for (int r = 0; r < NCM; ++r) gl[r] = group_sum<L>(gl[r]);
        gl0 = gl[0];
        lane_mode_grads<T, L>(gl, l, gA, gB);
    }

    // ---- bond forces on the centre (every lane of the body, no shuffles)
    if (act && (P.nbd > 0 || (USER && P.nubd > 0))) {
        const int bc = __ldg(d.bd_count + g);
        T bx = T(0), by = T(0);
        for (int q = 0; q < bc; ++q) {
            const int j = __ldg(d.bd_idx + (size_t)g * d.bcap + q);
            T xj, yj, rmj, wj;
            load_head(rc + (size_t)j * RECW, xj, yj, rmj, wj);
            const int tj = unpack_w(wj) & 7;
            const T d0 = minimum_image_exact(sub_rn(xi, xj), Lx);
            const T d1 = minimum_image_exact(sub_rn(yi, yj), Ly);
            T a0 = T(0), a1 = T(0);
            for (int u = P.nbd - 1; u >= 0; --u) {
                const uint32_t mk = P.bd_mask[u];
                if (!((mk >> ti) & 1u) || !((mk >> tj) & 1u)) continue;
                const T rr = t_sqrt(d0 * d0 + d1 * d1);
                const T k = P.bd_k[u], rb = P.bd_r0[u];
                const T f = rr > T(0) ? k * (T(1) - rb / rr) : (rb == T(0) ? k : T(0));
                a0 = f * d0 + a0;
                a1 = f * d1 + a1;
            }
            if constexpr (USER) {
#pragma unroll
                for (int u = 0; u < MUT; ++u) {
                    if (u >= P.nubd || !((P.ubd_mask[u] >> ti) & 1u) || !((P.ubd_mask[u] >> tj) & 1u)) continue;
                    T hx, hy;
                    fcc_user::bond_grad<T>(P.ubd_id[u], d0, d1, ti + 1, tj + 1, P.ubd_a[u], P.ubd_b[u], hx, hy);
                    a0 += hx;
                    a1 += hy;
                }
            }
            bx += a0;
            by += a1;
        }
        fx += bx;
        fy += by;
    }

    if (MODE == MODE_FORCES || MODE == MODE_DIAG) {
        if (act) {
            if (l == 0) {
                d.gx[g] = fx;
                d.gy[g] = fy;
                d.gth[g] = tt;
                d.E[g] = E;
            }
#pragma unroll
            for (int r = 0; r < NCM; ++r)
                if ((r & (L - 1)) == l) {
                    T v;
                    if constexpr (MMA) v = pullback_entry(reinterpret_cast<const float*>(wbase), lane / L, r);
                    else v = gl[r];
                    d.glab[(size_t)g * NCM + r] = v;
                }
        }
        if (MODE == MODE_DIAG && act) {
            // body-frame gradient gcoef (src/gradients.jl:347-362), frame = true
            const T* cf = d.coef + (size_t)g * NCM;
            const T a0 = ldcg(cf);
            const T ga0 = r0 * gl0;
            const T h0 = ga0 / (T(2) * a0);
            const T tho = th;
#pragma unroll
            for (int u = 0; u < MPL; ++u) {
                const int m = l + u * L;
                if (m >= P.K) continue;
                const T ga = gA[u] * r0, gb = gB[u] * r0;
                T so, co;
                t_sincos(T(m + 2) * tho, &so, &co);
                const T a = ldcg(cf + 1 + m), b = ldcg(cf + 1 + KM + m);
                d.gcoef[(size_t)g * NCM + 1 + m] = ga * co + gb * so - h0 * a;
                d.gcoef[(size_t)g * NCM + 1 + KM + m] = -ga * so + gb * co - h0 * b;
            }
            if (l == 0) d.gcoef[(size_t)g * NCM] = ga0;
        }
        return;
    }

    // the last step's centre gradients and body energy stay readable, as the
    // reference's sim.grad does after step!
    if (act && l == 0) {
        d.gx[g] = fx;
        d.gy[g] = fy;
        d.gth[g] = tt;
        d.E[g] = E;
    }
    if (valid && !act) carry_record_staged<T, L>(d, g, l, par, own);
    update_body<T, L>(d, P, act, g, s, l, par, clk, xi, yi, wf, th, r0, ti, fx, fy, tt, gl0, gA, gB, pre, fl, nz, false,
                      rbp);
}

// Phase B of the split step: displacement with parent drag + update of the
// bodies of warp group `wg`, from the forces phase A stored.
template <class T, int L>
__device__ __forceinline__ void update_warp_split(const DevPtrs<T>& d, int wg, int par, const SimDesc<T>* sim0,
                                                  int* rbp) {
    constexpr int BPW = 32 / L;
    const int lane = threadIdx.x & 31;
    const int l = lane & (L - 1);
    const int g = wg * BPW + lane / L;
    int s = 0;
    if (!sim0) {
        const int gf = wg * BPW;
        s = gf < d.Ntot ? __ldg(d.sim_of + gf) : -1;
        if (s < 0) return;
    }
    const SimDesc<T>& P = sim0 ? *sim0 : d.sims[s];
    const bool valid = sim0 ? g < d.Ntot : g < P.body_off + P.n;
    const int gg = valid ? g : (sim0 ? 0 : wg * BPW);
    const int fl = ldcg(d.flags + s);
    const bool act = valid && (fl & F_ACTIVE) && !(fl & (F_FROZEN | F_HOLD));
    const long long clk = ldcg(d.clock + s);
    T rv[RECW];
    load_rec(rec_cur(d, par) + (size_t)gg * RECW, rv);
    if (valid && !act) carry_record<T, L>(d, g, l, par, rv);
    T nz[2] = {T(0), T(0)};
    if (P.has_noise)
        philox_pair<T>(P.k0, P.k1, (uint32_t)(gg - P.body_off + 1), (uint64_t)clk, l == 1 ? 0u : 1u, nz[0], nz[1]);
    const int ti = unpack_w(rv[R_W]) & 7;
    const T r0 = __ldg(d.R0 + gg);
    UpdatePre<T, L> pre;
    load_update_pre(d, gg, l, P.K, pre);
    T gl[NCM];
#pragma unroll
    for (int r = 0; r < NCM; ++r) gl[r] = ldcg(d.glab + (size_t)gg * NCM + r);
    const T fx = ldcg(d.gx + gg), fy = ldcg(d.gy + gg), tt = ldcg(d.gth + gg);
    T gA[UpdatePre<T, L>::MPL], gB[UpdatePre<T, L>::MPL];
    lane_mode_grads<T, L>(gl, l, gA, gB);
    update_body<T, L>(d, P, act, g, s, l, par, clk, rv[R_X], rv[R_Y], rv[R_W], rv[R_TH], r0, ti, fx, fy, tt, gl[0], gA,
                      gB, pre, fl, nz, true, rbp);
}

template <class T>
__device__ __forceinline__ int book_one(const DevPtrs<T>& d, int s) {
    int any = 0;
    int f = ldcg(d.flags + s);
    if ((f & F_ACTIVE) && !(f & (F_FROZEN | F_HOLD))) {
        const long long c = ldcg(d.clock + s) + 1;
        d.clock[s] = c;
        if (d.stop && c >= ldcg(d.stop + s)) {
            // step limit reached: hold; F_REBUILD stays for the host's
            // rebuild decision when it releases the simulation
            f = (f & ~F_NEED) | F_HOLD;
        } else {
            const bool need = (f & F_CONTACT) && ((f & F_REBUILD) || !(f & F_VALID) || d.sims[s].skin == T(0));
            f &= ~(F_REBUILD | F_NEED);
            if (need) {
                f |= F_NEED;
                any = 1;
            }
        }
    } else {
        f &= ~F_NEED;
    }
    d.flags[s] = f;
    return any;
}

// A launch that advances one simulation with no step limit: its flags and
// clock are known to every block (decided by every block at each flat
// barrier, ticked locally), so the bookkeeping needs no global reads.
template <class T>
__device__ __forceinline__ bool lone_sim(const DevPtrs<T>& d) {
    return d.nsims == 1 && d.stop == nullptr;
}

// End of a step's closing barrier: tick the clocks of the simulations that
// stepped and decide the rebuilds of the next step (skin exceeded, list
// invalid, or skin = 0: src/simulation.jl:132-142).  Returns (in thread 0)
// the code: whether some simulation rebuilds at the next step, and for a
// lone simulation its new flags (<< 1).  `rebuilds`: blocks whose bodies
// exceeded their skin in this step.  A pool's last block to arrive runs it
// before releasing the barrier; for a lone simulation every block runs it on
// the flat barrier's counter value, with no global memory (its flags are
// block-local, its descriptor `P` in shared memory), and block 0 writes its
// global flags and clock (lone_book_writes).
template <class T>
__device__ int bookkeeping(const DevPtrs<T>& d, const BarrierLocal& bl, unsigned rebuilds, const SimDesc<T>* P) {
    if (lone_sim(d)) {
        if (threadIdx.x != 0) return 0;
        int f = bl.flags, need = 0;
        if ((f & F_ACTIVE) && !(f & (F_FROZEN | F_HOLD))) {
            need = (f & F_CONTACT) && (rebuilds != 0 || (f & F_REBUILD) || !(f & F_VALID) || P->skin == T(0));
            f &= ~(F_REBUILD | F_NEED);
            if (need) f |= F_NEED;
        } else {
            f &= ~F_NEED;
        }
        return need | ((f & 0xff) << 1);
    }
    if (d.nsims == 1) return threadIdx.x == 0 ? book_one(d, 0) : 0;  // one thread, no block barrier
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < d.nsims; s += blockDim.x)
        if (book_one(d, s)) s_any = 1;
    __syncthreads();
    return s_any;
}

// The global side of a lone simulation's bookkeeping, written by one block
// once the step barrier is passed: the host reads the clock and flags after
// the launch, the rebuild phases read F_NEED only after the first rebuild
// barrier (phase_count takes the decision from the block's own copy).  The
// flag updates are atomic: they keep the bits other blocks set (non-finite,
// overflow).
template <class T>
__device__ __forceinline__ void lone_book_writes(const DevPtrs<T>& d, const BarrierLocal& bl, int code) {
    const int f = bl.flags;
    if ((f & F_ACTIVE) && !(f & (F_FROZEN | F_HOLD))) {
        d.clock[0] = bl.clock + 1;
        atomicAnd(d.flags, ~(F_REBUILD | F_NEED));
        if (code & 1) atomicOr(d.flags, F_NEED);
    } else {
        atomicAnd(d.flags, ~F_NEED);
    }
}

// ============================================================= kernels ==
template <class T>
__device__ __forceinline__ bool rebuild_prologue(const DevPtrs<T>& d, int par, int tid, int nthr, BarrierLocal& bl,
                                                 const SimDesc<T>* sim0, int* wl_area, int wl_cap) {
    // the phases set F_VALID / F_FROZEN: a lone simulation's flags are re-read
    auto keep = [&](unsigned) { return lone_sim(d) ? (bl.any | ((ldcg(d.flags) & 0xff) << 1)) : -1; };
    if (FCC_FLAT_BARRIER && lone_sim(d)) {
        // a lone simulation: flat barriers, and each block tracks the flags the
        // phases set (F_VALID from the scan, F_FROZEN from an overflowing list,
        // voted at the last barrier) instead of re-reading them
        phase_count(d, par, tid, nthr, nullptr, bl.any);
        if (!flat_barrier(d.sync, bl, 0u)) return false;
        phase_scan(d, nullptr);
        if (!flat_barrier(d.sync, bl, 0u)) return false;
        phase_scatter(d, tid, nthr, nullptr);
        if (!flat_barrier(d.sync, bl, 0u)) return false;
        phase_sort(d, tid, nthr, nullptr);
        if (!flat_barrier(d.sync, bl, 0u)) return false;
        if (threadIdx.x == 0) bl.ovf = 0;
        __syncthreads();
        phase_neighbors(d, par, tid, nthr, sim0, nullptr, &bl.ovf);
        __syncthreads();
        if (!flat_barrier(d.sync, bl, bl.ovf ? 1u : 0u)) return false;
        if (threadIdx.x == 0) {
            bl.flags |= F_VALID;
            if (bl.bits) bl.flags |= F_FROZEN;
        }
        __syncthreads();
        return true;
    }
    WorkList wl{};
    wl.m = -1;
    if (!sim0) wl = build_worklist(d, wl_area, wl_cap);
    const WorkList* wlp = wl.m >= 0 ? &wl : nullptr;
    phase_count(d, par, tid, nthr, wlp, lone_sim(d) ? bl.any : -1);
    if (!grid_barrier(d.sync, bl, keep)) return false;
    phase_scan(d, wlp);
    if (!grid_barrier(d.sync, bl, keep)) return false;
    phase_scatter(d, tid, nthr, wlp);
    if (!grid_barrier(d.sync, bl, keep)) return false;
    phase_sort(d, tid, nthr, wlp);
    if (!grid_barrier(d.sync, bl, keep)) return false;
    phase_neighbors(d, par, tid, nthr, sim0, wlp);
    return grid_barrier(d.sync, bl, keep);
}

// A single simulation's descriptor is read from shared memory (copied once per
// block); an engine holding several reads each body's from global memory.
template <class T>
__device__ __forceinline__ const SimDesc<T>* copy_desc(const DevPtrs<T>& d) {
    __shared__ __align__(16) unsigned s_desc[(sizeof(SimDesc<T>) + 3) / 4];
    if (d.nsims != 1) return nullptr;
    const unsigned* src = reinterpret_cast<const unsigned*>(d.sims);
    for (int u = threadIdx.x; u < (int)((sizeof(SimDesc<T>) + 3) / 4); u += blockDim.x) s_desc[u] = src[u];
    __syncthreads();
    return reinterpret_cast<const SimDesc<T>*>(s_desc);
}

// Dynamic shared memory of the force kernels: the FP32 mode table (one
// contour chunk of nodes), then one neighbour stage per warp.
template <class T>
__device__ __forceinline__ T* warp_stage(size_t bytes_per_warp) {
    extern __shared__ __align__(16) unsigned char fcc_smem[];
    return reinterpret_cast<T*>(fcc_smem + basis_table_bytes<T>() + (threadIdx.x >> 5) * bytes_per_warp);
}
// the whole stage area of the block (every warp's stage, in order)
template <class T>
__device__ __forceinline__ unsigned char* block_stage_of() {
    extern __shared__ __align__(16) unsigned char fcc_smem[];
    return fcc_smem + basis_table_bytes<T>();
}

// Copy the mode table of the first min(nth, BASIS_NODES) nodes, and after it
// the tensor-core fragment table, into shared memory (FP32 single-chunk
// kernels); returns the mode table, or null when unused.
template <class T, bool ONE>
__device__ __forceinline__ const T* stage_basis(const DevPtrs<T>& d) {
    extern __shared__ __align__(16) unsigned char fcc_smem[];
    if (!(sizeof(T) == 4 && ONE)) return nullptr;
    T* tab = reinterpret_cast<T*>(fcc_smem);
    const int n = min(d.nth, BASIS_NODES) * KM * 4;
    for (int u = threadIdx.x; u < n; u += blockDim.x) tab[u] = __ldg(d.basis + u);
    if (d.mtab) {  // the tensor-core fragments follow the mode table
        float* mt = reinterpret_cast<float*>(fcc_smem) + BASIS_NODES * KM * 4;
        for (int u = threadIdx.x; u < MMA_TABLE_FLOATS; u += blockDim.x) mt[u] = __ldg(d.mtab + u);
    }
    __syncthreads();
    return tab;
}

// Persistent cooperative step kernel: `nsteps` whole time steps per launch.
// Each block takes a contiguous range of warp groups (balanced bodies per SM);
// within the block the warps take them statically, or (FP32, one simulation)
// each warp its first and then the block's next untaken one.
template <class T, int L, int S, bool ONE, bool SPLIT, int BLK, int MINB, bool USER = false>
__global__ void __launch_bounds__(BLK, MINB) k_step(DevPtrs<T> d, int nsteps, int par0) {
    constexpr int WPB = BLK / 32;
    const int warp = threadIdx.x >> 5;
    const int ngroups = (d.Ntot + (32 / L) - 1) / (32 / L);
    const int g0 = (int)((long long)ngroups * blockIdx.x / gridDim.x);
    const int g1 = (int)((long long)ngroups * (blockIdx.x + 1) / gridDim.x);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    T* stage = warp_stage<T>(stage_bytes_per_warp<T, L>());
    const T* tab = stage_basis<T, ONE>(d);
    const SimDesc<T>* sim0 = copy_desc(d);
    __shared__ BarrierLocal bl;
    const bool lone = lone_sim(d);
    barrier_start(d.sync, bl, lone, d.flags, d.clock);
    int cached = -1;  // simulation whose descriptor this warp's slot holds
    // FP32 with a single simulation: the warps of a block take its warp groups
    // dynamically (measured: 1% faster at N = 16384).  Pools keep the static
    // assignment (2% faster there: a warp that moves to another simulation's
    // group re-copies the descriptor), and so does FP64 (one block of 8 warps
    // per SM: 3% faster static).
    const bool dyn = FCC_DYN && sizeof(T) == 4 && sim0 != nullptr;
    __shared__ int s_next[2];  // next untaken warp group of the block, per step parity
    if (dyn && threadIdx.x == 0) s_next[0] = g0 + WPB;
    __syncthreads();
    for (int st = 0; st < nsteps; ++st) {
        const int par = (par0 + st) & 1;
        if (bl.any) {
            // the work list of a pool lives in the warps' stage area, free
            // between the closing barrier of a step and the forces
            if (!rebuild_prologue(d, par, tid, nthr, bl, sim0, reinterpret_cast<int*>(block_stage_of<T>()),
                                  (int)(WPB * stage_bytes_per_warp<T, L>() / sizeof(int))))
                return;
            cached = -1;  // the descriptor slots were overwritten
        }
        if (dyn) {
            // a warp's first group is its own; after that it takes the block's
            // next untaken group (groups cost unequal time: contacts, hits)
            if (threadIdx.x == 0) s_next[(st + 1) & 1] = g0 + WPB;  // last used by the previous step
            for (int wg = g0 + warp; wg < g1;) {
                forces_warp<T, L, S, ONE, SPLIT ? MODE_FORCES : MODE_FUSED, USER>(d, wg, stage, par, sim0, tab,
                                                                                   cached, &bl.rebuild,
                                                                                   lone ? &bl : nullptr);
                int nx = 0;
                if ((threadIdx.x & 31) == 0) nx = atomicAdd(&s_next[st & 1], 1);
                wg = __shfl_sync(0xffffffffu, nx, 0);
            }
        } else {
            for (int wg = g0 + warp; wg < g1; wg += WPB)
                forces_warp<T, L, S, ONE, SPLIT ? MODE_FORCES : MODE_FUSED, USER>(d, wg, stage, par, sim0, tab,
                                                                                   cached, &bl.rebuild,
                                                                                   lone ? &bl : nullptr);
        }
        if (SPLIT) {
            if (!grid_barrier(d.sync, bl, [](unsigned) { return -1; })) return;
            for (int wg = g0 + warp; wg < g1; wg += WPB) update_warp_split<T, L>(d, wg, par, sim0, &bl.rebuild);
        }
        const int f0 = bl.flags;  // fixed during the step (read before thread 0 may rewrite it)
        __syncthreads();          // every warp's skin verdict is in bl.rebuild
        unsigned rb = 0;
        if (threadIdx.x == 0) {  // reported with the arrival; cleared before the next forces phase
            rb = bl.rebuild ? 1u : 0u;
            bl.rebuild = 0;
        }
        // a lone simulation that stepped ticks its block-local clock inside the
        // barrier: the next step's warps read it for their noise
        const int tick = (lone && (f0 & F_ACTIVE) && !(f0 & (F_FROZEN | F_HOLD))) ? 1 : 0;
        if (FCC_FLAT_BARRIER && lone) {
            // every block decides the next step from the same counter value;
            // block 0 writes the global flags and clock
            // (the block barrier above is the flat barrier's entry barrier)
            auto decide = [&](int) {
                const int code = bookkeeping(d, bl, bl.bits, sim0);
                if (blockIdx.x == 0) {
                    d.sync->any_need = code & 1;
                    lone_book_writes(d, bl, code);
                }
                bl.any = code & 1;
                bl.flags = (code >> 1) & 0xff;
                bl.clock += tick;
            };
            if (!flat_barrier(d.sync, bl, rb, decide, false)) return;
            continue;
        }
        if (!grid_barrier(
                d.sync, bl, [&](unsigned rbs) { return bookkeeping(d, bl, rbs, sim0); }, rb,
                [&](int code) {
                    if (lone) lone_book_writes(d, bl, code);
                },
                tick))
            return;
    }
    if (FCC_FLAT_BARRIER && lone && threadIdx.x == 0) flat_end(d.sync);
}

// Self-test of the bounded barrier waits: the last block leaves without
// arriving, so the others wait for a release that never comes, first at a
// generation-word barrier on gs[0], then at a flat barrier on gs[1]; after
// SELFTEST_POLLS polls each wait records its GridSync's error and returns.
// Nothing else runs.
constexpr long long SELFTEST_POLLS = 1ll << 14;
__global__ void k_barrier_selftest(GridSync* gs) {
    __shared__ BarrierLocal bl;
    barrier_start(gs, bl, false, nullptr, nullptr);
    if (blockIdx.x == gridDim.x - 1) return;
    grid_barrier<SELFTEST_POLLS>(gs, bl, [](unsigned) { return -1; });
    flat_barrier<SELFTEST_POLLS>(gs + 1, bl, 0u);
}

// compute_gradients! (src/simulation.jl:150-158): forces and every gradient
// buffer of the current state, no update.
template <class T, int L, int S, bool ONE, bool USER = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_gradients(DevPtrs<T> d, int par) {
    const int wpb = blockDim.x >> 5;
    const int wg = blockIdx.x * wpb + (threadIdx.x >> 5);
    const int ngroups = (d.Ntot + (32 / L) - 1) / (32 / L);
    T* stage = warp_stage<T>(stage_bytes_per_warp<T, L>());
    const T* tab = stage_basis<T, ONE>(d);
    const SimDesc<T>* sim0 = copy_desc(d);
    int cached = -1;
    if (wg < ngroups) forces_warp<T, L, S, ONE, MODE_DIAG, USER>(d, wg, stage, par, sim0, tab, cached, nullptr, nullptr);
}

// Stand-alone rebuild phases (update_neighbors!, and the stateless neighbour
// build), one launch per phase.
template <class T>
__global__ void k_phase_count(DevPtrs<T> d, int par) {
    if (ldcg(&d.sync->any_need))
        phase_count<T>(d, par, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, nullptr);
}
template <class T>
__global__ void k_phase_scan(DevPtrs<T> d) {
    if (ldcg(&d.sync->any_need)) phase_scan<T>(d, nullptr);
}
template <class T>
__global__ void k_phase_scatter(DevPtrs<T> d) {
    if (ldcg(&d.sync->any_need))
        phase_scatter<T>(d, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, nullptr);
}
template <class T>
__global__ void k_phase_sort(DevPtrs<T> d) {
    if (ldcg(&d.sync->any_need))
        phase_sort<T>(d, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, nullptr);
}
template <class T>
__global__ void k_phase_neighbors(DevPtrs<T> d, int par) {
    if (ldcg(&d.sync->any_need))
        phase_neighbors<T>(d, par, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, nullptr, nullptr);
}

// Skin check of the current state (skin_check_kernel!, src/neighbors.jl:188-194).
template <class T>
__global__ void k_skin_check(DevPtrs<T> d, int par) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= d.Ntot) return;
    const int s = __ldg(d.sim_of + g);
    if (s < 0) return;
    const int f = ldcg(d.flags + s);
    if (!(f & F_CONTACT) || !(f & F_VALID)) return;
    const SimDesc<T>& P = d.sims[s];
    if (!(P.skin > T(0))) return;
    const T* r = rec_cur(d, par) + (size_t)g * RECW;
    const T dx = minimum_image_exact(sub_rn(ldcg(r + R_X), ldcg(d.x0 + g)), P.Lx);
    const T dy = minimum_image_exact(sub_rn(ldcg(r + R_Y), ldcg(d.y0 + g)), P.Ly);
    const T grow = sub_rn(ldcg(r + R_RMAX), ldcg(d.rmax0 + g));
    const T delta = add_rn(t_sqrt(add_rn(mul_rn(dx, dx), mul_rn(dy, dy))), grow > T(0) ? grow : T(0));
    if (mul_rn(T(2), delta) > P.skin) atomicOr(&d.flags[s], F_REBUILD);
}

// Decide which simulations rebuild in the stand-alone update_neighbors!.
template <class T>
__global__ void k_prepare_rebuild(DevPtrs<T> d, int force) {
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < d.nsims; s += blockDim.x) {
        int f = d.flags[s];
        const bool need = (f & F_ACTIVE) && (f & F_CONTACT) &&
                          (force || (f & F_REBUILD) || !(f & F_VALID) || d.sims[s].skin == T(0));
        f &= ~(F_REBUILD | F_NEED);
        if (need) {
            f |= F_NEED;
            s_any = 1;
        }
        d.flags[s] = f;
    }
    __syncthreads();
    if (threadIdx.x == 0) d.sync->any_need = s_any;
}

// After a stand-alone rebuild: the next step rebuilds again only with skin = 0.
template <class T>
__global__ void k_finish_rebuild(DevPtrs<T> d) {
    for (int s = threadIdx.x; s < d.nsims; s += blockDim.x) {
        int f = d.flags[s];
        const bool need = (f & F_ACTIVE) && (f & F_CONTACT) && !(f & F_FROZEN) && d.sims[s].skin == T(0);
        f &= ~(F_REBUILD | F_NEED);
        if (need) f |= F_NEED;
        d.flags[s] = f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int any = 0;
        for (int s = 0; s < d.nsims; ++s) any |= (d.flags[s] & F_NEED) ? 1 : 0;
        d.sync->any_need = any;
    }
}

// Simulation set-up and set_state: enforce_shape! (FP64 sums) and the lab
// frame of the given body state into rec[par] (src/simulation.jl:102-103,
// src/dynamics.jl:44-64, src/geometry.jl:208-227).  One thread per body.
// Bodies g0 .. g0+n-1; the inputs are indexed from i = 0 and are the caller's
// host values as they crossed the ABI (double), in the reference's
// coefficient layout: in_nc values per body, [a0; a_2..a_{in_K+1};
// b_2..b_{in_K+1}] (src/basis.jl:10-14), and the record words w = (parent <<
// 3) | type (0-based).  Each value is rounded to T here, exactly as a
// host-side conversion would round it.
// The inputs may be device memory or page-locked host memory the device
// reads directly (mapped under unified addressing): the block stages its
// bodies' coefficient rows through shared memory with consecutive threads
// reading consecutive doubles, so host reads cross PCIe in full lines.
// ix_in, iy_in (image counters; null: keep the device's) likewise.
// Launch with INIT_BLOCK threads and init_smem_bytes(in_nc) bytes.
constexpr int INIT_BLOCK = 256;
__host__ __device__ constexpr size_t init_smem_bytes(int in_nc) { return (size_t)INIT_BLOCK * in_nc * sizeof(double); }
template <class T>
__global__ void __launch_bounds__(INIT_BLOCK) k_init(DevPtrs<T> d, int par, int g0, int n, const double* __restrict__ x,
                                                    const double* __restrict__ y, const double* __restrict__ th_in,
                                                    const double* __restrict__ coef_in, int in_nc, int in_K,
                                                    const int* __restrict__ w, const int* __restrict__ ix_in,
                                                    const int* __restrict__ iy_in) {
    extern __shared__ double s_coef[];
    const int i0 = blockIdx.x * INIT_BLOCK;
    const int nb = min(INIT_BLOCK, n - i0);
    for (int u = threadIdx.x; u < nb * in_nc; u += INIT_BLOCK) s_coef[u] = coef_in[(size_t)i0 * in_nc + u];
    __syncthreads();
    const int i = i0 + threadIdx.x;
    if (i >= n) return;
    const int g = g0 + i;
    if (ix_in) d.imgx[g] = ix_in[i];
    if (iy_in) d.imgy[g] = iy_in[i];
    const int s = d.sim_of[g];
    const SimDesc<T>& P = d.sims[s];
    const int K = P.K;
    const int wi = w[i];
    const int kt = min(in_K, P.kmax[wi & 7]);  // modes above the body type's maxmode enter as zero
    T c[NCM];
    const double* ci = s_coef + (size_t)threadIdx.x * in_nc;
    c[0] = T(ci[0]);
#pragma unroll
    for (int m = 0; m < KM; ++m) {
        c[1 + m] = m < kt ? T(ci[1 + m]) : T(0);
        c[1 + KM + m] = m < kt ? T(ci[1 + in_K + m]) : T(0);
    }
    const T th_i = T(th_in[i]);
    // enforce_shape! and the lab frame with the arithmetic of the update's
    // end of step (update_body): modes spread over 8 lanes as m = lane + 8u,
    // per-lane sums in u order, lanes combined by the xor butterfly of
    // group_sum<8>, so a state written by a run and loaded again continues
    // bit for bit (for the 8-lane launch shapes)
    constexpr int LV = 8, MV = (KM + LV - 1) / LV;
    auto tree8 = [](auto* v) {  // ((v0+v4)+(v2+v6)) + ((v1+v5)+(v3+v7)), as group_sum<8>
        return ((v[0] + v[4]) + (v[2] + v[6])) + ((v[1] + v[5]) + (v[3] + v[7]));
    };
    double spl[LV];
#pragma unroll
    for (int l = 0; l < LV; ++l) {
        double sp = 0.0;
#pragma unroll
        for (int u = 0; u < MV; ++u) {
            const int m = l + u * LV;
            if (m < K) sp += (double)mode_norm(c[1 + m], c[1 + KM + m]);
        }
        spl[l] = sp;
    }
    const double ssum = tree8(spl);
    if (ssum > SHAPE_BOUND) {
        const double f = SHAPE_BOUND / ssum;
        for (int m = 0; m < K; ++m) {
            c[1 + m] = T((double)c[1 + m] * f);
            c[1 + KM + m] = T((double)c[1 + KM + m] * f);
        }
    }
    double qpl[LV];
#pragma unroll
    for (int l = 0; l < LV; ++l) {
        double qp = 0.0;
#pragma unroll
        for (int u = 0; u < MV; ++u) {
            const int m = l + u * LV;
            qp += m < K ? mode_sq(c[1 + m], c[1 + KM + m]) : 0.0;
        }
        qpl[l] = qp;
    }
    c[0] = T(sqrt(1.0 - tree8(qpl) * 0.5));
    const T r0 = d.R0[g];
    T* rn = rec_cur_mut(d, par) + (size_t)g * RECW;
    T* ro = rec_next(d, par) + (size_t)g * RECW;
    for (int r = 0; r < RECW; ++r) ro[r] = T(0);
    T s1, c1;
    t_sincos(th_i, &s1, &c1);
    T bpl[LV];
#pragma unroll
    for (int l = 0; l < LV; ++l) {
        T bp = T(0);
#pragma unroll
        for (int u = 0; u < MV; ++u) {
            const int m = l + u * LV;
            if (m >= KM) continue;
            T al = T(0), be = T(0);
            if (m < K) {
                T so, co;
                cis_pow(c1, s1, m + 2, co, so);
                to_lab(c[1 + m], c[1 + KM + m], co, so, al, be);
                bp += mode_norm(c[1 + m], c[1 + KM + m]);
            }
            rn[r_al(m)] = r0 * al;
            rn[r_be(m)] = r0 * be;
        }
        bpl[l] = bp;
    }
    const T bound = c[0] + tree8(bpl);
    rn[R_X] = T(x[i]);
    rn[R_Y] = T(y[i]);
    rn[R_RMAX] = r0 * bound;
    rn[R_A0] = r0 * c[0];
    T* tag = nullptr;
    rn[R_W] = pack_w(wi, tag);  // (parent, type)
    rn[R_TH] = th_i;
#pragma unroll
    for (int r = 0; r < NCM; ++r) d.coef[(size_t)g * NCM + r] = c[r];
}

// get_state on the device: x, y, theta of the current record, the
// body-frame coefficients and the image counters of bodies g0 .. g0+n-1,
// widened to double in the reference's layout, written to x, y, th (n each),
// coef_out (out_nc values per body, [a0; a_2..a_{out_K+1}; b_2..b_{out_K+1}])
// and ix, iy (null: skipped).  The outputs may be device memory or
// page-locked host memory the device writes directly: every output is written
// with consecutive threads on consecutive elements (the coefficients as one
// flat array), so host writes cross PCIe in full lines.  Grid-stride loops.
template <class T>
__global__ void k_store_host(DevPtrs<T> d, int par, int g0, int n, double* __restrict__ x, double* __restrict__ y,
                             double* __restrict__ th, double* __restrict__ coef_out, int out_nc, int out_K,
                             int* __restrict__ ix, int* __restrict__ iy) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    const T* rc = rec_cur(d, par);
    for (int i = tid; i < n; i += nthr) {
        const T* r = rc + (size_t)(g0 + i) * RECW;
        if (x) x[i] = (double)r[R_X];
        if (y) y[i] = (double)r[R_Y];
        if (th) th[i] = (double)r[R_TH];
        if (ix) ix[i] = d.imgx[g0 + i];
        if (iy) iy[i] = d.imgy[g0 + i];
    }
    if (coef_out) {
        const long long tot = (long long)n * out_nc;
        for (long long u = tid; u < tot; u += nthr) {
            const int i = (int)(u / out_nc), j = (int)(u - (long long)i * out_nc);
            // j = 0: a0; 1..out_K: a_{j+1}; out_K+1..2 out_K: b_{j-out_K+1}
            const int r = j == 0 ? 0 : (j <= out_K ? j : KM + (j - out_K));
            coef_out[u] = (double)d.coef[(size_t)(g0 + i) * NCM + r];
        }
    }
}

// Geometry of the current state for get_geometry: lab, labR0, rmax, and
// R, R', R'' at the nodes (src/geometry.jl:13-32, 248-257).  Outputs in the
// engine's fixed coefficient layout [a0; a_2..a_10; b_2..b_10].
template <class T>
__global__ void k_geometry(DevPtrs<T> d, int par, T* lab, T* labR0, T* R, T* dR, T* ddR, T* rmax) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= d.Ntot) return;
    const int s = d.sim_of[g];
    if (s < 0) return;
    const SimDesc<T>& P = d.sims[s];
    const T* rc = rec_cur(d, par) + (size_t)g * RECW;
    const T* cf = d.coef + (size_t)g * NCM;
    const T r0 = d.R0[g];
    const T th = rc[R_TH];
    lab[(size_t)g * NCM] = cf[0];
    labR0[(size_t)g * NCM] = rc[R_A0];
    for (int m = 0; m < KM; ++m) {
        T al = T(0), be = T(0);
        if (m < P.K) {
            T so, co;
            t_sincos(T(m + 2) * th, &so, &co);
            al = cf[1 + m] * co - cf[1 + KM + m] * so;
            be = cf[1 + m] * so + cf[1 + KM + m] * co;
        }
        lab[(size_t)g * NCM + 1 + m] = al;
        lab[(size_t)g * NCM + 1 + KM + m] = be;
        labR0[(size_t)g * NCM + 1 + m] = rc[r_al(m)];
        labR0[(size_t)g * NCM + 1 + KM + m] = rc[r_be(m)];
    }
    rmax[g] = rc[R_RMAX];
    for (int k = 0; k < P.nth; ++k) {
        const T c1 = d.cs[2 * k], s1 = d.cs[2 * k + 1];
        T c = c1, sn = s1, r = rc[R_A0], r1 = T(0), r2 = T(0);
        for (int m = 0; m < KM; ++m) {
            const T n = T(m + 2);
            const T cn = c * c1 - sn * s1;
            sn = sn * c1 + c * s1;
            c = cn;
            const T al = rc[r_al(m)], be = rc[r_be(m)];
            const T t = al * c + be * sn;
            r += t;
            r1 += n * (be * c - al * sn);
            r2 -= n * n * t;
        }
        R[(size_t)g * P.nth + k] = r;
        dR[(size_t)g * P.nth + k] = r1;
        ddR[(size_t)g * P.nth + k] = r2;
    }
}

// perimeters, areas, shape index with FP64 node sums (src/observables.jl:7-18).
// Bodies g0 .. g0+n-1, out indexed from g0.
template <class T>
__global__ void k_observables(DevPtrs<T> d, int par, int g0, int n, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = g0 + i;
    const int s = d.sim_of[g];
    if (s < 0) return;
    const SimDesc<T>& P = d.sims[s];
    const T* rc = rec_cur(d, par) + (size_t)g * RECW;
    double per = 0.0, area = 0.0;
    for (int k = 0; k < P.nth; ++k) {
        const T c1 = d.cs[2 * k], s1 = d.cs[2 * k + 1];
        T c = c1, sn = s1, r = rc[R_A0], r1 = T(0);
        for (int m = 0; m < KM; ++m) {
            const T n = T(m + 2);
            const T cn = c * c1 - sn * s1;
            sn = sn * c1 + c * s1;
            c = cn;
            const T al = rc[r_al(m)], be = rc[r_be(m)];
            r += al * c + be * sn;
            r1 += n * (be * c - al * sn);
        }
        per += sqrt((double)r * r + (double)r1 * r1);
        area += (double)r * r;
    }
    per *= (double)P.dphi;
    area *= (double)P.dphi / 2.0;
    out[3 * (size_t)i] = per;
    out[3 * (size_t)i + 1] = area;
    out[3 * (size_t)i + 2] = per / sqrt(area);
}

// philox_noise! (src/random.jl:113-130): first three normals of body i.
template <class T>
__global__ void k_noise(uint32_t k0, uint32_t k1, uint64_t draw, int n, T* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T z1, z2, z3, z4;
    philox_pair<T>(k0, k1, (uint32_t)(i + 1), draw, 0u, z1, z2);
    philox_pair<T>(k0, k1, (uint32_t)(i + 1), draw, 1u, z3, z4);
    out[3 * (size_t)i] = z1;
    out[3 * (size_t)i + 1] = z2;
    out[3 * (size_t)i + 2] = z3;
}

// Pack caller x, y, rmax into records for the stateless neighbour build.
template <class T>
__global__ void k_pack_head(T* rec, const T* x, const T* y, const T* rmax, int n) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    rec[(size_t)g * RECW + R_X] = x[g];
    rec[(size_t)g * RECW + R_Y] = y[g];
    rec[(size_t)g * RECW + R_RMAX] = rmax[g];
}

}  // namespace fcc
