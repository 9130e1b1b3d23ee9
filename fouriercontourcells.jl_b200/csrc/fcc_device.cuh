// fcc_device.cuh — device data layout and helpers of the B200 time step.
//
// Layout in HBM (all bodies of all simulations of one engine, global body
// index g; a single Simulation is an engine with one simulation):
//
//   rec[2][g][24]  geometry record, ping-pong by the parity of the engine's
//                  step counter (current = rec[par]).  Neighbours read it,
//                  so a step reads rec[par] and writes rec[par^1]:
//                    [0] x  [1] y  [2] rmax  [3] w = parent_global<<3 | (type-1)
//                    [4] R0*a0  [5 + 2m] R0*alpha_n  [6 + 2m] R0*beta_n  [23] theta
//                    (n = m + 2; alpha/beta interleaved so a mode is one 8-byte pair)
//                  (lab-frame coefficients scaled by R0, src/geometry.jl:208-227;
//                  modes n = 2..10 at fixed slots, unused modes stay zero).
//                  96 B (FP32) per body = six 16-byte vector loads.
//   coef[g][19]    body-frame coefficients [a0; a_2..a_10; b_2..b_10], owned
//                  by body g and updated in place.
//   imgx, imgy     periodic image counters (in place).
//   nb_idx[g][cap], nb_count[g]   neighbour lists, body-major like the
//                  reference's cap x N column-major matrix (neighbors.jl:110).
//   cellid/slot/perm/cstart/cstop/ccount   counting-sort cell list.
//
// Kernels never read `rec` through the non-coherent (texture) path: the
// persistent step kernel rewrites it between grid barriers.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fcc {

constexpr int KM = 9;        // shape modes n = 2..10
constexpr int NCM = 2 * KM + 1;
constexpr int RECW = 24;     // record width (values)
constexpr int MT = 8;        // max body types
constexpr int MTERM = 16;    // max terms
constexpr int MUT = 4;       // max compiled user terms of each kind (FCC_MAX_USER_TERMS)
constexpr double SHAPE_BOUND = 0.816496580927726;  // sqrt(2/3), src/dynamics.jl:26

// record slots
constexpr int R_X = 0, R_Y = 1, R_RMAX = 2, R_W = 3, R_A0 = 4, R_TH = 23;
__host__ __device__ constexpr int r_al(int m) { return 5 + 2 * m; }  // R0*alpha of mode n = m + 2
__host__ __device__ constexpr int r_be(int m) { return 6 + 2 * m; }  // R0*beta of mode n = m + 2

// per-simulation flags
enum : int {
    F_REBUILD = 1,     // skin exceeded: rebuild before the next force evaluation
    F_FROZEN = 2,      // neighbour overflow: steps do nothing until the host regrows the list
    F_VALID = 4,       // neighbour list built
    F_NEED = 8,        // rebuild at the start of the next step
    F_ACTIVE = 16,     // slot holds a simulation
    F_NONFINITE = 32,  // a body state became non-finite
    F_CONTACT = 64,    // simulation has contact terms (uses neighbour lists)
    F_HOLD = 128,      // reached its step limit: keeps its state until the host releases it
};

enum : int { BT_TENSION = 1, BT_PERIMETER = 2 };

template <class T>
struct SimDesc {
    T Lx, Ly, invLx, invLy;
    T dt, skin, nbrange, crange, dphi;  // nbrange = contact range + skin
    T wx, wy;
    int ncx, ncy, cell_off, ncells;
    int body_off, n, nth, K;
    uint32_t k0, k1;  // Philox key
    int ntypes, rewrap, has_contact, has_parent_drag, has_noise;
    int nbt, nbd;
    T v0[MT], Dr[MT], Dt[MT], mur[MT], muth[MT], muab[MT];
    T sigr[MT], sigt[MT];  // sqrt(2 Dr dt), sqrt(2 Dt dt) in T (noise amplitudes; set with dt)
    int parent_drag[MT];
    int kmax[MT];  // shape modes a type may carry (modes m >= kmax stay zero), <= K
    int bt_kind[MTERM];
    uint32_t bt_mask[MTERM];
    T bt_a[MTERM], bt_b[MTERM];  // Tension: a = eta; PerimeterElasticity: a = lambda, b = p0*sqrt(pi)
    T cA[2][MT][MT];             // summed Overlap couplings [related][ti][tj] (applied at d >= 0)
    T cB[MT];                    // summed LinearRepulsion k of terms applying to ti (k*d at d > 0)
    uint32_t bd_mask[MTERM];
    T bd_k[MTERM], bd_r0[MTERM];
    // compiled user terms (include/fcc_user_terms.h): table index, type mask, parameters a, b
    int nub, nuc, nubd;  // body, contact, bond terms
    int ub_id[MUT], uc_id[MUT], ubd_id[MUT];
    uint32_t ub_mask[MUT], uc_mask[MUT], ubd_mask[MUT];
    T ub_a[MUT], ub_b[MUT], uc_a[MUT], uc_b[MUT], ubd_a[MUT], ubd_b[MUT];
};

struct GridSync {
    unsigned count;   // arrivals at even-numbered barriers
    unsigned gen;
    int error;        // 1: a barrier wait ran out (the kernel returned early)
    int any_need;     // some simulation rebuilds its neighbour list this step
    unsigned count2;  // arrivals at odd-numbered barriers
    unsigned fexit;   // blocks done with a launch's flat step barriers
    // flat step barriers of a lone simulation, by parity: arrivals (low 32
    // bits) and skin votes (high 32 bits); zero between launches
    unsigned long long fcnt[2];
};

template <class T>
struct DevPtrs {
    const SimDesc<T>* sims;
    int nsims, Ntot, Ctot, nth, cap;
    const int* sim_of;
    T* rec0;
    T* rec1;
    T* coef;
    int* imgx;
    int* imgy;
    const T* R0;
    T* x0;
    T* y0;
    T* rmax0;
    int* nb_idx;
    int* nb_count;
    int* cellid;
    int* slot;
    int* perm;
    int* cstart;
    int* cstop;
    int* ccount;
    const int* cell_sim;
    int ccap;
    const int* ch_idx;
    const int* ch_count;
    int bcap;
    const int* bd_idx;
    const int* bd_count;
    int* flags;
    long long* clock;
    const long long* stop;  // per simulation: clock value at which it holds (null: no limit)
    long long* builds;
    int* maxcount;
    GridSync* sync;
    const T* cs;     // cos/sin of the node angles, 2*nth
    const T* basis;  // [nth][KM][4]: cos n phi_k, sin n phi_k, n cos n phi_k, n sin n phi_k (n = 2..10)
    const float* mtab;  // FP32: tensor-core fragment table of the contour contractions (null: none)
    // forces of the split (parent drag) step and of compute_gradients
    T* gx;
    T* gy;
    T* gth;
    T* glab;  // [g][19]
    T* E;
    // diagnostics of compute_gradients (ntheta per body) and the body-frame gradient
    T* P;
    T* GR;
    T* GD;
    T* GDD;
    T* gcoef;  // [g][19]
};

// ------------------------------------------------------------ arithmetic
// Exactly rounded single operations (no FMA contraction) for the integer
// decisions that must agree bit for bit with the oracle: cell index,
// neighbour test, skin test, wrap.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float t_rint(float a) { return rintf(a); }
__device__ __forceinline__ double t_rint(double a) { return rint(a); }
__device__ __forceinline__ float t_floor(float a) { return floorf(a); }
__device__ __forceinline__ double t_floor(double a) { return floor(a); }
__device__ __forceinline__ float t_sqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double t_sqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float t_log(float a) { return logf(a); }
__device__ __forceinline__ double t_log(double a) { return log(a); }
__device__ __forceinline__ void t_sincos(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ void t_sincos(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ float t_pi(float*) { return 3.14159265358979323846f; }
__device__ __forceinline__ double t_pi(double*) { return 3.14159265358979323846; }

// minimum_image, src/box.jl:14, exactly rounded as the reference evaluates it.
// For |d| < L/2 the rounded quotient is at most 1/2 and rint gives ±0, so the
// result is d - (±0) = d + 0: returned without the division (same bits).
template <class T>
__device__ __forceinline__ T minimum_image_exact(T d, T L) {
    if (fabs(d) < T(0.5) * L) return add_rn(d, T(0));
    return sub_rn(d, mul_rn(L, t_rint(div_rn(d, L))));
}
// minimum image with a precomputed 1/L (force evaluation; differs from the
// exact form only when d/L rounds across a half-integer, i.e. at distances
// ~L/2 that the contact pre-check rejects)
template <class T>
__device__ __forceinline__ T minimum_image_fast(T d, T L, T invL) {
    return d - L * t_rint(d * invL);
}

// wrap, src/box.jl:21-30.  For 0 <= x < L the rounded quotient x/L stays
// below 1 (the largest value below L is at least one ulp of 1 away), so the
// floor is 0 and the result is x - 0 = x + 0: returned without the division
// (same bits).
template <class T>
__device__ __forceinline__ T wrap_exact(T x, T L, int& shift) {
    if (x >= T(0) && x < L) {
        shift = 0;
        return add_rn(x, T(0));
    }
    T s = t_floor(div_rn(x, L));
    T xp = sub_rn(x, mul_rn(s, L));
    if (xp >= L) {
        xp = T(0);
        s = add_rn(s, T(1));
    }
    shift = (int)s;
    return xp;
}

// record field w <-> (parent, type)
__device__ __forceinline__ float pack_w(int v, float*) { return __int_as_float(v); }
__device__ __forceinline__ double pack_w(int v, double*) { return (double)v; }
__device__ __forceinline__ int unpack_w(float w) { return __float_as_int(w); }
__device__ __forceinline__ int unpack_w(double w) { return (int)w; }

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (src/random.jl:15-36).
__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// src/random.jl:42-44
__device__ __forceinline__ float uniform_open(float*, uint32_t a, uint32_t) {
    return ((float)(a >> 9) + 0.5f) * 0x1p-23f;
}
__device__ __forceinline__ double uniform_open(double*, uint32_t a, uint32_t b) {
    return ((double)(((((uint64_t)a) << 32) | b) >> 12) + 0.5) * 0x1p-52;
}

// Two standard normals of body i (1-based within its simulation) in draw n
// from Philox block `block` (src/random.jl:47-51, 75-78).
template <class T>
__device__ __forceinline__ void philox_pair(uint32_t k0, uint32_t k1, uint32_t i, uint64_t n, uint32_t block, T& z1,
                                            T& z2) {
    uint32_t c[4] = {i, (uint32_t)n, (uint32_t)(n >> 32), block};
    philox(c, k0, k1);
    T* tag = nullptr;
    T u1 = uniform_open(tag, c[0], c[1]);
    T u2 = uniform_open(tag, c[2], c[3]);
    T r = t_sqrt(mul_rn(T(-2), t_log(u1)));
    T s, co;
    t_sincos(mul_rn(mul_rn(T(2), t_pi(tag)), u2), &s, &co);
    z1 = mul_rn(r, co);
    z2 = mul_rn(r, s);
}

// ---------------------------------------------------------------- warps
template <int L, class V>
__device__ __forceinline__ V group_sum(V v) {
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off, L);
    return v;
}
template <int L>
__device__ __forceinline__ int group_max(int v) {
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off, L));
    return v;
}

// ------------------------------------------------- coherent global loads
// Data that other blocks write during the persistent kernel (records,
// neighbour lists, flags, clocks, forces of the split step) is read at L2
// (ld.global.cg), never through a possibly stale L1 line.
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ long long ldcg(const long long* p) { return __ldcg(p); }
__device__ __forceinline__ float4 ldcg(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldcg(const double2* p) { return __ldcg(p); }

// ------------------------------------------------------------ async copies
// 16-byte global -> shared copies that bypass L1 (cp.async.cg): the
// neighbour records a body needs are staged in shared memory while the warp
// synthesises its own contour.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// wait until at most N of this thread's committed copy groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ------------------------------------------------------------ grid barrier
// Barrier over all blocks of a cooperative launch (all co-resident).  Arrival
// is an acq_rel atomic, the release a release store, the wait an acquire
// load, so every write before the barrier is visible after it.  The last
// block to arrive runs `last()` with all its threads before it releases the
// others.  Waits are bounded: after SPIN_LIMIT polls a waiting block records
// sync->error and the kernel returns (the host reports FCC_ERR_DEVICE)
// instead of hanging.
// Barriers alternate between two arrival counters by the parity of their
// number; the last block clears the counter just used after its release
// store, off the critical path: that counter is used again two barriers
// later, and the clear precedes the block's own next arrival (an acq_rel
// atomic), which every later barrier's release follows.
constexpr long long SPIN_LIMIT = 1ll << 22;  // ~0.1-4 s with the back-off below

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_add_release(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

#ifndef FCC_BARRIER_FENCE
#define FCC_BARRIER_FENCE 0  // 1: full fence before the release store (measured: not needed, 1% slower)
#endif
#ifndef FCC_BARRIER_SLEEP
#define FCC_BARRIER_SLEEP 20  // ns between polls of the generation word
#endif
// What a block of a persistent launch knows of the barrier: the generation
// word it last saw (bit 0 carries the released any_need flag, the rest counts
// barriers), so neither the generation nor the rebuild flag costs a global
// read at the next barrier or step.
struct BarrierLocal {
    unsigned gen;
    int any;
    int flags;        // one simulation: its flags as of the last barrier
    long long clock;  // one simulation: its clock, ticked by every block
    int rebuild;      // a body of this block exceeded its skin in this step
    int released;     // this block arrived last and released the barrier itself
    int err;          // this block's wait gave up
    unsigned bits;    // arrival bits summed up to this block's arrival
    // flat step barriers (one simulation): arrivals and votes this block has
    // seen complete on each parity's counter, and the next barrier's parity
    unsigned ftgt[2], fvote[2];
    int fpar;
    int ovf;          // a neighbour list of this block overflowed in this rebuild
};

// Generation word: bit 0 the released any_need flag, bits 1-8 the flags of a
// lone simulation, bits 9-31 a barrier counter.
constexpr int GEN_FLAG_BITS = 9;

// Read once per launch (the host may have set flags or any_need between
// launches).  `one`: the launch advances a single simulation.
__device__ __forceinline__ void barrier_start(GridSync* gs, BarrierLocal& bl, bool one, const int* flags,
                                              const long long* clock) {
    if (threadIdx.x == 0) {
        bl.gen = ld_acquire(&gs->gen);
        bl.any = ld_acquire(&gs->any_need);
        bl.flags = one ? ld_acquire(flags) : 0;
        bl.clock = one ? *(volatile const long long*)clock : 0;
        bl.rebuild = 0;
        bl.released = 0;
        bl.err = 0;
        bl.ftgt[0] = bl.ftgt[1] = 0u;
        bl.fvote[0] = bl.fvote[1] = 0u;
        bl.fpar = 0;
    }
    __syncthreads();
}

// A grid barrier in two halves.  barrier_arrive: the block arrives; the
// last block to arrive runs `last(sum_bits)` with all its threads, which
// returns (in thread 0) the code to release — any_need | flags << 1 — or -1
// to keep the current one, releases the barrier and runs `after(code)` in
// thread 0 (writes that no block reads before the next barrier).  Arrival
// carries `bits` (summed over blocks into the upper half of the counter).
// `tick` is added to bl.clock (a lone simulation's noise counter) before the
// closing block barrier, so every warp of the block leaves with the new
// clock.  barrier_wait: the block waits for the release and takes the
// released rebuild flag and lone-simulation flags.  Between the halves a
// block may only do work that reads no other block's writes of the step.
struct NoAfter {
    __device__ void operator()(int) const {}
};
template <class F, class A = NoAfter>
__device__ __forceinline__ void barrier_arrive(GridSync* gs, BarrierLocal& bl, F&& last, unsigned bits = 0,
                                               A&& after = A{}, int tick = 0) {
    unsigned* cnt = ((bl.gen >> GEN_FLAG_BITS) & 1u) ? &gs->count2 : &gs->count;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned prev = atom_add_acq_rel(cnt, 1u + (bits << 16));
        bl.released = ((prev & 0xffffu) == gridDim.x - 1);
        bl.bits = (prev >> 16) + bits;
        bl.err = 0;
    }
    __syncthreads();
    if (bl.released) {
        int code = last(bl.bits);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (code < 0) code = bl.any | (bl.flags << 1);
#if FCC_BARRIER_FENCE
            __threadfence();
#endif
            const unsigned ng = (((bl.gen >> GEN_FLAG_BITS) + 1u) << GEN_FLAG_BITS) | ((unsigned)code & 0x1ffu);
            st_release(&gs->gen, ng);  // release: the block's writes before it
            *cnt = 0;
            gs->any_need = code & 1;   // for the host and the stand-alone kernels
            after(code);
            bl.gen = ng;
        }
    }
    if (threadIdx.x == 0) bl.clock += tick;
    __syncthreads();
}

// LIMIT: polls before a waiting block gives up (a self-test lowers it).
template <long long LIMIT = SPIN_LIMIT>
__device__ __forceinline__ bool barrier_wait(GridSync* gs, BarrierLocal& bl) {
    if (threadIdx.x == 0) {
        if (!bl.released) {
            long long it = 0;
            unsigned v;
            while ((v = ld_acquire(&gs->gen)) == bl.gen) {
                if (++it > LIMIT) {
                    atomicExch(&gs->error, 1);
                    bl.err = 1;
                    break;
                }
#if FCC_BARRIER_SLEEP > 0
                __nanosleep(FCC_BARRIER_SLEEP);
#endif
            }
            bl.gen = v;
        }
        bl.any = (int)(bl.gen & 1u);
        bl.flags = (int)((bl.gen >> 1) & 0xffu);
    }
    __syncthreads();
    return bl.err == 0;
}

// Both halves, nothing between them.
template <long long LIMIT = SPIN_LIMIT, class F, class A = NoAfter>
__device__ __forceinline__ bool grid_barrier(GridSync* gs, BarrierLocal& bl, F&& last, unsigned bits = 0,
                                             A&& after = A{}, int tick = 0) {
    barrier_arrive(gs, bl, static_cast<F&&>(last), bits, static_cast<A&&>(after), tick);
    return barrier_wait<LIMIT>(gs, bl);
}

// Step barrier of a lone simulation without a releasing block: each block
// adds its arrival and its skin vote (`vote`, into the high half) to the
// counter of the barrier's parity with a release reduction, then polls the
// counter until every block has arrived.  Every block thus reads the same
// final value and runs the same bookkeeping on it, and the release costs one
// trip to L2 instead of an atomic round trip, a store and a poll.  The value
// read on completion is exact: a counter is next added to two step barriers
// later, which no block reaches before every block has passed this one.  On
// return (thread 0) bl.bits holds the votes of this barrier.  Counters run
// from zero within a launch; flat_end clears them when the last block is
// done.  `done` runs in thread 0 once the wait is over, before the closing
// block barrier; `entry_sync` = false when the caller's own block barrier
// just preceded the call (thread 0 alone may have worked since).
template <long long LIMIT = SPIN_LIMIT, class F = NoAfter>
__device__ __forceinline__ bool flat_barrier(GridSync* gs, BarrierLocal& bl, unsigned vote, F&& done = F{},
                                             bool entry_sync = true) {
    if (entry_sync) __syncthreads();
    if (threadIdx.x == 0) {
        const int p = bl.fpar;
        unsigned long long* c = &gs->fcnt[p];
        red_add_release(c, 1ull | ((unsigned long long)vote << 32));
        const unsigned tgt = bl.ftgt[p] + gridDim.x;
        bl.err = 0;
        long long it = 0;
        unsigned long long v;
        while ((int)((unsigned)(v = ld_acquire(c)) - tgt) < 0) {
            if (++it > LIMIT) {
                atomicExch(&gs->error, 1);
                bl.err = 1;
                break;
            }
#if FCC_BARRIER_SLEEP > 0
            __nanosleep(FCC_BARRIER_SLEEP);
#endif
        }
        const unsigned hv = (unsigned)(v >> 32);
        bl.bits = hv - bl.fvote[p];
        bl.fvote[p] = hv;
        bl.ftgt[p] = tgt;
        bl.fpar = p ^ 1;
        if (!bl.err) done(0);
    }
    __syncthreads();
    return bl.err == 0;
}

// End of a launch that used flat barriers (thread 0 of each block, after its
// last wait): the last block to get here clears the counters for the next
// launch; every block has then read them for the last time.  A launch whose
// wait ran out returns early and leaves them set; its error status stays set
// too (every later step call fails) until fcc_set_state writes the whole
// GridSync anew.
__device__ __forceinline__ void flat_end(GridSync* gs) {
    if (atomicAdd(&gs->fexit, 1u) == gridDim.x - 1) {
        gs->fcnt[0] = 0ull;
        gs->fcnt[1] = 0ull;
        gs->fexit = 0u;
    }
}

// Fast reciprocal square root for the FP32 force path (rsqrt, ~2 ulp);
// FP64 keeps the correctly rounded 1/sqrt.
__device__ __forceinline__ float fast_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double fast_rsqrt(double x) { return 1.0 / sqrt(x); }

}  // namespace fcc
