// SESPH and IISPH timestep phases as gather kernels over the neighbor lists.
//
// Each kernel restates one parallel loop of the reference solver; the
// comments give the loop and the float expression order it follows.
// Neighbor sums are accumulated with Acc<R, KAHAN>: plain sums in the
// reference's operation order (FP32 / FP64 modes), or Kahan-compensated sums.
#pragma once

#include "fs_common.cuh"

namespace fsb {

template <typename R> struct SolverConsts {
    SplineKernel<R> kern;
    R rest_density;
    R rho0_sq;        // Math::pow2(rest_density)
    R inv_rho0_sq;    // 1 / rho0^2 (fast mode)
    R gravity;
    R visc_eps;       // (0.01f * particle_size) * particle_size
    R two_nu;         // 2.0f * viscosity
    R omega, gamma;
    R two_gamma;      // 2.0f * gamma
    R gamma1, gamma2;
    R stiffness;
    bool single_layer;
    int dim;
    R max_density_error;
    int min_iterations, max_iterations;
};

struct Lists {
    const uint32_t* FSB_R nbr;
    const uint32_t* FSB_R count;
    int64_t stride;
    int K;
    __device__ __forceinline__ uint32_t size(int64_t k) const { return min(count[k], (uint32_t)K); }
    __device__ __forceinline__ uint32_t at(int64_t k, uint32_t s) const { return nbr[(int64_t)s * stride + k]; }
};

// Visits particle k's list in order, handing f(entry, position of the
// neighbor). Entries and positions are loaded a batch at a time before any of
// them is used, so that a thread keeps several independent gathers in flight
// instead of one dependent load chain per neighbor. The summation order (list
// order) is unchanged.
constexpr int kBatch = 4;
template <typename R, typename F>
__device__ __forceinline__ void for_neighbors(const Lists& L, int64_t k, const V4<R>* FSB_R pos, F&& f) {
    const uint32_t n = L.size(k);
    uint32_t q = 0;
    for (; q + kBatch <= n; q += kBatch) {
        uint32_t e[kBatch];
        V4<R> p[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; b++) e[b] = FSB_LDG(&L.nbr[(int64_t)(q + b) * L.stride + k]);
#pragma unroll
        for (int b = 0; b < kBatch; b++) p[b] = pos[e[b] & kIndexMask];
#pragma unroll
        for (int b = 0; b < kBatch; b++) f(e[b], p[b]);
    }
    for (; q < n; q++) {
        const uint32_t e = FSB_LDG(&L.nbr[(int64_t)q * L.stride + k]);
        f(e, pos[e & kIndexMask]);
    }
}

// As for_neighbors, also handing d = x_k - x_j and gradW(d).
template <typename R, bool FAST, typename F>
__device__ __forceinline__ void for_neighbors_grad(const Lists& L, int64_t k, const V4<R>* FSB_R pos, V3<R> xk,
                                                   const SplineKernel<R>& kern, F&& f) {
    for_neighbors<R>(L, k, pos, [&](uint32_t e, const V4<R>& pj) {
        const V3<R> d = xk - xyz<R>(pj);
        f(e, pj, d, kern.template grad<FAST>(d));
    });
}

template <typename R> struct State {
    V4<R>* FSB_R pos;
    V4<R>* FSB_R vel;
    V4<R>* FSB_R acc;
    V4<R>* FSB_R ext;
    R* FSB_R rho;       // density of this step (written by the density phase)
    R* FSB_R rho_prev;  // density read by the viscosity term
    R* FSB_R p;
    V4<R>* FSB_R vstar; // w: source term
    V4<R>* FSB_R anp;   // w: diagonal element
    R* FSB_R err;
    V4<R>* FSB_R gbnd;  // xyz: sum over boundary neighbors of m_j gradW, w: diagonal a_ii (second loop, tile passes)
    const uint8_t* FSB_R type;
    const uint32_t* FSB_R hidx;
    const uint16_t* FSB_R scene;  // per-particle scene (batched contexts), else null
    __device__ __forceinline__ int scene_of(int64_t k) const { return scene ? scene[k] : 0; }
};

__device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmax_(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double fmin_(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float abs_(float a) { return fabsf(a); }
__device__ __forceinline__ double abs_(double a) { return fabs(a); }

// float maxima of non-negative values, kept as ordered bit patterns; NaN is
// ignored like std::fmax ignores it
__device__ __forceinline__ void atomic_max_nonneg(unsigned int* a, float v) {
    if (v >= 0.0f) atomicMax(a, __float_as_uint(v));
}

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ===========================================================================
// viscosity term (IISPHFluidSolver3D.hpp:43-76, SESPHFluidSolver3D.hpp:293-324,
// IISPHFluidSolver.hpp:240-277, SESPHFluidSolver.hpp:254-285):
//   tmp += (m_j / rho_j) * (dot(v_ij, x_ij) / (dot(x_ij, x_ij) + eps)) * gradW
//   return (2 nu) * tmp
// rho_of(j, entry) supplies the neighbor density the reference reads.
// ===========================================================================
template <typename R, bool KAHAN, typename RhoOf>
__device__ __forceinline__ V3<R> viscosity(int64_t k, const State<R>& s, const Lists& L, const SolverConsts<R>& c,
                                           V3<R> xi, V3<R> vi, RhoOf&& rho_of) {
    Acc3<R, KAHAN> tmp;
    for_neighbors_grad<R, KAHAN>(L, k, s.pos, xi, c.kern, [&](uint32_t e, const V4<R>& pj, V3<R> xij, V3<R> g) {
        const uint32_t j = e & kIndexMask;
        const R rj = rho_of(j, e);
        if (rj == R(0)) return;
        const V4<R> vj = s.vel[j];
        const V3<R> vij = vi - xyz<R>(vj);
        const R f = KAHAN ? fdiv<true>(pj.w * dotf<true>(vij, xij), rj * (dotf<true>(xij, xij) + c.visc_eps))
                          : (pj.w / rj) * (dot(vij, xij) / (dot(xij, xij) + c.visc_eps));
        tmp.add(f * g);
    });
    return c.two_nu * tmp.get();
}

// ===========================================================================
// IISPH 3D, first loop (IISPHFluidSolver3D.hpp:141-212): p = 0; non-pressure
// acceleration (gravity + viscosity) for non-boundary particles; v*; store
// a_np; reset ExternalForces; density for fluid particles.
// SPLIT = false: one pass, viscosity reads the previous density for every j.
// SPLIT = true : density in k_iisph3d_density first, then this kernel reads the
//                new density of fluid neighbors with a smaller host index and
//                the previous one otherwise -- the order the reference's serial
//                loop produces (it overwrites densities while reading them).
// ===========================================================================
template <typename R, bool KAHAN, bool SPLIT>
__device__ __forceinline__ void iisph3d_l1_one(int64_t k, const State<R>& s, const Lists& L, const SolverConsts<R>& c,
                                               R dt) {
    const uint8_t t = s.type[k];
    if (t == FS_TYPE_INACTIVE) {
        if (!SPLIT) s.rho[k] = s.rho_prev[k];  // carry the density through the double buffer
        return;
    }
    const V4<R> pk = s.pos[k];
    const V4<R> vk = s.vel[k];
    s.p[k] = R(0);
    V3<R> npa = xyz<R>(s.ext[k]);
    if (t != FS_TYPE_BOUNDARY) {
        npa = npa + v3<R>(R(0), -c.gravity, R(0));
        V3<R> visc;
        if (SPLIT) {
            const uint32_t hk = s.hidx[k];
            visc = viscosity<R, KAHAN>(k, s, L, c, xyz<R>(pk), xyz<R>(vk), [&](uint32_t j, uint32_t e) -> R {
                if (!(e & kBoundaryBit) && s.hidx[j] < hk) return s.rho[j];
                return s.rho_prev[j];
            });
        } else {
            visc = viscosity<R, KAHAN>(k, s, L, c, xyz<R>(pk), xyz<R>(vk),
                                       [&](uint32_t j, uint32_t) -> R { return s.rho_prev[j]; });
        }
        npa = npa + visc;
    }
    const V3<R> vstar = xyz<R>(vk) + dt * npa;
    s.vstar[k] = v4<R>(vstar, R(0));
    s.anp[k] = v4<R>(npa, R(0));
    s.ext[k] = v4<R>(v3<R>(R(0), R(0), R(0)), R(0));
    if (t == FS_TYPE_BOUNDARY) {
        if (!SPLIT) s.rho[k] = s.rho_prev[k];
        return;
    }
    if (!SPLIT) {
        Acc<R, KAHAN> rho;
        for_neighbors<R>(L, k, s.pos, [&](uint32_t e, const V4<R>& pj) {
            R m = pj.w;
            if (c.single_layer && (e & kBoundaryBit)) m = m * c.gamma1;
            rho.add(m * c.kern.template w<KAHAN>(xyz<R>(pk) - xyz<R>(pj)));
        });
        s.rho[k] = rho.get();
    }
}

template <typename R, bool KAHAN, bool SPLIT>
__global__ void k_iisph3d_l1(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const StepScalars* FSB_R sc,
                             const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph3d_l1_one<R, KAHAN, SPLIT>(k, s, L, c, (R)sc->dt);
}

// density only (IISPHFluidSolver3D.hpp:184-210), for the split first loop
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph3d_density_at(int64_t k, const State<R>& s, const Lists& L,
                                                   const SolverConsts<R>& c) {
    const uint8_t t = s.type[k];
    if (t != FS_TYPE_NORMAL) {
        s.rho[k] = s.rho_prev[k];
        return;
    }
    const V3<R> xk = xyz<R>(s.pos[k]);
    Acc<R, KAHAN> rho;
    const uint32_t nn = L.size(k);
    for (uint32_t q = 0; q < nn; q++) {
        const uint32_t e = L.at(k, q);
        const V4<R> pj = s.pos[e & kIndexMask];
        R m = pj.w;
        if (c.single_layer && (e & kBoundaryBit)) m = m * c.gamma1;
        rho.add(m * c.kern.template w<KAHAN>(xk - xyz<R>(pj)));
    }
    s.rho[k] = rho.get();
}
template <typename R, bool KAHAN>
__global__ void k_iisph3d_density(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph3d_density_at<R, KAHAN>(k, s, L, c);
}

// ===========================================================================
// IISPH 3D, second loop (IISPHFluidSolver3D.hpp:216-339): source term and
// diagonal element for fluid particles.
//   s_i   = (rho0 - rho_i) - dt * sum_j m_j dot(v*_i - v*_j, gradW)   (boundary: v*_j dropped)
//   d_i   = - sum_j w_j m_j / rho0^2 gradW          (w_j = 2 gamma / 2 for boundary)
//   a_ii  = dt^2 [ sum_j m_j dot(d_i, gradW) + sum_fluid m_j dot(-(m_i/rho0^2) gradW, gradW) ]
// TWO_PASS = true walks the list a second time for a_ii exactly as the
// reference does; otherwise a_ii is assembled from the same single pass as
// dot(d_i, sum_j m_j gradW) - (m_i/rho0^2) sum_fluid m_j |gradW|^2 (the same sum
// regrouped, used with the compensated sums).
// ===========================================================================
template <typename R, bool KAHAN, bool TWO_PASS>
__device__ __forceinline__ void iisph3d_l2_one(int64_t k, const State<R>& s, const Lists& L, const SolverConsts<R>& c,
                                               R dt) {
    const V4<R> pk = s.pos[k];
    const V3<R> xk = xyz<R>(pk);
    const V4<R> vsk4 = s.vstar[k];
    const V3<R> vsk = xyz<R>(vsk4);
    Acc<R, KAHAN> contrib;
    Acc3<R, KAHAN> inner;
    Acc3<R, KAHAN> mg;    // sum_j m_j gradW      (single-pass a_ii)
    Acc<R, KAHAN> mg2;    // sum_fluid m_j |gradW|^2
    for_neighbors_grad<R, KAHAN>(L, k, s.pos, xk, c.kern, [&](uint32_t e, const V4<R>& pj, V3<R>, V3<R> g) {
        const uint32_t j = e & kIndexMask;
        if (!(e & kBoundaryBit)) {
            const V3<R> vsj = xyz<R>(s.vstar[j]);
            contrib.add(pj.w * dotf<KAHAN>(vsk - vsj, g));
            inner.sub((KAHAN ? pj.w * c.inv_rho0_sq : pj.w / c.rho0_sq) * g);
            if (!TWO_PASS) mg2.add(pj.w * dotf<KAHAN>(g, g));
        } else {
            contrib.add(pj.w * dotf<KAHAN>(vsk, g));
            const R w = c.single_layer ? c.two_gamma * pj.w : R(2) * pj.w;
            inner.sub((KAHAN ? w * c.inv_rho0_sq : w / c.rho0_sq) * g);
        }
        if (!TWO_PASS) mg.add(pj.w * g);
    });
    const R source = (c.rest_density - s.rho[k]) - dt * contrib.get();
    const V3<R> in = inner.get();
    R diag;
    if (TWO_PASS) {
        Acc<R, KAHAN> d;
        const R mi = pk.w / c.rho0_sq;
        for_neighbors<R>(L, k, s.pos, [&](uint32_t e, const V4<R>& pj) {
            const V3<R> g = c.kern.template grad<KAHAN>(xk - xyz<R>(pj));
            d.add(pj.w * dot(in, g));
            // gradW(x_j - x_i) == -gradW(x_i - x_j) bit for bit
            if (!(e & kBoundaryBit)) d.add(pj.w * dot(mi * (-g), g));
        });
        diag = d.get() * (dt * dt);
    } else {
        diag = (dot(in, mg.get()) - (pk.w / c.rho0_sq) * mg2.get()) * (dt * dt);
    }
    s.vstar[k] = v4<R>(vsk, source);
    s.anp[k].w = diag;
}

template <typename R, bool KAHAN, bool TWO_PASS>
__global__ void k_iisph3d_l2(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const StepScalars* FSB_R sc,
                             const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    if (s.type[k] != FS_TYPE_NORMAL) return;
    iisph3d_l2_one<R, KAHAN, TWO_PASS>(k, s, L, c, (R)sc->dt);
}

// ===========================================================================
// IISPH 3D iteration (a): pressure acceleration (IISPHFluidSolver3D.hpp:348-397)
//   a_i = - sum_fluid m_j (p_i/rho0^2 + p_j/rho0^2) gradW
//         - sum_bdy (gamma m_j 2 p_i / rho0^2) gradW       (single layer; no gamma otherwise)
// ===========================================================================
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph3d_pressure_acc_one(int64_t k, const State<R>& s, const Lists& L,
                                                         const SolverConsts<R>& c) {
    const V3<R> xk = xyz<R>(s.pos[k]);
    const R pk = s.p[k];
    Acc3<R, KAHAN> pa;
    for_neighbors_grad<R, KAHAN>(L, k, s.pos, xk, c.kern, [&](uint32_t e, const V4<R>& pj, V3<R>, V3<R> g) {
        const uint32_t j = e & kIndexMask;
        if (KAHAN) {
            const R f = !(e & kBoundaryBit) ? pj.w * (pk + s.p[j])
                                            : (c.single_layer ? c.two_gamma : R(2)) * pj.w * pk;
            pa.sub((f * c.inv_rho0_sq) * g);
        } else if (!(e & kBoundaryBit)) {
            pa.sub((pj.w * (pk / c.rho0_sq + s.p[j] / c.rho0_sq)) * g);
        } else if (c.single_layer) {
            pa.sub(((((c.gamma * pj.w) * R(2)) * pk) / c.rho0_sq) * g);
        } else {
            pa.sub((((pj.w * R(2)) * pk) / c.rho0_sq) * g);
        }
    });
    s.acc[k] = v4<R>(pa.get(), R(0));
}

template <typename R, bool KAHAN>
__global__ void k_iisph3d_pressure_acc(int64_t n, State<R> s, Lists L, SolverConsts<R> c,
                                       const StepScalars* FSB_R sc, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status || sc->done) return;
    if (s.type[k] != FS_TYPE_NORMAL) return;
    iisph3d_pressure_acc_one<R, KAHAN>(k, s, L, c);
}

// ===========================================================================
// IISPH 3D iteration (b): A p, relaxed Jacobi update and the per-particle
// density error (IISPHFluidSolver3D.hpp:402-461), fused with the convergence
// scan of :467-512 (block partial sums into StepScalars, FP64 residual).
// ===========================================================================
// per-particle contribution to the convergence scan and the CFL maxima
struct ErrPart {
    double e_sum = 0.0;
    unsigned int e_cnt = 0;
    float e_max = 0.f, a2 = 0.f, v2 = 0.f;
};

// the update of particle k given its pressure acceleration ak and the
// neighbor sum sum_j m_j dot(a_k - a_j, gradW)
// vs: v* with the source term in w; aii: diagonal element; p: current pressure
template <typename R>
__device__ __forceinline__ ErrPart iisph3d_pressure_update_tail(int64_t k, const State<R>& s, const SolverConsts<R>& c,
                                                                R dt, V3<R> ak, R ap_sum, V4<R> vs, R aii, R p) {
    ErrPart o;
    const R Ap = ap_sum * (dt * dt);
    const bool has_diag = abs_(aii) > R(kFltEps);
    if (has_diag) p = fmax_(R(0), p + c.omega * ((vs.w - Ap) / aii));
    else p = R(0);
    s.p[k] = p;
    R perr = abs_(vs.w - Ap);
    if (has_diag) {
        if (abs_(p) <= R(kFltEps)) perr = R(0);
        s.err[k] = perr;
        o.e_sum = (double)perr;
        o.e_cnt = 1;
        o.e_max = (float)perr;
    }
    // max |a|^2 and |v* + dt a|^2 of the fluid particles (CFL input)
    o.a2 = (float)dot(ak, ak);
    const V3<R> vf = xyz<R>(vs) + dt * ak;
    o.v2 = (float)dot(vf, vf);
    if (!(o.a2 >= 0.f)) o.a2 = 0.f;
    if (!(o.v2 >= 0.f)) o.v2 = 0.f;
    if (!(o.e_max >= 0.f)) o.e_max = 0.f;
    return o;
}

template <typename R, bool KAHAN>
__device__ __forceinline__ ErrPart iisph3d_pressure_update_one(int64_t k, const State<R>& s, const Lists& L,
                                                               const SolverConsts<R>& c, R dt) {
    const V3<R> xk = xyz<R>(s.pos[k]);
    const V3<R> ak = xyz<R>(s.acc[k]);
    Acc<R, KAHAN> ap;
    for_neighbors_grad<R, KAHAN>(L, k, s.pos, xk, c.kern, [&](uint32_t e, const V4<R>& pj, V3<R>, V3<R> g) {
        const uint32_t j = e & kIndexMask;
        if (!(e & kBoundaryBit)) ap.add(pj.w * dotf<KAHAN>(ak - xyz<R>(s.acc[j]), g));
        else ap.add(pj.w * dotf<KAHAN>(ak, g));
    });
    return iisph3d_pressure_update_tail<R>(k, s, c, dt, ak, ap.get(), s.vstar[k], s.anp[k].w, s.p[k]);
}

// adds one thread's ErrPart to its scene's scalars
__device__ __forceinline__ void add_err_part(const ErrPart& o, StepScalars* FSB_R q) {
    if (o.e_cnt) {
        atomicAdd(&q->err_sum, o.e_sum);
        atomicAdd(&q->err_count, (unsigned long long)o.e_cnt);
    }
    atomic_max_nonneg(&q->max_err_bits, o.e_max);
    atomic_max_nonneg(&q->max_a2_bits, o.a2);
    atomic_max_nonneg(&q->max_v2_bits, o.v2);
}

// The first pressure iteration without neighbor sums (fast mode). The first
// loop sets every pressure to 0 (IISPHFluidSolver3D.hpp:141-212), so the
// iteration's pressure accelerations are 0 (the sums of :348-397 over p = 0)
// and so is A p (:402-461): the update is p = max(0, omega s / a_ii), the
// error |s|, the acceleration 0. vs: v* with the source term in w; aii: the
// diagonal element, as the second loop just computed them.
template <typename R>
__device__ __forceinline__ ErrPart iisph3d_first_iteration(int64_t k, const State<R>& s, const SolverConsts<R>& c,
                                                           R dt, V4<R> vs, R aii) {
    s.acc[k] = v4<R>(v3<R>(R(0), R(0), R(0)), R(0));
    return iisph3d_pressure_update_tail<R>(k, s, c, dt, v3<R>(R(0), R(0), R(0)), R(0), vs, aii, R(0));
}

// block reduction of the ErrParts into StepScalars (FP64 residual sum); every
// thread of the block calls it. scene: the scene of the thread's particle.
// A block whose threads all belong to one scene reduces first; a block that
// spans scenes adds thread by thread.
__device__ __forceinline__ void reduce_err_parts(ErrPart o, StepScalars* FSB_R sc, int scene = 0) {
    __shared__ int s_scene;
    if (threadIdx.x == 0) s_scene = scene;
    __syncthreads();
    const int s0 = s_scene;
    if (!__syncthreads_and(scene == s0)) {
        add_err_part(o, sc + scene);
        return;
    }
    sc += s0;
    double e_sum = warp_sum(o.e_sum);
    unsigned int e_cnt = warp_sum(o.e_cnt);
    float e_max = warp_max(o.e_max), a2 = warp_max(o.a2), v2 = warp_max(o.v2);
    __shared__ double s_sum[32];
    __shared__ unsigned int s_cnt[32];
    __shared__ float s_max[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_sum[wid] = e_sum; s_cnt[wid] = e_cnt;
        s_max[0][wid] = e_max; s_max[1][wid] = a2; s_max[2][wid] = v2;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        e_sum = lane < nw ? s_sum[lane] : 0.0;
        e_cnt = lane < nw ? s_cnt[lane] : 0u;
        e_max = lane < nw ? s_max[0][lane] : 0.f;
        a2 = lane < nw ? s_max[1][lane] : 0.f;
        v2 = lane < nw ? s_max[2][lane] : 0.f;
        e_sum = warp_sum(e_sum);
        e_cnt = warp_sum(e_cnt);
        e_max = warp_max(e_max);
        a2 = warp_max(a2);
        v2 = warp_max(v2);
        if (lane == 0) {
            if (e_cnt) {
                atomicAdd(&sc->err_sum, e_sum);
                atomicAdd(&sc->err_count, (unsigned long long)e_cnt);
            }
            atomic_max_nonneg(&sc->max_err_bits, e_max);
            atomic_max_nonneg(&sc->max_a2_bits, a2);
            atomic_max_nonneg(&sc->max_v2_bits, v2);
        }
    }
}

template <typename R, bool KAHAN>
__global__ void k_iisph3d_pressure_update(int64_t n, State<R> s, Lists L, SolverConsts<R> c,
                                          StepScalars* FSB_R sc, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (*status || sc->done) return;
    ErrPart o;
    if (k < n && s.type[k] == FS_TYPE_NORMAL) o = iisph3d_pressure_update_one<R, KAHAN>(k, s, L, c, (R)sc->dt);
    reduce_err_parts(o, sc);
}

// Convergence test after each iteration (IISPHFluidSolver3D.hpp:463-522) and
// the 2D variant (IISPHFluidSolver.hpp:400-402, 513-523). One thread.
//   FP32 mode : avg = (float)sum / (float)count, compared in float
//   otherwise : avg compared in FP64
//
// Inside a CUDA graph the kernel ends the conditional WHILE loop through
// `handle`. The loop is bounded independently of the state: loop_guard counts
// executions of the body and stops it after max_it, whatever the status word
// or the residual say.
// One scene's test after an iteration; returns whether its loop is done and
// resets the iteration's accumulators.
// The accumulators are read through volatile loads: the small-scene kernel
// runs the test in the kernel whose atomics produced them, where this SM may
// hold an older copy of the line.
__device__ __forceinline__ bool check_scene(StepScalars* FSB_R sc, int min_it, int max_it, float max_err,
                                            bool fp64_test, bool two_d) {
    const volatile StepScalars* v = sc;
    const int it = v->iteration;  // iterations completed before this one
    const unsigned long long cnt = v->err_count;
    const double sum = v->err_sum;
    float avg = 0.f;
    double avg64 = 0.0;
    if (cnt > 0) {
        avg64 = sum / (double)cnt;
        avg = fp64_test ? (float)avg64 : (float)sum / (float)cnt;
    }
    sc->avg_err = avg;
    sc->avg_err64 = avg64;
    sc->max_err = __uint_as_float(v->max_err_bits);
    sc->final_max_a2 = __uint_as_float(v->max_a2_bits);
    sc->final_max_v2 = __uint_as_float(v->max_v2_bits);
    const int done_it = it + 1;
    sc->iteration = done_it;
    bool done = false;
    const bool below = fp64_test ? (avg64 <= (double)max_err) : (avg <= max_err);
    if (two_d) {
        // while ((it < min || abs(err) > max) && it < max). The reference's
        // unqualified abs there is the C int abs: the float error is
        // truncated to an integer before the comparison.
        const float e = fp64_test ? (float)avg64 : avg;
        const float trunc_abs = (e >= 2147483647.0f || e <= -2147483647.0f) ? fabsf(e) : (float)abs((int)e);
        done = (done_it >= min_it && trunc_abs <= max_err) || done_it >= max_it;
    } else {
        // if (iteration >= min - 1 && avg <= max) break;  (size_t: min == 0 never breaks early)
        done = (min_it >= 1 && it >= min_it - 1 && below) || done_it >= max_it;
    }
    sc->done = done ? 1 : 0;
    sc->err_sum = 0.0;
    sc->err_count = 0ull;
    sc->max_err_bits = 0u;
    sc->max_a2_bits = 0u;
    sc->max_v2_bits = 0u;
    return done;
}

// The test of a single-scene context (one thread).
__device__ __forceinline__ void iisph_check_one(StepScalars* FSB_R sc, int min_it, int max_it, float max_err,
                                                bool fp64_test, bool two_d, const int* FSB_R status,
                                                cudaGraphConditionalHandle handle, bool set_condition) {
    const int guard = ++sc->loop_guard;
    bool stop = guard >= max_it;
    if (*(const volatile int*)status || sc->done) {
        if (set_condition) cudaGraphSetConditional(handle, 0u);
        return;
    }
    stop = check_scene(sc, min_it, max_it, max_err, fp64_test, two_d) || stop;
    if (set_condition) cudaGraphSetConditional(handle, stop ? 0u : 1u);
}

// Batched contexts: every scene still iterating is tested on its own (the
// 3D test, FP64 average); the loop goes on while any scene iterates. Every
// thread of one block calls it; the guard in scene 0 counts executions of
// the loop body.
__device__ __forceinline__ void iisph_check_scenes_block(StepScalars* FSB_R sc, int scenes, int min_it,
                                                         int max_it, float max_err, const int* FSB_R status,
                                                         cudaGraphConditionalHandle handle, bool set_condition) {
    __shared__ int s_guard;
    if (threadIdx.x == 0) s_guard = ++sc[0].loop_guard;
    __syncthreads();
    const bool stop_all = s_guard >= max_it || *(const volatile int*)status != 0;
    int active = 0;
    for (int i = threadIdx.x; i < scenes; i += blockDim.x) {
        StepScalars* q = sc + i;
        if (q->done) continue;
        const bool done = check_scene(q, min_it, max_it, max_err, true, false) || stop_all;
        q->done = done ? 1 : 0;
        if (!done) active = 1;
    }
    const int any = __syncthreads_or(active);
    if (threadIdx.x == 0 && set_condition) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

static __global__ void k_iisph_check(StepScalars* FSB_R sc, int min_it, int max_it, float max_err, bool fp64_test,
                              bool two_d, const int* FSB_R status, cudaGraphConditionalHandle handle,
                              bool set_condition) {
    grid_dependency_wait();
    iisph_check_one(sc, min_it, max_it, max_err, fp64_test, two_d, status, handle, set_condition);
}

static __global__ void k_iisph_check_scenes(StepScalars* FSB_R sc, int scenes, int min_it, int max_it, float max_err,
                                     const int* FSB_R status, cudaGraphConditionalHandle handle,
                                     bool set_condition) {
    grid_dependency_wait();
    iisph_check_scenes_block(sc, scenes, min_it, max_it, max_err, status, handle, set_condition);
}

// CFL clamp (IISPHFluidSolver3D.hpp:525-535, SESPHFluidSolver3D.hpp:109-116) with
// ConstantTimestepGenerator::get_non_cfl_validating_timestep
// (ConstantTimestepGenerator.cpp:17-41). The reference evaluates
// sqrt(size / a) * lambda_a in double (its unqualified sqrt is the C double
// function) and rounds the product to float; the rest is float.
__device__ __forceinline__ void cfl_one(StepScalars* FSB_R sc, float particle_size, float timestep,
                                        float lambda_v, float lambda_a) {
    const float max_v = sqrtf(sc->final_max_v2);
    const float max_a = sqrtf(sc->final_max_a2);
    float dta = timestep, dtv = timestep;
    if (max_a > 0.0f) dta = (float)(sqrt((double)(particle_size / max_a)) * (double)lambda_a);
    if (max_v > 0.0f) dtv = particle_size / max_v * lambda_v;
    float nt = fmaxf(fminf(dta, dtv), 0.000001f);
    nt = fminf(nt, sc->desired_dt);
    sc->dt = nt;
}

// ---------------------------------------------------------------------------
// DynamicCflTimestepGenerator (DynamicCflTimestepGenerator.cpp:6-61) on the
// device, so that the time step is chosen inside the step's CUDA graph.
// k_generator_max: the largest |v|^2 and |a|^2 (float, ((x x + y y) + z z),
// glm::length's dot) over the particles that are not inactive -- boundary
// included, as the reference's loop over the whole collection -- per scene,
// as ordered bits. max |v| = sqrt(max |v|^2) since sqrt is monotonic and
// correctly rounded. k_generator_finish: the generator's clamp, per scene.
// ---------------------------------------------------------------------------
// |v|^2 and |a|^2 of particle k as the generator computes them (0 when inactive)
template <typename R>
__device__ __forceinline__ bool generator_at(int64_t k, const State<R>& s, float& v2, float& a2) {
    if (s.type[k] == FS_TYPE_INACTIVE) return false;
    const V4<R> v = s.vel[k], a = s.acc[k];
    const float vx = (float)v.x, vy = (float)v.y, vz = (float)v.z;
    const float ax = (float)a.x, ay = (float)a.y, az = (float)a.z;
    v2 = (vx * vx + vy * vy) + vz * vz;
    a2 = (ax * ax + ay * ay) + az * az;
    return true;
}
template <typename R>
__global__ void k_generator_max(int64_t n, State<R> s, StepScalars* FSB_R sc,
                                const int* FSB_R status) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    float v2 = 0.f, a2 = 0.f;
    int scene = 0;
    const bool active = k < n && generator_at<R>(k, s, v2, a2);
    if (active) scene = s.scene_of(k);
    // one atomic per warp and quantity where the warp's particles share a scene
    const int s0 = __shfl_sync(0xffffffffu, scene, 0);
    if (__all_sync(0xffffffffu, scene == s0)) {
        v2 = warp_max(v2);
        a2 = warp_max(a2);
        if ((threadIdx.x & 31) == 0 && !*status) {
            atomic_max_nonneg(&sc[s0].gen_v2_bits, v2);
            atomic_max_nonneg(&sc[s0].gen_a2_bits, a2);
        }
    } else if (active) {
        atomic_max_nonneg(&sc[scene].gen_v2_bits, v2);
        atomic_max_nonneg(&sc[scene].gen_a2_bits, a2);
    }
}

// DynamicCflTimestepGenerator::generate_next_timestep (:45-59) and its
// get_non_cfl_validating_timestep (:82-107), whose default is max_timestep
__device__ __forceinline__ float dynamic_cfl_timestep(float max_v, float max_a, float particle_size, float min_ts,
                                                      float max_ts, float lambda_v, float lambda_a) {
    float ts = min_ts;
    if (max_v > kFltEps && max_a > kFltEps) {
        float dta = max_ts, dtv = max_ts;
        if (max_a > 0.0f) dta = (float)(sqrt((double)(particle_size / max_a)) * (double)lambda_a);
        if (max_v > 0.0f) dtv = particle_size / max_v * lambda_v;
        const float allowed = fmaxf(fminf(dta, dtv), 0.000001f);
        ts = fmaxf(ts, fminf(max_ts, allowed));
    }
    return ts;
}

// (the maxima come from atomics: read through volatile loads, as the small-scene
// step kernel runs this in the kernel that issued them)
__device__ __forceinline__ void generator_finish_one(StepScalars* FSB_R q, float particle_size, float min_ts,
                                                     float max_ts, float lambda_v, float lambda_a) {
    const volatile StepScalars* v = q;
    const float max_v = sqrtf(__uint_as_float(v->gen_v2_bits));
    const float max_a = sqrtf(__uint_as_float(v->gen_a2_bits));
    const float ts = dynamic_cfl_timestep(max_v, max_a, particle_size, min_ts, max_ts, lambda_v, lambda_a);
    q->desired_dt = ts;
    q->dt = ts;
}
static __global__ void k_generator_finish(StepScalars* FSB_R sc, int scenes, float particle_size, float min_ts,
                                   float max_ts, float lambda_v, float lambda_a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < scenes; i += gridDim.x * blockDim.x)
        generator_finish_one(sc + i, particle_size, min_ts, max_ts, lambda_v, lambda_a);
}

// the clamp for scenes [0, scenes) (one in a single-scene context)
static __global__ void k_cfl(StepScalars* FSB_R sc, int scenes, float particle_size, float timestep, float lambda_v,
                      float lambda_a, const int* FSB_R status) {
    if (*status) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < scenes; i += gridDim.x * blockDim.x)
        cfl_one(sc + i, particle_size, timestep, lambda_v, lambda_a);
}

// ===========================================================================
// IISPH 3D integration (IISPHFluidSolver3D.hpp:539-561), all active particles:
//   if dt changed: v* = (v* - old_dt a_np) + dt a_np
//   v = v* + dt a ;  x = x + dt v
// ===========================================================================
template <typename R>
__device__ __forceinline__ void iisph3d_integrate_at(int64_t k, const State<R>& s, const StepScalars* FSB_R sc) {
    if (s.type[k] == FS_TYPE_INACTIVE) return;
    const StepScalars* q = sc + s.scene_of(k);
    const R dt = (R)q->dt, old = (R)q->desired_dt;
    V3<R> vs = xyz<R>(s.vstar[k]);
    if (q->dt != q->desired_dt) {
        const V3<R> a = xyz<R>(s.anp[k]);
        vs = (vs - old * a) + dt * a;
    }
    const V3<R> v = vs + dt * xyz<R>(s.acc[k]);
    const V4<R> p = s.pos[k];
    const V3<R> x = xyz<R>(p) + dt * v;
    s.vel[k] = v4<R>(v, s.vel[k].w);
    s.pos[k] = v4<R>(x, p.w);
}
template <typename R>
__global__ void k_iisph3d_integrate(int64_t n, State<R> s, const StepScalars* FSB_R sc,
                                    const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph3d_integrate_at<R>(k, s, sc);
}

// ===========================================================================
// SESPH (SESPHFluidSolver3D.hpp:49-130, SESPHFluidSolver.hpp:49-111)
// ===========================================================================
// density and pressure of fluid particles
//   3D: boundary j contributes (gamma_1 m_j) W if single layer (:216-225)
//   p = max(k (rho / rho0 - 1), 0)  (std::max: NaN propagates)
template <typename R, bool KAHAN>
__device__ __forceinline__ void sesph_density_one(int64_t k, const State<R>& s, const Lists& L,
                                                  const SolverConsts<R>& c) {
    const V3<R> xk = xyz<R>(s.pos[k]);
    Acc<R, KAHAN> rho;
    const uint32_t nn = L.size(k);
    for (uint32_t q = 0; q < nn; q++) {
        const uint32_t e = L.at(k, q);
        const V4<R> pj = s.pos[e & kIndexMask];
        const R w = c.kern.template w<KAHAN>(xk - xyz<R>(pj));
        if ((e & kBoundaryBit) && c.single_layer) rho.add((c.gamma1 * pj.w) * w);
        else rho.add(pj.w * w);
    }
    const R r = rho.get();
    s.rho[k] = r;
    const R pr = c.stiffness * (r / c.rest_density - R(1));
    s.p[k] = (pr < R(0)) ? R(0) : pr;
}

template <typename R, bool KAHAN>
__global__ void k_sesph_density(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    if (s.type[k] != FS_TYPE_NORMAL) return;
    sesph_density_one<R, KAHAN>(k, s, L, c);
}

// accelerations of fluid particles: a = pressure acc + (gravity + viscosity)
//   pressure acc (:245-290): pdd = (rho == 0) ? 0 : p / rho^2
//     fluid j   : += (-m_j (pdd_i + pdd_j)) gradW
//     boundary j: += (-m_i (pdd_i + pdd_i)) gradW [* gamma_2 if single layer, 3D]
template <typename R, bool KAHAN>
__device__ __forceinline__ void sesph_accel_one(int64_t k, const State<R>& s, const Lists& L,
                                                const SolverConsts<R>& c) {
    const V4<R> pk = s.pos[k];
    const V3<R> xk = xyz<R>(pk);
    const R rk = s.rho[k];
    const R pdd = rk == R(0) ? R(0) : s.p[k] / (rk * rk);
    V3<R> npa = v3<R>(R(0), R(0), R(0)) + v3<R>(R(0), -c.gravity, R(0));
    npa = npa + viscosity<R, KAHAN>(k, s, L, c, xk, xyz<R>(s.vel[k]),
                                    [&](uint32_t j, uint32_t) -> R { return s.rho[j]; });
    Acc3<R, KAHAN> pa;
    for_neighbors_grad<R, KAHAN>(L, k, s.pos, xk, c.kern, [&](uint32_t e, const V4<R>& pj, V3<R>, V3<R> g) {
        const uint32_t j = e & kIndexMask;
        if (e & kBoundaryBit) {
            const R f = -pk.w * (pdd + pdd);
            if (c.single_layer) pa.add((f * g) * c.gamma2);
            else pa.add(f * g);
        } else {
            const R rj = s.rho[j];
            const R pddj = rj == R(0) ? R(0) : fdiv<KAHAN>(s.p[j], rj * rj);
            pa.add((-pj.w * (pdd + pddj)) * g);
        }
    });
    s.acc[k] = v4<R>(pa.get() + npa, R(0));
}

template <typename R, bool KAHAN>
__global__ void k_sesph_accel(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    if (s.type[k] != FS_TYPE_NORMAL) return;
    sesph_accel_one<R, KAHAN>(k, s, L, c);
}

// max |a|^2, |v + dt a|^2 over ALL particles (SESPHFluidSolver3D.hpp:93-107)
template <typename R>
__device__ __forceinline__ void sesph_maxima_at(int64_t k, const State<R>& s, const StepScalars* FSB_R sc, float& a2,
                                                float& v2) {
    const R dt = (R)sc->desired_dt;
    const V3<R> a = xyz<R>(s.acc[k]);
    a2 = (float)dot(a, a);
    const V3<R> v = xyz<R>(s.vel[k]) + dt * a;
    v2 = (float)dot(v, v);
    if (!(a2 >= 0.f)) a2 = 0.f;
    if (!(v2 >= 0.f)) v2 = 0.f;
}
template <typename R>
__global__ void k_sesph_maxima(int64_t n, State<R> s, StepScalars* FSB_R sc, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (*status) return;
    float a2 = 0.f, v2 = 0.f;
    if (k < n) sesph_maxima_at<R>(k, s, sc, a2, v2);
    a2 = warp_max(a2);
    v2 = warp_max(v2);
    if ((threadIdx.x & 31) == 0) {
        atomic_max_nonneg(&sc->max_a2_bits, a2);
        atomic_max_nonneg(&sc->max_v2_bits, v2);
    }
}

__device__ __forceinline__ void sesph_maxima_final_one(StepScalars* FSB_R sc) {
    const volatile StepScalars* v = sc;   // maxima from atomics (see generator_finish_one)
    sc->final_max_a2 = __uint_as_float(v->max_a2_bits);
    sc->final_max_v2 = __uint_as_float(v->max_v2_bits);
    sc->max_a2_bits = 0u;
    sc->max_v2_bits = 0u;
}
static __global__ void k_sesph_maxima_final(StepScalars* FSB_R sc) { sesph_maxima_final_one(sc); }

// Euler-Cromer for every active particle: v += dt a; x += dt v
template <typename R>
__device__ __forceinline__ void sesph_integrate_at(int64_t k, const State<R>& s, const StepScalars* FSB_R sc) {
    if (s.type[k] == FS_TYPE_INACTIVE) return;
    const R dt = (R)sc->dt;
    const V4<R> vv = s.vel[k];
    const V3<R> v = xyz<R>(vv) + dt * xyz<R>(s.acc[k]);
    const V4<R> p = s.pos[k];
    s.vel[k] = v4<R>(v, vv.w);
    s.pos[k] = v4<R>(xyz<R>(p) + dt * v, p.w);
}
template <typename R>
__global__ void k_sesph_integrate(int64_t n, State<R> s, const StepScalars* FSB_R sc,
                                  const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    sesph_integrate_at<R>(k, s, sc);
}

// ===========================================================================
// IISPH 2D (IISPHFluidSolver.hpp:139-525)
// ===========================================================================
// first loop (:160-167, 196-237): density (fluid), then non-pressure
// acceleration + v* (all active); viscosity reads neighbor densities as in the
// 3D first loop (SPLIT selects the serial-order emulation).
template <typename R, bool KAHAN, bool SPLIT>
__device__ __forceinline__ void iisph2d_l1_at(int64_t k, const State<R>& s, const Lists& L, const SolverConsts<R>& c,
                                              R dt) {
    const uint8_t t = s.type[k];
    if (t == FS_TYPE_INACTIVE) {
        if (!SPLIT) s.rho[k] = s.rho_prev[k];  // carry the density through the double buffer
        return;
    }
    const V4<R> pk = s.pos[k];
    const V4<R> vk = s.vel[k];
    R rho_k = s.rho_prev[k];
    if (t == FS_TYPE_NORMAL && !SPLIT) {
        Acc<R, KAHAN> rho;
        const uint32_t nn = L.size(k);
        for (uint32_t q = 0; q < nn; q++) {
            const V4<R> pj = s.pos[L.at(k, q) & kIndexMask];
            rho.add(pj.w * c.kern.template w<KAHAN>(xyz<R>(pk) - xyz<R>(pj)));
        }
        rho_k = rho.get();
    }
    if (SPLIT) rho_k = s.rho[k];
    V3<R> npa = xyz<R>(s.ext[k]);
    if (t != FS_TYPE_BOUNDARY) {
        npa = npa + v3<R>(R(0), -c.gravity, R(0));
        V3<R> visc;
        if (SPLIT) {
            const uint32_t hk = s.hidx[k];
            visc = viscosity<R, KAHAN>(k, s, L, c, xyz<R>(pk), xyz<R>(vk), [&](uint32_t j, uint32_t e) -> R {
                if (j == (uint32_t)k) return rho_k;
                if (!(e & kBoundaryBit) && s.hidx[j] < hk) return s.rho[j];
                return s.rho_prev[j];
            });
        } else {
            visc = viscosity<R, KAHAN>(k, s, L, c, xyz<R>(pk), xyz<R>(vk), [&](uint32_t j, uint32_t) -> R {
                return j == (uint32_t)k ? rho_k : s.rho_prev[j];
            });
        }
        npa = npa + visc;
    }
    s.vstar[k] = v4<R>(xyz<R>(vk) + dt * npa, R(0));
    s.ext[k] = v4<R>(v3<R>(R(0), R(0), R(0)), R(0));
    if (!SPLIT) s.rho[k] = rho_k;
}
template <typename R, bool KAHAN, bool SPLIT>
__global__ void k_iisph2d_l1(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const StepScalars* FSB_R sc,
                             const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph2d_l1_at<R, KAHAN, SPLIT>(k, s, L, c, (R)sc->dt);
}

// density for the split 2D first loop
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph2d_density_at(int64_t k, const State<R>& s, const Lists& L,
                                                   const SolverConsts<R>& c) {
    if (s.type[k] != FS_TYPE_NORMAL) {
        s.rho[k] = s.rho_prev[k];
        return;
    }
    const V3<R> xk = xyz<R>(s.pos[k]);
    Acc<R, KAHAN> rho;
    const uint32_t nn = L.size(k);
    for (uint32_t q = 0; q < nn; q++) {
        const V4<R> pj = s.pos[L.at(k, q) & kIndexMask];
        rho.add(pj.w * c.kern.template w<KAHAN>(xk - xyz<R>(pj)));
    }
    s.rho[k] = rho.get();
}
template <typename R, bool KAHAN>
__global__ void k_iisph2d_density(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph2d_density_at<R, KAHAN>(k, s, L, c);
}

// second loop (:170-180, 280-376): source term, diagonal element, p = 0.
// The reference's O(n^2) diagonal recomputes the same inner sum for every
// outer neighbor; it is computed once here (the value is identical).
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph2d_l2_at(int64_t k, const State<R>& s, const Lists& L, const SolverConsts<R>& c,
                                              R dt) {
    if (s.type[k] != FS_TYPE_NORMAL) return;
    const V4<R> pk = s.pos[k];
    const V3<R> xk = xyz<R>(pk);
    const V3<R> vsk = xyz<R>(s.vstar[k]);
    const uint32_t nn = L.size(k);
    Acc<R, KAHAN> sum;
    Acc3<R, KAHAN> internal;
    for (uint32_t q = 0; q < nn; q++) {
        const uint32_t e = L.at(k, q);
        const uint32_t j = e & kIndexMask;
        const V4<R> pj = s.pos[j];
        const V3<R> g = c.kern.template grad<KAHAN>(xk - xyz<R>(pj));
        sum.add(pj.w * dot(vsk - xyz<R>(s.vstar[j]), g));
        if (!(e & kBoundaryBit)) internal.add(((pj.w / c.rest_density) / c.rest_density) * g);
        else internal.add((((c.two_gamma * pj.w) / c.rest_density) / c.rest_density) * g);
    }
    const R source = (c.rest_density - s.rho[k]) - dt * sum.get();
    const V3<R> neg_in = -internal.get();
    const R mi = (pk.w / c.rest_density) / c.rest_density;
    Acc<R, KAHAN> d;
    for (uint32_t q = 0; q < nn; q++) {
        const V4<R> pj = s.pos[L.at(k, q) & kIndexMask];
        d.add(pj.w * dot(neg_in, c.kern.template grad<KAHAN>(xk - xyz<R>(pj))));
    }
    for (uint32_t q = 0; q < nn; q++) {
        const uint32_t e = L.at(k, q);
        if (e & kBoundaryBit) continue;
        const V4<R> pj = s.pos[e & kIndexMask];
        const V3<R> g = c.kern.template grad<KAHAN>(xk - xyz<R>(pj));
        d.add(pj.w * dot(mi * (-g), g));
    }
    s.vstar[k] = v4<R>(vsk, source);
    s.anp[k] = v4<R>(v3<R>(R(0), R(0), R(0)), (dt * dt) * d.get());
    s.p[k] = R(0);
}
template <typename R, bool KAHAN>
__global__ void k_iisph2d_l2(int64_t n, State<R> s, Lists L, SolverConsts<R> c, const StepScalars* FSB_R sc,
                             const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph2d_l2_at<R, KAHAN>(k, s, L, c, (R)sc->dt);
}

// 2D iteration (a) (:408-444): a_i = -sum
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph2d_pressure_acc_at(int64_t k, const State<R>& s, const Lists& L,
                                                        const SolverConsts<R>& c) {
    if (s.type[k] != FS_TYPE_NORMAL) return;
    const V3<R> xk = xyz<R>(s.pos[k]);
    const R pk = s.p[k];
    const R pr = (pk / c.rest_density) / c.rest_density;
    const uint32_t nn = L.size(k);
    Acc3<R, KAHAN> sum;
    for (uint32_t q = 0; q < nn; q++) {
        const uint32_t e = L.at(k, q);
        const uint32_t j = e & kIndexMask;
        const V4<R> pj = s.pos[j];
        const V3<R> g = c.kern.template grad<KAHAN>(xk - xyz<R>(pj));
        if (!(e & kBoundaryBit)) sum.add((pj.w * (pr + (s.p[j] / c.rest_density) / c.rest_density)) * g);
        else sum.add((((c.gamma * pj.w) * R(2)) * pr) * g);
    }
    s.acc[k] = v4<R>(-sum.get(), R(0));
}
template <typename R, bool KAHAN>
__global__ void k_iisph2d_pressure_acc(int64_t n, State<R> s, Lists L, SolverConsts<R> c,
                                       const StepScalars* FSB_R sc, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status || sc->done) return;
    iisph2d_pressure_acc_at<R, KAHAN>(k, s, L, c);
}

// 2D iteration (b) (:447-511): Ap = dt^2 sum, update, density error
// particle k's update; adds its error to e_sum / e_cnt
template <typename R, bool KAHAN>
__device__ __forceinline__ void iisph2d_pressure_update_at(int64_t k, const State<R>& s, const Lists& L,
                                                           const SolverConsts<R>& c, R dt, double& e_sum,
                                                           unsigned int& e_cnt) {
    if (s.type[k] == FS_TYPE_NORMAL) {
        const V3<R> xk = xyz<R>(s.pos[k]);
        const V3<R> ak = xyz<R>(s.acc[k]);
        const uint32_t nn = L.size(k);
        Acc<R, KAHAN> sum;
        for (uint32_t q = 0; q < nn; q++) {
            const uint32_t e = L.at(k, q);
            const uint32_t j = e & kIndexMask;
            const V4<R> pj = s.pos[j];
            const V3<R> g = c.kern.template grad<KAHAN>(xk - xyz<R>(pj));
            if (!(e & kBoundaryBit)) sum.add(pj.w * dot(ak - xyz<R>(s.acc[j]), g));
            else sum.add(pj.w * dot(ak, g));
        }
        const R Ap = (dt * dt) * sum.get();
        const R aii = s.anp[k].w;
        const R src = s.vstar[k].w;
        R p = s.p[k];
        const bool has_diag = abs_(aii) > R(kFltEps);
        if (has_diag) p = fmax_(R(0), p + c.omega * ((src - Ap) / aii));
        else p = R(0);
        s.p[k] = p;
        R perr = abs_(src - Ap);
        if (has_diag) {
            if (abs_(p) <= R(kFltEps)) perr = R(0);
            e_sum += (double)perr;
            e_cnt += 1;
        }
    }
}
template <typename R, bool KAHAN>
__global__ void k_iisph2d_pressure_update(int64_t n, State<R> s, Lists L, SolverConsts<R> c,
                                          StepScalars* FSB_R sc, const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (*status || sc->done) return;
    double e_sum = 0.0;
    unsigned int e_cnt = 0;
    if (k < n) iisph2d_pressure_update_at<R, KAHAN>(k, s, L, c, (R)sc->dt, e_sum, e_cnt);
    e_sum = warp_sum(e_sum);
    e_cnt = warp_sum(e_cnt);
    if ((threadIdx.x & 31) == 0 && e_cnt) {
        atomicAdd(&sc->err_sum, e_sum);
        atomicAdd(&sc->err_count, (unsigned long long)e_cnt);
    }
}

// 2D integration (:379-392): v = v* + dt a; x += dt v (no CFL clamp)
template <typename R>
__device__ __forceinline__ void iisph2d_integrate_at(int64_t k, const State<R>& s, const StepScalars* FSB_R sc) {
    if (s.type[k] == FS_TYPE_INACTIVE) return;
    const R dt = (R)sc->dt;
    const V3<R> v = xyz<R>(s.vstar[k]) + dt * xyz<R>(s.acc[k]);
    const V4<R> p = s.pos[k];
    s.vel[k] = v4<R>(v, s.vel[k].w);
    s.pos[k] = v4<R>(xyz<R>(p) + dt * v, p.w);
}
template <typename R>
__global__ void k_iisph2d_integrate(int64_t n, State<R> s, const StepScalars* FSB_R sc,
                                    const int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    iisph2d_integrate_at<R>(k, s, sc);
}

}  // namespace fsb
