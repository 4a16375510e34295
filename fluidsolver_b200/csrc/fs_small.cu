// The small-scene step kernel (fs_small.cuh): search and solver phases of
// whole steps in one block, in the order of the step-by-step path
// (fs_api.cu: search_impl, begin_solver_phases, step_sesph, step_iisph3d,
// step_iisph2d), each phase a block-stride loop over the particles that
// calls the same per-particle device function as the separate kernel does.
#define FSB_COHERENT_LOADS 1

#include <climits>

#include "fs_small.cuh"
#include "fs_sort.cuh"

namespace fsb {
namespace {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int status_now(const int* status) { return *(const volatile int*)status; }

// whether the status word is clear, decided once for the whole block (a
// barrier): every branch that holds a barrier depends on block-uniform values
__device__ __forceinline__ bool block_ok(const int* status) { return !__syncthreads_or(status_now(status)); }

template <typename R> __device__ __forceinline__ State<R> small_state(const SmallStepArgs<R>& a, int cur, R* rho) {
    State<R> s;
    const SmallBuffers& b = a.buf[cur];
    s.pos = (V4<R>*)b.pos;
    s.vel = (V4<R>*)b.vel;
    s.acc = (V4<R>*)b.acc;
    s.ext = (V4<R>*)b.ext;
    s.rho = rho;
    s.rho_prev = nullptr;
    s.p = (R*)b.p;
    s.vstar = (V4<R>*)a.vstar;
    s.anp = (V4<R>*)a.anp;
    s.err = (R*)a.err;
    s.gbnd = (V4<R>*)a.gbnd;
    s.type = b.type;
    s.hidx = b.hidx;
    s.scene = nullptr;
    return s;
}

// the search of one step (search_impl); returns the buffer set now current
template <typename R>
__device__ __forceinline__ int small_search(const SmallStepArgs<R>& a, int cur, R* const (&rho)[2],
                                            unsigned char* smem) {
    const int t = threadIdx.x;
    const int64_t n = a.n;
    {
        // bounding box of the cells (k_bbox; the bounds start from the
        // table's reset pattern) and the grid origin (k_origin)
        const V4<R>* pos = (const V4<R>*)a.buf[cur].pos;
        const uint8_t* type = a.buf[cur].type;
        int mn[3] = {0x7f7f7f7f, 0x7f7f7f7f, 0x7f7f7f7f};
        int mx[3] = {(int)0x80808080, (int)0x80808080, (int)0x80808080};
        for (int64_t k = t; k < n; k += kSmallThreads) {
            if (!a.include_inactive && type[k] == FS_TYPE_INACTIVE) continue;
            const V4<R> p = pos[k];
            const int cc[3] = {cell_coord<R>(p.x, a.radius, a.trunc), cell_coord<R>(p.y, a.radius, a.trunc),
                               cell_coord<R>(p.z, a.radius, a.trunc)};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                mn[d] = min(mn[d], cc[d]);
                mx[d] = max(mx[d], cc[d]);
            }
        }
        __shared__ int s_b[6][kSmallThreads / 32];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            mn[d] = __reduce_min_sync(0xffffffffu, mn[d]);
            mx[d] = __reduce_max_sync(0xffffffffu, mx[d]);
        }
        if ((t & 31) == 0) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                s_b[d][t >> 5] = mn[d];
                s_b[3 + d][t >> 5] = mx[d];
            }
        }
        __syncthreads();
        if (t < 32) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int lo = __reduce_min_sync(0xffffffffu, s_b[d][t]);
                const int hi = __reduce_max_sync(0xffffffffu, s_b[3 + d][t]);
                if (t == 0) {
                    a.bbox[d] = lo;
                    a.bbox[3 + d] = hi;
                }
            }
            if (t == 0) grid_origin_at(0, a.bbox, a.grids, 1);
        }
        __syncthreads();
    }
    // keys (k_keys)
    for (int64_t k = t; k < n; k += kSmallThreads)
        keys_at<R>(k, (const V4<R>*)a.buf[cur].pos, a.buf[cur].type, a.buf[cur].hidx, a.include_inactive,
                   a.single_region, a.radius, a.trunc, a.grids, nullptr, a.key_bits, a.keys[0], a.keys64[0],
                   a.perm[0], a.h2d_cell, a.h2d_rank, a.status);
    __syncthreads();
    // The reference-order keys carry the order inside a cell in their low 32
    // bits: a host index or a rank below kSmallMax, or an arrival flagged by
    // the top bit. Below kSmallMax particles it fits kOrderBits bits with the
    // flag moved down, which keeps every comparison and saves two or three
    // radix passes.
    const bool k64 = a.keys64[0] != nullptr;
    constexpr int kOrderBits = 14;
    static_assert(kSmallMax <= (1 << (kOrderBits - 1)), "the order field's values must fit below its flag bit");
    if (k64) {
        for (int64_t k = t; k < n; k += kSmallThreads) {
            const unsigned long long x = a.keys64[0][k];
            const uint32_t order = (uint32_t)x;
            const uint32_t o = (order & 0x80000000u) ? (1u << (kOrderBits - 1)) | (order & 0x7fffffffu) : order;
            a.keys64[0][k] = ((x >> 32) << kOrderBits) | o;
        }
        __syncthreads();
    }
    // stable sort of (key, index) in shared memory (sort_pairs: one block)
    int res = 0;
    if (n > 1) {
        if (k64)
            sort_small_block<unsigned long long>(n, kOrderBits + a.key_bits + 2, a.keys64[0], a.perm[0], a.keys64[1],
                                                 a.perm[1], smem);
        else
            sort_small_block<uint32_t>(n, a.key_bits + 2, a.keys[0], a.perm[0], a.keys[1], a.perm[1], smem);
        res = 1;
    }
    __syncthreads();
    // gather every persistent field into the other buffer set (k_reorder)
    const int nx = cur ^ 1;
    {
        const SmallBuffers &f = a.buf[cur], &g = a.buf[nx];
        for (int64_t k = t; k < n; k += kSmallThreads)
            reorder_at<R>(k, a.perm[res], (const V4<R>*)f.pos, (V4<R>*)g.pos, (const V4<R>*)f.vel, (V4<R>*)g.vel,
                          (const V4<R>*)f.acc, (V4<R>*)g.acc, (const V4<R>*)f.ext, (V4<R>*)g.ext, rho[cur], rho[nx],
                          (const R*)f.p, (R*)g.p, f.type, g.type, f.hidx, g.hidx, nullptr, nullptr);
    }
    __syncthreads();
    cur = nx;
    // cell-start table: zero, run counts, exclusive scan (cell_start_table)
    const int64_t table = (int64_t)a.regions * (a.cells + 1);
    for (int64_t i = t; i < table; i += kSmallThreads) a.cell_start[i] = 0u;
    __syncthreads();
    for (int64_t k = t; k < a.n_struct; k += kSmallThreads) {
        if (k64)
            cell_count_at<unsigned long long>(k, a.n_struct, a.keys64[res], kOrderBits, a.key_bits, a.cells,
                                              a.cell_start);
        else
            cell_count_at<uint32_t>(k, a.n_struct, a.keys[res], 0, a.key_bits, a.cells, a.cell_start);
    }
    __syncthreads();
    scan_exclusive_block<uint32_t, uint32_t>(a.cell_start, a.cell_start, table);
    __syncthreads();
    if (a.h2d_cell) {
        for (int64_t k = t; k < a.n_struct; k += kSmallThreads)
            h2d_rank_at(k, a.keys64[res], a.cells, a.key_bits, a.cell_start, a.buf[cur].hidx, a.h2d_rank, kOrderBits);
        __syncthreads();
    }
    // solver lists (k_build_lists; an overflow elsewhere does not stop the counting)
    {
        WalkParams w;
        w.r = a.radius;
        w.r2 = a.radius2;
        w.dim = a.dim;
        w.regions = a.regions;
        w.candidates_inactive = false;
        w.trunc = a.trunc;
        w.length_test = a.dim == 2;
        w.grids = a.grids;
        w.scene = nullptr;
        w.cells = a.cells;
        const int err = status_now(a.status);
        if (!err || err == FS_ERR_CAPACITY)
            for (int64_t k = t; k < a.n_owners; k += kSmallThreads)
                list_owner_at<R>(k, (const V4<R>*)a.buf[cur].pos, a.buf[cur].type, a.cell_start, w, a.owner_mask,
                                 a.rows, a.nbr, a.stride, a.K, a.count, a.status, a.sc);
        __syncthreads();
    }
    if (a.sort_by_host) {
        for (int64_t k = t; k < a.n_owners; k += kSmallThreads)
            sort_list_by_host_at(k, a.nbr, a.stride, a.K, a.count, a.buf[cur].hidx);
        __syncthreads();
    }
    return cur;
}

// the per-step scalars (k_step_begin) and, with the dynamic generator, the
// time step from the state (begin_solver_phases)
template <typename R>
__device__ __forceinline__ void small_begin_solver(const SmallStepArgs<R>& a, const State<R>& s) {
    const int t = threadIdx.x;
    if (t == 0) {
        StepScalars z{};
        z.desired_dt = a.desired_dt;
        z.dt = a.desired_dt;
        z.max_neighbors = ((const volatile StepScalars*)a.sc)->max_neighbors;
        *a.sc = z;
    }
    __syncthreads();
    if (!a.dynamic_generator) return;
    float v2 = 0.f, a2 = 0.f;
    for (int64_t k = t; k < a.n; k += kSmallThreads) {
        float x = 0.f, y = 0.f;
        if (generator_at<R>(k, s, x, y)) {
            v2 = fmaxf(v2, x);
            a2 = fmaxf(a2, y);
        }
    }
    v2 = warp_max(v2);
    a2 = warp_max(a2);
    if ((t & 31) == 0 && !status_now(a.status)) {
        atomic_max_nonneg(&a.sc->gen_v2_bits, v2);
        atomic_max_nonneg(&a.sc->gen_a2_bits, a2);
    }
    __syncthreads();
    if (t == 0) generator_finish_one(a.sc, a.particle_size, a.min_ts, a.max_ts, a.lambda_v, a.lambda_a);
    __syncthreads();
}

__device__ __forceinline__ void stamp(unsigned long long* stamps, int i) {
    if (threadIdx.x == 0) stamps[i] = global_ns();
}

template <typename R, bool KAHAN, int SOLVER>
__global__ void __launch_bounds__(kSmallThreads, 1) k_small_steps(SmallStepArgs<R> a) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    const int t = threadIdx.x;
    const int64_t n = a.n, no = a.n_owners;
    int cur = a.cur;
    R* rho[2] = {(R*)a.buf[0].rho, (R*)a.buf[1].rho};
    R* rho_prev = a.rho_prev;
    StepScalars* sc = a.sc;
    const Lists L{a.nbr, a.count, a.stride, a.K};
    for (int step = 0; step < a.steps; step++) {
        stamp(a.stamps, 0);
        if (t == 0) {
            StepScalars z{};
            z.desired_dt = a.desired_dt;
            z.dt = a.desired_dt;
            *sc = z;
        }
        __syncthreads();
        cur = small_search<R>(a, cur, rho, small_smem);
        if (SOLVER != kSmallSESPH) {
            // density double buffer: the current density becomes rho_prev
            R* x = rho[cur];
            rho[cur] = rho_prev;
            rho_prev = x;
        }
        State<R> s = small_state<R>(a, cur, rho[cur]);
        s.rho_prev = rho_prev;
        small_begin_solver<R>(a, s);
        stamp(a.stamps, 1);
        if constexpr (SOLVER == kSmallSESPH) {
            if (!status_now(a.status))
                for (int64_t k = t; k < no; k += kSmallThreads)
                    if (s.type[k] == FS_TYPE_NORMAL) sesph_density_one<R, KAHAN>(k, s, L, a.c);
            __syncthreads();
            stamp(a.stamps, 2);
            if (!status_now(a.status))
                for (int64_t k = t; k < no; k += kSmallThreads)
                    if (s.type[k] == FS_TYPE_NORMAL) sesph_accel_one<R, KAHAN>(k, s, L, a.c);
            __syncthreads();
            stamp(a.stamps, 3);
            if (a.dim == 3) {
                // maxima, CFL clamp (k_sesph_maxima, k_sesph_maxima_final, k_cfl)
                float a2 = 0.f, v2 = 0.f;
                if (!status_now(a.status))
                    for (int64_t k = t; k < n; k += kSmallThreads) {
                        float x = 0.f, y = 0.f;
                        sesph_maxima_at<R>(k, s, sc, x, y);
                        a2 = fmaxf(a2, x);
                        v2 = fmaxf(v2, y);
                    }
                a2 = warp_max(a2);
                v2 = warp_max(v2);
                if ((t & 31) == 0) {
                    atomic_max_nonneg(&sc->max_a2_bits, a2);
                    atomic_max_nonneg(&sc->max_v2_bits, v2);
                }
                __syncthreads();
                if (t == 0) {
                    sesph_maxima_final_one(sc);
                    if (!status_now(a.status)) cfl_one(sc, a.particle_size, a.cfl_timestep, a.lambda_v, a.lambda_a);
                }
                __syncthreads();
            }
            stamp(a.stamps, 4);
            if (!status_now(a.status))
                for (int64_t k = t; k < n; k += kSmallThreads) sesph_integrate_at<R>(k, s, sc);
            __syncthreads();
        } else {
            constexpr bool two_d = SOLVER == kSmallIISPH2D;
            // first loop
            const bool ok1 = block_ok(a.status);
            if (ok1 && a.split) {
                for (int64_t k = t; k < n; k += kSmallThreads) {
                    if (two_d) iisph2d_density_at<R, KAHAN>(k, s, L, a.c);
                    else iisph3d_density_at<R, KAHAN>(k, s, L, a.c);
                }
            }
            if (a.split) __syncthreads();
            if (ok1) {
                const R dt = (R)sc->dt;
                for (int64_t k = t; k < n; k += kSmallThreads) {
                    if (two_d) {
                        if (a.split) iisph2d_l1_at<R, KAHAN, true>(k, s, L, a.c, dt);
                        else iisph2d_l1_at<R, KAHAN, false>(k, s, L, a.c, dt);
                    } else {
                        if (a.split) iisph3d_l1_one<R, KAHAN, true>(k, s, L, a.c, dt);
                        else iisph3d_l1_one<R, KAHAN, false>(k, s, L, a.c, dt);
                    }
                }
            }
            __syncthreads();
            stamp(a.stamps, 2);
            // second loop
            if (!status_now(a.status)) {
                const R dt = (R)sc->dt;
                for (int64_t k = t; k < no; k += kSmallThreads) {
                    if (two_d) {
                        iisph2d_l2_at<R, KAHAN>(k, s, L, a.c, dt);
                    } else if (s.type[k] == FS_TYPE_NORMAL) {
                        if (a.fp32) iisph3d_l2_one<R, KAHAN, true>(k, s, L, a.c, dt);
                        else iisph3d_l2_one<R, KAHAN, false>(k, s, L, a.c, dt);
                    }
                }
            }
            __syncthreads();
            stamp(a.stamps, 3);
            // pressure iterations, each ended by the convergence test (k_iisph_check)
            const bool fp64_test = !a.fp32;
            for (int it = 0; it < a.max_it; it++) {
                const bool run = !__syncthreads_or(status_now(a.status) || ((const volatile StepScalars*)sc)->done);
                if (run)
                    for (int64_t k = t; k < no; k += kSmallThreads) {
                        if (two_d) iisph2d_pressure_acc_at<R, KAHAN>(k, s, L, a.c);
                        else if (s.type[k] == FS_TYPE_NORMAL) iisph3d_pressure_acc_one<R, KAHAN>(k, s, L, a.c);
                    }
                __syncthreads();
                if (run) {
                    const R dt = (R)sc->dt;
                    if (two_d) {
                        double e_sum = 0.0;
                        unsigned int e_cnt = 0;
                        for (int64_t k = t; k < no; k += kSmallThreads)
                            iisph2d_pressure_update_at<R, KAHAN>(k, s, L, a.c, dt, e_sum, e_cnt);
                        e_sum = warp_sum(e_sum);
                        e_cnt = warp_sum(e_cnt);
                        if ((t & 31) == 0 && e_cnt) {
                            atomicAdd(&sc->err_sum, e_sum);
                            atomicAdd(&sc->err_count, (unsigned long long)e_cnt);
                        }
                    } else {
                        ErrPart o;
                        for (int64_t k = t; k < no; k += kSmallThreads) {
                            if (s.type[k] != FS_TYPE_NORMAL) continue;
                            const ErrPart q = iisph3d_pressure_update_one<R, KAHAN>(k, s, L, a.c, dt);
                            o.e_sum += q.e_sum;
                            o.e_cnt += q.e_cnt;
                            o.e_max = fmaxf(o.e_max, q.e_max);
                            o.a2 = fmaxf(o.a2, q.a2);
                            o.v2 = fmaxf(o.v2, q.v2);
                        }
                        reduce_err_parts(o, sc);
                    }
                }
                __threadfence_block();
                __syncthreads();
                if (t == 0)
                    iisph_check_one(sc, a.min_it, a.max_it, a.max_err, fp64_test, two_d, a.status,
                                    cudaGraphConditionalHandle{}, false);
                const volatile StepScalars* v = sc;
                if (__syncthreads_or(status_now(a.status) || v->done)) break;
            }
            stamp(a.stamps, 4);
            if (!two_d) {
                if (t == 0 && !status_now(a.status))
                    cfl_one(sc, a.particle_size, a.cfl_timestep, a.lambda_v, a.lambda_a);
                __syncthreads();
            }
            if (!status_now(a.status))
                for (int64_t k = t; k < n; k += kSmallThreads) {
                    if (two_d) iisph2d_integrate_at<R>(k, s, sc);
                    else iisph3d_integrate_at<R>(k, s, sc);
                }
            __syncthreads();
        }
        stamp(a.stamps, 5);
    }
}

}  // namespace

size_t small_steps_smem(bool keys64) {
    return keys64 ? small_sort_smem<unsigned long long>() : small_sort_smem<uint32_t>();
}

template <typename R, bool KAHAN, int SOLVER>
cudaError_t launch_small_steps(const SmallStepArgs<R>& a, cudaStream_t st) {
    const size_t smem = small_steps_smem(a.keys64[0] != nullptr);
    static bool prepared = false;   // per process: the largest shared-memory size the kernel may ask for
    if (!prepared) {
        const cudaError_t e = cudaFuncSetAttribute(k_small_steps<R, KAHAN, SOLVER>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)small_steps_smem(true));
        if (e != cudaSuccess) return e;
        prepared = true;
    }
    k_small_steps<R, KAHAN, SOLVER><<<1, kSmallThreads, smem, st>>>(a);
    return cudaGetLastError();
}

#define FSB_SMALL_INSTANCE(R, KAHAN, SOLVER) \
    template cudaError_t launch_small_steps<R, KAHAN, SOLVER>(const SmallStepArgs<R>&, cudaStream_t);
FSB_SMALL_INSTANCE(float, true, kSmallSESPH)
FSB_SMALL_INSTANCE(float, true, kSmallIISPH3D)
FSB_SMALL_INSTANCE(float, true, kSmallIISPH2D)
FSB_SMALL_INSTANCE(float, false, kSmallSESPH)
FSB_SMALL_INSTANCE(float, false, kSmallIISPH3D)
FSB_SMALL_INSTANCE(float, false, kSmallIISPH2D)
FSB_SMALL_INSTANCE(double, false, kSmallSESPH)
FSB_SMALL_INSTANCE(double, false, kSmallIISPH3D)
FSB_SMALL_INSTANCE(double, false, kSmallIISPH2D)
#undef FSB_SMALL_INSTANCE

}  // namespace fsb
