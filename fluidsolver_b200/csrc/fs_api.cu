// C-ABI of the B200 hot path (declared in include/fluidsolver_b200.h):
// context management, host transfers, the neighborhood-search pipeline and
// the per-solver step sequences.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "fs_context.cuh"
#include "fs_search.cuh"
#include "fs_solvers.cuh"
#include "fs_entities.cuh"
#include "fs_io.hpp"
#include "fs_render.cuh"
#include "fs_small.cuh"

using namespace fsb;

namespace {

thread_local std::string g_error;

fs_status fail(fs_status s, const std::string& msg) {
    g_error = msg;
    return s;
}

#define FS_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(FS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

#define FS_TRY(call)                       \
    do {                                   \
        fs_status s_ = (call);             \
        if (s_ != FS_OK) return s_;        \
    } while (0)

constexpr int kBlock = 128;

inline unsigned grid_for(int64_t n, int block = kBlock) {
    int64_t g = (n + block - 1) / block;
    return (unsigned)std::max<int64_t>(g, 1);
}

template <typename T> fs_status dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    FS_CUDA(cudaMalloc((void**)p, count * sizeof(T)));
    return FS_OK;
}

// host-side replicas of the reference's float constants
float kernel_alpha(int dim, float h) {
    const float pi = 3.14159265358979323846f;
    if (dim == 2) return 5.0f / (14.0f * pi * (h * h));
    return 1.0f / (4.0f * pi * ((h * h) * h));
}

bool contract_is_2d(int search) {
    return search == FS_SEARCH_QUADRATIC_2D || search == FS_SEARCH_HASHED_2D || search == FS_SEARCH_COMPACT_2D;
}

// owners of the contract's lists, as a bit mask over particle types
uint32_t contract_owner_mask(int search) {
    const uint32_t normal = 1u << FS_TYPE_NORMAL, bnd = 1u << FS_TYPE_BOUNDARY, ina = 1u << FS_TYPE_INACTIVE;
    switch (search) {
        case FS_SEARCH_QUADRATIC_2D: return normal | bnd | ina;
        case FS_SEARCH_HASHED_2D: return normal;
        default: return normal | bnd;
    }
}

int contract_capacity(int search) {
    if (search == FS_SEARCH_COMPRESSED_3D) return 97;   // CompressedNeighbors.hpp:29-33 (first + 96 deltas)
    if (search == FS_SEARCH_COMPACT_2D) return 40;      // CompactHashingNeighborhoodSearch.cpp:5
    return 0;
}

template <typename R> State<R> state_of(fs_ctx* c) {
    State<R> s;
    s.pos = (V4<R>*)c->pos[c->cur];
    s.vel = (V4<R>*)c->vel[c->cur];
    s.acc = (V4<R>*)c->acc[c->cur];
    s.ext = (V4<R>*)c->ext[c->cur];
    s.rho = (R*)c->rho[c->cur];
    s.rho_prev = (R*)c->rho_prev;
    s.p = (R*)c->p[c->cur];
    s.vstar = (V4<R>*)c->vstar;
    s.anp = (V4<R>*)c->anp;
    s.err = (R*)c->err;
    s.gbnd = (V4<R>*)c->gbnd;
    s.type = c->type[c->cur];
    s.hidx = c->hidx[c->cur];
    s.scene = c->scene_of[c->cur];
    return s;
}

template <typename R> SolverConsts<R> consts_of(fs_ctx* c) {
    const fs_params& p = c->prm;
    SolverConsts<R> k;
    k.kern.h = (R)c->kernel_h;
    k.kern.alpha = (R)c->kernel_alpha;
    k.rest_density = (R)p.rest_density;
    k.rho0_sq = (R)(p.rest_density * p.rest_density);
    k.gravity = (R)p.gravity;
    k.visc_eps = (R)((0.01f * p.particle_size) * p.particle_size);
    k.two_nu = (R)(2.0f * p.viscosity);
    k.omega = (R)p.omega;
    k.gamma = (R)p.gamma;
    k.two_gamma = (R)(2.0f * p.gamma);
    k.gamma1 = (R)p.single_layer_gamma_1;
    k.gamma2 = (R)p.single_layer_gamma_2;
    k.stiffness = (R)p.stiffness;
    k.single_layer = c->dim == 3 && p.single_layer_boundary != 0;
    k.dim = c->dim;
    k.max_density_error = (R)p.max_density_error;
    k.min_iterations = p.min_iterations;
    k.max_iterations = p.max_iterations;
    if (std::is_same<R, double>::value) {
        // the FP64 build evaluates the same formulas in double
        const double h = (double)p.particle_size * 2.0 / 2.0;
        const double pi = 3.14159265358979323846;
        k.kern.h = (R)h;
        k.kern.alpha = (R)(c->dim == 2 ? 5.0 / (14.0 * pi * h * h) : 1.0 / (4.0 * pi * h * h * h));
        k.rho0_sq = (R)((double)p.rest_density * p.rest_density);
        k.visc_eps = (R)(0.01 * p.particle_size * p.particle_size);
        k.two_nu = (R)(2.0 * p.viscosity);
        k.two_gamma = (R)(2.0 * p.gamma);
    }
    k.inv_rho0_sq = R(1) / k.rho0_sq;
    k.kern.inv_h = R(1) / k.kern.h;
    k.kern.alpha_h = k.kern.alpha * k.kern.h;
    return k;
}

// The compensated-sum (fast) mode stores every list entry's kernel-gradient
// factor next to it; the exact modes evaluate the kernel in each pass.
// the 3D IISPH fast path runs on tile lists (fs_tiles.cuh)
bool tiled_mode(const fs_ctx* c) {
    return c->precision == FS_PRECISION_FP32_KAHAN && !c->reference_order && c->dim == 3 &&
           (c->prm.solver == FS_SOLVER_IISPH_3D || c->prm.solver == FS_SOLVER_SESPH_3D);
}

Lists lists_of(fs_ctx* c) {
    Lists L;
    L.nbr = c->nbr;
    L.count = c->nbr_count;
    L.stride = c->nbr_stride;
    L.K = c->nbr_capacity;
    return L;
}

TileLists tile_lists_of(fs_ctx* c) {
    TileLists T;
    T.desc = c->tile_desc;
    T.ent = c->tile_ent;
    T.count = c->nbr_count;
    T.stride = c->tile_stride;
    T.K = c->nbr_capacity;
    T.cap = c->tuning.cap;
    return T;
}

WalkParams walk_of(fs_ctx* c, bool for_solver) {
    WalkParams w;
    w.r = c->search_radius;
    w.r2 = c->radius2;
    w.dim = c->dim;
    w.regions = c->reference_order ? 1 : (c->include_inactive && !for_solver ? 3 : 2);
    w.candidates_inactive = c->include_inactive && !for_solver;
    w.trunc = c->truncate_cells;
    w.length_test = c->dim == 2;
    w.grids = c->grids;
    w.scene = c->scene_of[c->cur];
    w.cells = c->cells;
    w.table = c->hash_table;
    w.table_mask = c->hash_mask;
    return w;
}

fs_status check_params(const fs_params* p) {
    if (!p) return fail(FS_ERR_INVALID, "params is null");
    if (p->dim != 2 && p->dim != 3) return fail(FS_ERR_INVALID, "dim must be 2 or 3");
    if (p->search < FS_SEARCH_QUADRATIC_2D || p->search > FS_SEARCH_COMPRESSED_3D)
        return fail(FS_ERR_INVALID, "unknown search kind");
    if (contract_is_2d(p->search) != (p->dim == 2))
        return fail(FS_ERR_INVALID, "search kind does not match the dimension");
    if (p->solver == FS_SOLVER_SESPH_2D || p->solver == FS_SOLVER_IISPH_2D) {
        if (p->dim != 2) return fail(FS_ERR_INVALID, "2D solver needs dim 2");
    } else if (p->solver == FS_SOLVER_SESPH_3D || p->solver == FS_SOLVER_IISPH_3D) {
        if (p->dim != 3) return fail(FS_ERR_INVALID, "3D solver needs dim 3");
    } else if (p->solver != FS_SOLVER_NONE) {
        return fail(FS_ERR_INVALID, "unknown solver kind");
    }
    if (p->precision < 0 || p->precision > 2) return fail(FS_ERR_INVALID, "unknown precision");
    if (!(p->particle_size > 0.0f)) return fail(FS_ERR_INVALID, "Search radius is smaller or equal to zero.");
    if (p->solver == FS_SOLVER_IISPH_2D || p->solver == FS_SOLVER_IISPH_3D) {
        if (p->max_iterations < p->min_iterations)
            return fail(FS_ERR_INVALID, "Max iterations are less than min number of iterations.");
        if (!(p->max_density_error > 0.0f))
            return fail(FS_ERR_INVALID, "MaxDensityErrorAllowed is smaller or equal to zero.");
        if (p->min_iterations < 0) return fail(FS_ERR_INVALID, "min iterations must be >= 0");
    }
    if (p->timestep_generator != FS_TIMESTEP_CONSTANT && p->timestep_generator != FS_TIMESTEP_DYNAMIC_CFL)
        return fail(FS_ERR_INVALID, "unknown time step generator");
    if (p->timestep_generator == FS_TIMESTEP_CONSTANT) {
        if (p->solver != FS_SOLVER_NONE && !(p->timestep > 0.0f))
            return fail(FS_ERR_INVALID, "Timestep is smaller or equal to zero.");
    } else if (!(p->min_timestep > 0.0f) || !(p->max_timestep >= p->min_timestep)) {
        return fail(FS_ERR_INVALID, "the dynamic time step bounds need 0 < min_timestep <= max_timestep");
    }
    if (p->max_particles <= 0 || p->max_particles > (int64_t)0x7fffffff)
        return fail(FS_ERR_INVALID, "max_particles must be in [1, 2^31)");
    return FS_OK;
}

void derive(fs_ctx* c) {
    const fs_params& p = c->prm;
    c->dim = p.dim;
    c->precision = p.precision;
    c->real_size = p.precision == FS_PRECISION_FP64 ? 8 : 4;
    c->search_radius = p.particle_size * 2.0f;                 // kernel_support_factor (LibFluidMath.hpp:11)
    c->radius2 = c->search_radius * c->search_radius;         // HashedNeighborhoodSearch3D.cpp:305
    c->kernel_h = (p.particle_size * 2.0f) / 2.0f;             // CubicSplineKernel3D.cpp:69
    c->kernel_alpha = kernel_alpha(p.dim, c->kernel_h);
    c->reference_order = (p.flags & FS_FLAG_REFERENCE_ORDER) != 0;
    c->include_inactive = p.search == FS_SEARCH_QUADRATIC_2D || p.search == FS_SEARCH_HASHED_2D;
    c->truncate_cells = c->reference_order && p.search == FS_SEARCH_HASHED_2D;
    c->sort_lists_by_host = c->reference_order && (p.search == FS_SEARCH_QUADRATIC_2D || p.search == FS_SEARCH_QUADRATIC_3D);
}

// graphs bake in buffer pointers, sizes and settings: dropped whenever one changes
void clear_graphs(fs_ctx* c) {
    for (auto& g : c->solve_graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    c->solve_graphs.clear();
}

fs_status free_all(fs_ctx* c) {
    void* ptrs[] = {c->pos[0], c->pos[1], c->vel[0], c->vel[1], c->acc[0], c->acc[1], c->ext[0], c->ext[1],
                    c->rho[0], c->rho[1], c->p[0], c->p[1], c->type[0], c->type[1], c->hidx[0], c->hidx[1],
                    c->rho_prev, c->vstar, c->anp, c->err, c->gbnd, c->tile_desc, c->tile_ent, c->keys[0], c->keys[1], c->keys64[0], c->keys64[1],
                    c->perm[0], c->perm[1], c->h2d_cell, c->h2d_rank, c->sort_hist, c->hash_table, c->cell_start, c->cell_partials, c->bbox, c->grids, c->nbr, c->nbr_count,
                    c->scene_of[0], c->scene_of[1], c->d_scene_offsets,
                    c->csr_offsets, c->csr_indices, c->csr_counts, c->staging, c->status, c->small_stamps, c->scalars,
                    c->stats_parts, c->stats_out};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->scalars_host) cudaFreeHost(c->scalars_host);
    clear_graphs(c);
    if (c->body_stream) cudaStreamDestroy(c->body_stream);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    return FS_OK;
}

fs_status ensure_staging(fs_ctx* c, size_t bytes) {
    if (c->staging_bytes >= bytes) return FS_OK;
    if (c->staging) cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    FS_CUDA(cudaMalloc(&c->staging, bytes));
    c->staging_bytes = bytes;
    return FS_OK;
}

fs_status ensure_lists(fs_ctx* c, int K) {
    const int64_t stride = ((c->cap + 31) / 32) * 32;
    const bool tiled = tiled_mode(c);
    if (tiled) K = (K + 7) & ~7;   // tile lists hold octets of entries
    if (tiled && tile_build_smem(K, kTileCapMax) > (size_t)227 * 1024)
        return fail(FS_ERR_CAPACITY, "more neighbors per particle than the fast mode's list builder holds (704)");
    if (c->nbr && c->nbr_capacity >= K && c->nbr_stride == stride && (!tiled || c->tile_ent)) return FS_OK;
    clear_graphs(c);
    if (c->nbr) cudaFree(c->nbr);
    if (c->tile_ent) cudaFree(c->tile_ent);
    if (c->tile_desc) cudaFree(c->tile_desc);
    c->nbr = nullptr;
    c->tile_ent = nullptr;
    c->tile_desc = nullptr;
    FS_TRY(dalloc(&c->nbr, (size_t)K * stride));
    if (tiled) {
        const int64_t tiles = (c->cap + kTileOwners - 1) / kTileOwners;
        c->tile_stride = tiles * kTileOwners;
        FS_TRY(dalloc(&c->tile_desc, (size_t)tiles));
        FS_TRY(dalloc(&c->tile_ent, (size_t)(K / 8) * c->tile_stride));
        FS_CUDA(cudaFuncSetAttribute(k_build_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tile_build_smem(K, kTileCapMax)));
        FS_CUDA(set_tile_pass_smem(K));
    }
    c->nbr_capacity = K;
    c->nbr_stride = stride;
    return FS_OK;
}

// A scene's grid dims from the cell bounding box of its particles (lo > hi on
// an axis: no finite coordinate there): the box plus a margin of a sixteenth
// of its extent (at least 2 cells, which the 9-row walk needs) on each side,
// shrunk until the grid has at most max_cells cells. Particles that later
// leave the grid are clamped into its border cells and take the exact
// per-cell walk.
void choose_dims(int dim, int64_t max_cells, const int* lo_in, const int* hi_in, int* dims) {
    int lo[3] = {lo_in[0], lo_in[1], lo_in[2]}, hi[3] = {hi_in[0], hi_in[1], hi_in[2]};
    int64_t ext[3] = {1, 1, 1};
    for (int a = 0; a < dim; a++) {
        if (lo[a] > hi[a]) { lo[a] = hi[a] = 0; }
        int64_t e = (int64_t)hi[a] - lo[a] + 1;
        int64_t margin = std::max<int64_t>(2, e / 16);
        ext[a] = std::min<int64_t>(int64_t(1) << 20, e + 2 * margin);
    }
    while (ext[0] * ext[1] * ext[2] > max_cells) {
        int a = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
        ext[a] = std::max<int64_t>(1, (ext[a] * 3) / 4);
    }
    for (int a = 0; a < 3; a++) dims[a] = (int)ext[a];
}

// every scene's grid from its box (lo[3 s + a], hi[3 s + a]); scene s may
// hold up to max(4M, 8 * its particles) cells, and all scenes 2^30
fs_status choose_grids(fs_ctx* c, const int* lo, const int* hi) {
    const int S = c->nsc();
    c->grids_host.assign(S, SceneGrid{});
    int64_t base = 0;
    for (int sidx = 0; sidx < S; sidx++) {
        const int64_t np = c->scenes > 0 ? c->scene_offsets[sidx + 1] - c->scene_offsets[sidx] : c->cap;
        const int64_t max_cells = std::max<int64_t>(int64_t(1) << 22, 8 * std::max<int64_t>(np, 1));
        int d[3];
        choose_dims(c->dim, max_cells, lo + 3 * sidx, hi + 3 * sidx, d);
        SceneGrid& g = c->grids_host[sidx];
        g.d0 = d[0];
        g.d1 = d[1];
        g.d2 = d[2];
        g.base = base;
        base += (int64_t)d[0] * d[1] * d[2];
    }
    if (base > (int64_t(1) << 30)) return fail(FS_ERR_INVALID, "the scenes' cell grids exceed 2^30 cells");
    for (int a = 0; a < 3; a++) c->dims[a] = a == 0 ? c->grids_host[0].d0 : (a == 1 ? c->grids_host[0].d1 : c->grids_host[0].d2);
    c->cells = base;
    FS_CUDA(cudaMemcpyAsync(c->grids, c->grids_host.data(), sizeof(SceneGrid) * S, cudaMemcpyHostToDevice, c->stream));
    return FS_OK;
}

// cell tables for the current dims
fs_status ensure_cells(fs_ctx* c) {
    c->key_bits = 1;
    while ((int64_t(1) << c->key_bits) < c->cells) c->key_bits++;
    c->regions = c->reference_order ? 1 : (c->include_inactive ? 3 : 2);
    const int64_t need = c->cells + 1;
    if (!c->cell_start || c->cell_alloc < need) {
        clear_graphs(c);
        if (c->cell_start) cudaFree(c->cell_start);
        if (c->cell_partials) cudaFree(c->cell_partials);
        c->cell_start = c->cell_partials = nullptr;
        FS_TRY(dalloc(&c->cell_start, (size_t)3 * need));
        FS_TRY(dalloc(&c->cell_partials, (size_t)scan_tiles(3 * need)));
        c->cell_alloc = need;
    }
    return FS_OK;
}

// ---------------------------------------------------------------------------
// upload / download
// ---------------------------------------------------------------------------
// scene of host particle i: the last s with offsets[s] <= i
__device__ __forceinline__ int scene_of_host(const int64_t* __restrict__ offsets, int scenes, int64_t i) {
    int lo = 0, hi = scenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename R>
__global__ void k_pack(int64_t n, int dim, const float* __restrict__ pos, const float* __restrict__ vel,
                       const float* __restrict__ acc, const float* __restrict__ ext, const float* __restrict__ mass,
                       const float* __restrict__ rho, const float* __restrict__ p, const uint8_t* __restrict__ type,
                       float rest_density, State<R> s, uint8_t* __restrict__ type_out, uint32_t* __restrict__ hidx_out,
                       const int64_t* __restrict__ offsets, int scenes, uint16_t* __restrict__ scene_out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto ld = [&](const float* a) -> V3<R> {
        if (!a) return v3<R>(R(0), R(0), R(0));
        return dim == 2 ? v3<R>((R)a[2 * i], (R)a[2 * i + 1], R(0)) : v3<R>((R)a[3 * i], (R)a[3 * i + 1], (R)a[3 * i + 2]);
    };
    s.pos[i] = v4<R>(ld(pos), mass ? (R)mass[i] : R(1));
    s.vel[i] = v4<R>(ld(vel), R(0));
    s.acc[i] = v4<R>(ld(acc), R(0));
    s.ext[i] = v4<R>(ld(ext), R(0));
    s.rho[i] = rho ? (R)rho[i] : (R)rest_density;
    s.p[i] = p ? (R)p[i] : R(0);
    type_out[i] = type ? type[i] : (uint8_t)FS_TYPE_NORMAL;
    hidx_out[i] = (uint32_t)i;
    if (scene_out) scene_out[i] = (uint16_t)scene_of_host(offsets, scenes, i);
}

// field f of the sorted state, scattered to host order
template <typename R>
__global__ void k_unpack(int64_t n, int dim, int field, State<R> s, float* __restrict__ out, uint8_t* __restrict__ out_u8,
                         uint32_t* __restrict__ out_u32) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t h = s.hidx[k];
    auto st = [&](V3<R> v) {
        out[(int64_t)h * dim] = (float)v.x;
        out[(int64_t)h * dim + 1] = (float)v.y;
        if (dim == 3) out[(int64_t)h * dim + 2] = (float)v.z;
    };
    switch (field) {
        case 0: st(xyz<R>(s.pos[k])); break;
        case 1: st(xyz<R>(s.vel[k])); break;
        case 2: st(xyz<R>(s.acc[k])); break;
        case 3: st(xyz<R>(s.ext[k])); break;
        case 4: out[h] = (float)s.pos[k].w; break;
        case 5: out[h] = (float)s.rho[k]; break;
        case 6: out[h] = (float)s.p[k]; break;
        case 7: out_u8[h] = s.type[k]; break;
        case 8: out_u32[h] = h; break;
        case 9: st(xyz<R>(s.vstar[k])); break;
        case 10: st(xyz<R>(s.anp[k])); break;
        case 11: out[h] = (float)s.vstar[k].w; break;
        case 12: out[h] = (float)s.anp[k].w; break;
    }
}

// Upload census over the staged host arrays: particles per type (index 3:
// invalid types) and, per axis, the min/max of floor(x / r) over the finite
// coordinates (|x| < 1e30, clamped to +-1e9) of the particles that take part
// in the cell structure.
struct UploadCensus {
    unsigned long long counts[4];
};

// one particle per thread; per-scene boxes in bbox (mins [3 scenes], maxs
// [3 scenes]), reduced per block when the block lies in one scene
__global__ void k_census(int64_t n, int dim, const float* __restrict__ pos, const uint8_t* __restrict__ type, float r,
                         bool include_inactive, const int64_t* __restrict__ offsets, int scenes,
                         UploadCensus* __restrict__ out, int* __restrict__ bbox) {
    __shared__ unsigned int s_cnt[4];
    __shared__ int s_first;
    __shared__ int s_b[6][32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int sk = (i < n && offsets) ? scene_of_host(offsets, scenes, i) : 0;
    if (threadIdx.x < 4) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_first = sk;
    __syncthreads();
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    if (i < n) {
        const uint8_t t = type ? type[i] : (uint8_t)FS_TYPE_NORMAL;
        atomicAdd(&s_cnt[t <= 2 ? t : 3], 1u);
        if (include_inactive || t != FS_TYPE_INACTIVE) {
            for (int a = 0; a < dim; a++) {
                const float x = pos[i * dim + a];
                if (!(fabsf(x) < 1e30f)) continue;
                const int cc = (int)fmaxf(-1.0e9f, fminf(1.0e9f, floorf(x / r)));
                lo[a] = cc;
                hi[a] = cc;
            }
        }
    }
    const int s0 = s_first;
    const bool uniform = __syncthreads_and(i >= n || sk == s0);
    if (threadIdx.x < 4 && s_cnt[threadIdx.x]) atomicAdd(&out->counts[threadIdx.x], (unsigned long long)s_cnt[threadIdx.x]);
    if (!uniform) {
        for (int a = 0; a < 3; a++) {
            if (lo[a] != INT_MAX) atomicMin(&bbox[3 * sk + a], lo[a]);
            if (hi[a] != INT_MIN) atomicMax(&bbox[3 * scenes + 3 * sk + a], hi[a]);
        }
        return;
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int a = 0; a < 3; a++) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; a++) {
            s_b[a][wid] = lo[a];
            s_b[3 + a][wid] = hi[a];
        }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        for (int a = 0; a < 3; a++) {
            int l = lane < nw ? s_b[a][lane] : INT_MAX, h = lane < nw ? s_b[3 + a][lane] : INT_MIN;
            for (int o = 16; o > 0; o >>= 1) {
                l = min(l, __shfl_xor_sync(0xffffffffu, l, o));
                h = max(h, __shfl_xor_sync(0xffffffffu, h, o));
            }
            if (lane == 0) {
                if (l != INT_MAX) atomicMin(&bbox[3 * s0 + a], l);
                if (h != INT_MIN) atomicMax(&bbox[3 * scenes + 3 * s0 + a], h);
            }
        }
    }
}

// host arrays of one upload, staged in device memory
struct StagedUpload {
    const float *pos = nullptr, *vel = nullptr, *acc = nullptr, *ext = nullptr;
    const float *mass = nullptr, *rho = nullptr, *p = nullptr;
    const uint8_t* type = nullptr;
    UploadCensus* census = nullptr;
};

// resets the per-scene box table (mins high, maxs low)
fs_status reset_bbox(fs_ctx* c) {
    const int S = c->nsc();
    FS_CUDA(cudaMemsetAsync(c->bbox, 0x7f, 3 * S * sizeof(int), c->stream));
    FS_CUDA(cudaMemsetAsync(c->bbox + 3 * S, 0x80, 3 * S * sizeof(int), c->stream));
    return FS_OK;
}

// boxes: per-scene census box (mins [3 scenes], maxs [3 scenes])
fs_status stage_upload(fs_ctx* c, const fs_particles* in, StagedUpload& d, UploadCensus& h, std::vector<int>& boxes) {
    const int64_t n = in->n;
    const size_t vec = (size_t)n * c->dim * sizeof(float), sc = (size_t)n * sizeof(float);
    FS_TRY(ensure_staging(c, 4 * vec + 3 * sc + (size_t)n + 16 * 9 + sizeof(UploadCensus)));
    char* st = (char*)c->staging;
    size_t off = 0;
    cudaError_t e = cudaSuccess;
    auto put = [&](const void* src, size_t bytes) -> const void* {
        if (!src) return nullptr;
        char* dst = st + off;
        off += (bytes + 15) & ~size_t(15);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
        return dst;
    };
    d.pos = (const float*)put(in->position, vec);
    d.vel = (const float*)put(in->velocity, vec);
    d.acc = (const float*)put(in->acceleration, vec);
    d.ext = (const float*)put(in->external, vec);
    d.mass = (const float*)put(in->mass, sc);
    d.rho = (const float*)put(in->density, sc);
    d.p = (const float*)put(in->pressure, sc);
    d.type = (const uint8_t*)put(in->type, (size_t)n);
    d.census = (UploadCensus*)(st + off);
    h = UploadCensus{{0, 0, 0, 0}};
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.census, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, cudaGetErrorString(e));
    FS_TRY(reset_bbox(c));
    const int S = c->nsc();
    if (n > 0) {
        c->launches++;
        k_census<<<grid_for(n, 256), 256, 0, c->stream>>>(n, c->dim, d.pos, d.type, c->search_radius,
                                                           c->include_inactive, c->d_scene_offsets, S, d.census,
                                                           c->bbox);
        FS_CUDA(cudaGetLastError());
    }
    boxes.assign(6 * (size_t)S, 0);
    FS_CUDA(cudaMemcpyAsync(&h, d.census, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaMemcpyAsync(boxes.data(), c->bbox, sizeof(int) * 6 * S, cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

template <typename R> fs_status pack_upload(fs_ctx* c, const StagedUpload& d, int64_t n) {
    c->cur = 0;
    if (n == 0) return FS_OK;
    State<R> s = state_of<R>(c);
    c->launches++;
    k_pack<R><<<grid_for(n), kBlock, 0, c->stream>>>(n, c->dim, d.pos, d.vel, d.acc, d.ext, d.mass, d.rho, d.p, d.type,
                                                     c->prm.rest_density, s, c->type[0], c->hidx[0],
                                                     c->d_scene_offsets, c->nsc(), c->scene_of[0]);
    FS_CUDA(cudaGetLastError());
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

template <typename R> fs_status download_impl(fs_ctx* c, fs_particles* out) {
    const int64_t n = c->n;
    const int dim = c->dim;
    const size_t vec = (size_t)n * dim * sizeof(float);
    FS_TRY(ensure_staging(c, std::max<size_t>(vec, (size_t)n * 4) + 64));
    State<R> s = state_of<R>(c);
    struct F {
        int field;
        void* dst;
        size_t bytes;
    } fields[] = {
        {0, out->position, vec}, {1, out->velocity, vec}, {2, out->acceleration, vec}, {3, out->external, vec},
        {4, out->mass, (size_t)n * 4}, {5, out->density, (size_t)n * 4}, {6, out->pressure, (size_t)n * 4},
        {7, out->type, (size_t)n}, {8, out->tag, (size_t)n * 4}, {9, out->predicted_velocity, vec},
        {10, out->non_pressure_acceleration, vec}, {11, out->source_term, (size_t)n * 4},
        {12, out->diagonal_element, (size_t)n * 4},
    };
    for (auto& f : fields) {
        if (!f.dst) continue;
    c->launches++;
        k_unpack<R><<<grid_for(n), kBlock, 0, c->stream>>>(n, dim, f.field, s, (float*)c->staging,
                                                           (uint8_t*)c->staging, (uint32_t*)c->staging);
        FS_CUDA(cudaGetLastError());
        FS_CUDA(cudaMemcpyAsync(f.dst, c->staging, f.bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

// ---------------------------------------------------------------------------
// neighborhood search
// ---------------------------------------------------------------------------
// Compact hashing (2D): sort by the full (region, cell) key, gather, and
// enter the occupied cells into the hashed table (fs_search.cuh); the walks
// then look cells up by key, with no dense grid to clamp into.
template <typename R> fs_status compact_search_impl(fs_ctx* c, State<R> s, bool solver_lists) {
    const int64_t n = c->n;
    cudaStream_t st = c->stream;
    c->launches++;
    k_compact_keys<R><<<grid_for(n), kBlock, 0, st>>>(n, s.pos, s.type, c->include_inactive, c->reference_order,
                                                      c->search_radius, c->keys64[0], c->perm[0], c->status);
    FS_CUDA(cudaGetLastError());
    uint32_t* const vals[2] = {c->perm[0], c->perm[1]};
    unsigned long long* const kk[2] = {c->keys64[0], c->keys64[1]};
    const int res = sort_pairs(n, 64, kk, vals, c->sort_hist, st, c->launches);
    FS_CUDA(cudaGetLastError());
    const int nx = c->cur ^ 1;
    c->launches++;
    k_reorder<R><<<grid_for(n), kBlock, 0, st>>>(
        n, c->perm[res], (const V4<R>*)c->pos[c->cur], (V4<R>*)c->pos[nx], (const V4<R>*)c->vel[c->cur],
        (V4<R>*)c->vel[nx], (const V4<R>*)c->acc[c->cur], (V4<R>*)c->acc[nx], (const V4<R>*)c->ext[c->cur],
        (V4<R>*)c->ext[nx], (const R*)c->rho[c->cur], (R*)c->rho[nx], (const R*)c->p[c->cur], (R*)c->p[nx],
        c->type[c->cur], c->type[nx], c->hidx[c->cur], c->hidx[nx], c->scene_of[c->cur], c->scene_of[nx]);
    FS_CUDA(cudaGetLastError());
    c->cur = nx;
    s = state_of<R>(c);
    FS_CUDA(cudaMemsetAsync(c->hash_table, 0xff, sizeof(HashCell) * ((size_t)c->hash_mask + 1), st));
    c->launches++;
    k_hash_insert<<<grid_for(c->n_struct), kBlock, 0, st>>>(c->n_struct, c->keys64[res], c->hash_table, c->hash_mask);
    FS_CUDA(cudaGetLastError());
    if (solver_lists) {
        WalkParams w = walk_of(c, true);
        c->launches++;
        k_build_lists<R><<<grid_for(c->n_owners), kBlock, 0, st>>>(
            c->n_owners, s.pos, s.type, c->cell_start, w, 1u << FS_TYPE_NORMAL, false, c->nbr, c->nbr_stride,
            c->nbr_capacity, c->nbr_count, c->status, c->scalars);
        FS_CUDA(cudaGetLastError());
        c->have_lists = true;
    }
    c->have_cells = true;
    return FS_OK;
}

template <typename R> fs_status search_impl(fs_ctx* c, bool solver_lists) {
    const int64_t n = c->n;
    cudaStream_t st = c->stream;
    const bool single = c->reference_order;
    if (n == 0) {
        c->have_lists = solver_lists;
        c->have_cells = true;
        return FS_OK;
    }
    State<R> s = state_of<R>(c);
    if (c->hash_table) return compact_search_impl<R>(c, s, solver_lists);
    // bbox of the structure's cells -> grid origin
    FS_TRY(reset_bbox(c));
    c->launches++;
    const unsigned gb = c->scenes > 0 ? grid_for(n, 256) : std::min<unsigned>(grid_for(n, 256), 148u * 8u);
    k_bbox<R><<<gb, 256, 0, st>>>(n, s.pos, s.type, s.scene, c->nsc(), c->include_inactive,
                                                 c->search_radius, c->truncate_cells, c->bbox);
    c->launches++;
    k_origin<<<grid_for(c->nsc(), 128), 128, 0, st>>>(c->bbox, c->grids, c->nsc());
    // keys + sort
    unsigned long long* k64 = single ? c->keys64[0] : nullptr;
    const int pb = c->tuning.block;   // the per-particle kernels' block size (fs_autotune)
    c->launches++;
    k_keys<R><<<grid_for(n, pb), pb, 0, st>>>(n, s.pos, s.type, s.hidx, c->include_inactive, single, c->search_radius,
                                              c->truncate_cells, c->grids, s.scene, c->key_bits, c->keys[0], k64,
                                              c->perm[0], c->h2d_cell, c->h2d_rank, c->status);
    FS_CUDA(cudaGetLastError());
    // stable radix sort of (key, current index) over the key's bits (fs_sort.cuh)
    uint32_t* const vals[2] = {c->perm[0], c->perm[1]};
    int res;
    if (single) {
        unsigned long long* const kk[2] = {c->keys64[0], c->keys64[1]};
        res = sort_pairs(n, 32 + c->key_bits + 2, kk, vals, c->sort_hist, st, c->launches);
    } else {
        uint32_t* const kk[2] = {c->keys[0], c->keys[1]};
        res = sort_pairs(n, c->key_bits + 2, kk, vals, c->sort_hist, st, c->launches);
    }
    FS_CUDA(cudaGetLastError());
    // gather every persistent field into the other buffer
    const int nx = c->cur ^ 1;
    c->launches++;
    k_reorder<R><<<grid_for(n, pb), pb, 0, st>>>(
        n, c->perm[res], (const V4<R>*)c->pos[c->cur], (V4<R>*)c->pos[nx], (const V4<R>*)c->vel[c->cur],
        (V4<R>*)c->vel[nx], (const V4<R>*)c->acc[c->cur], (V4<R>*)c->acc[nx], (const V4<R>*)c->ext[c->cur],
        (V4<R>*)c->ext[nx], (const R*)c->rho[c->cur], (R*)c->rho[nx], (const R*)c->p[c->cur], (R*)c->p[nx],
        c->type[c->cur], c->type[nx], c->hidx[c->cur], c->hidx[nx], c->scene_of[c->cur], c->scene_of[nx]);
    FS_CUDA(cudaGetLastError());
    c->cur = nx;
    s = state_of<R>(c);
    // cell-start table of the concatenated per-region tables, read off the
    // sorted keys (regions are consecutive blocks of the sorted order)
    const int64_t table = (int64_t)c->regions * (c->cells + 1);
    if (single)
        cell_start_table<unsigned long long>(c->n_struct, c->keys64[res], 32, c->key_bits, c->cells, table,
                                             c->cell_start, c->cell_partials, pb, st, c->launches);
    else
        cell_start_table<uint32_t>(c->n_struct, c->keys[res], 0, c->key_bits, c->cells, table, c->cell_start,
                                   c->cell_partials, pb, st, c->launches);
    FS_CUDA(cudaGetLastError());
    if (c->h2d_cell) {
        c->launches++;
        k_h2d_rank<<<grid_for(c->n_struct), kBlock, 0, st>>>(c->n_struct, c->keys64[res], c->cells, c->key_bits,
                                                             c->cell_start, s.hidx, c->h2d_rank);
        FS_CUDA(cudaGetLastError());
    }
    if (solver_lists) {
        WalkParams w = walk_of(c, true);
        const uint32_t owners = 1u << FS_TYPE_NORMAL;
        const bool rows = !c->reference_order && c->dim == 3;
        bool built = false;
        if constexpr (std::is_same<R, float>::value) {
            if (tiled_mode(c) && c->n_owners > 0) {
                const int64_t tiles = (c->n_owners + kTileOwners - 1) / kTileOwners;
                c->launches++;
                k_build_tiles<<<(unsigned)tiles, kTileOwners, tile_build_smem(c->nbr_capacity, c->tuning.cap), st>>>(
                    c->n_owners, s.pos, s.type, c->cell_start, w, c->tile_desc, c->tile_ent, c->tile_stride, c->nbr,
                    c->nbr_stride, c->nbr_capacity, c->tuning.cap, c->nbr_count, c->status, c->scalars);
                built = true;
            }
        }
        if (!built) {
            c->launches++;
            k_build_lists<R><<<grid_for(c->n_owners), kBlock, 0, st>>>(
                c->n_owners, s.pos, s.type, c->cell_start, w, owners, rows, c->nbr, c->nbr_stride,
                c->nbr_capacity, c->nbr_count, c->status, c->scalars);
        }
        FS_CUDA(cudaGetLastError());
        if (c->sort_lists_by_host) {
    c->launches++;
            k_sort_lists_by_host<<<grid_for(c->n_owners), kBlock, 0, st>>>(c->n_owners, c->nbr, c->nbr_stride,
                                                                           c->nbr_capacity, c->nbr_count, s.hidx);
            FS_CUDA(cudaGetLastError());
        }
        c->have_lists = true;
    }
    c->have_cells = true;
    return FS_OK;
}

// layout bookkeeping after an upload: counts per type and owner range
void set_layout(fs_ctx* c, int64_t n, int64_t nf, int64_t nb, int64_t ni) {
    c->n = n;
    c->n_fluid = nf;
    c->n_boundary = nb;
    c->n_inactive = ni;
    c->n_struct = c->include_inactive ? n : nf + nb;
    c->n_owners = c->reference_order ? c->n_struct : nf;
}

fs_status read_scalars(fs_ctx* c) {
    FS_CUDA(cudaMemcpyAsync(c->scalars_host, c->scalars, sizeof(StepScalars) * c->nsc(), cudaMemcpyDeviceToHost,
                            c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

fs_status read_status(fs_ctx* c, int* st) {
    FS_CUDA(cudaMemcpyAsync(st, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

// Phase timestamp i on stream st. While the stream is being captured the
// event becomes an event-record node of the graph (recorded when the graph
// runs), so the phase times stay measurable in graph mode.
fs_status mark(fs_ctx* c, int i, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    FS_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs == cudaStreamCaptureStatusActive) FS_CUDA(cudaEventRecordWithFlags(c->ev[i], st, cudaEventRecordExternal));
    else FS_CUDA(cudaEventRecord(c->ev[i], st));
    return FS_OK;
}

// resets the per-step scalars; keep_search keeps the statistics of the
// search that precedes the solver phases
__global__ void k_step_begin(StepScalars* sc, int scenes, float desired_dt, bool keep_search) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= scenes) return;
    StepScalars z{};
    z.desired_dt = desired_dt;
    z.dt = desired_dt;
    if (keep_search) z.max_neighbors = sc[i].max_neighbors;
    sc[i] = z;
}

bool dynamic_timestep(const fs_ctx* c) { return c->prm.timestep_generator == FS_TIMESTEP_DYNAMIC_CFL; }

// the desired time step a step call starts from: the caller's (or the
// constant generator's); with the dynamic generator a placeholder, which the
// device replaces (a fixed value, so that one CUDA graph serves every step)
float desired_of(const fs_ctx* c, float desired_dt) {
    if (dynamic_timestep(c)) return c->prm.max_timestep;
    return desired_dt > 0.0f ? desired_dt : c->prm.timestep;
}

// the default of get_non_cfl_validating_timestep: the constant generator's
// time step or the dynamic generator's max_timestep
float cfl_default(const fs_ctx* c) { return dynamic_timestep(c) ? c->prm.max_timestep : c->prm.timestep; }

// Resets the step scalars before the solver phases; with the dynamic
// generator also chooses the desired time step from the state on the device
// (Simulator.cpp:18-25 runs the generator before the step).
fs_status begin_solver_phases(fs_ctx* c, float dt, cudaStream_t st) {
    c->launches++;
    k_step_begin<<<grid_for(c->nsc(), 128), 128, 0, st>>>(c->scalars, c->nsc(), dt, true);
    FS_CUDA(cudaGetLastError());
    if (!dynamic_timestep(c)) return FS_OK;
    const fs_params& p = c->prm;
    c->launches += 2;
    if (c->precision == FS_PRECISION_FP64)
        k_generator_max<double><<<grid_for(c->n, 256), 256, 0, st>>>(c->n, state_of<double>(c), c->scalars, c->status);
    else
        k_generator_max<float><<<grid_for(c->n, 256), 256, 0, st>>>(c->n, state_of<float>(c), c->scalars, c->status);
    k_generator_finish<<<grid_for(c->nsc(), 128), 128, 0, st>>>(c->scalars, c->nsc(), p.particle_size, p.min_timestep,
                                                                 p.max_timestep, p.lambda_v, p.lambda_a);
    FS_CUDA(cudaGetLastError());
    return FS_OK;
}

// ---------------------------------------------------------------------------
// solver steps
// ---------------------------------------------------------------------------
// Launches kernel<<<grid, block, smem, st>>>(args...), as a programmatic
// dependent of the kernel before it on st when pdl is set (the kernel then
// calls grid_dependency_wait before it reads that kernel's results).
template <typename... KArgs, typename... Args>
void launch_pdl(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// The IISPH pressure iterations. Eagerly, the host reads the exit flag after
// every iteration. While the stream is being captured, the loop becomes a
// conditional WHILE node: its body is the iteration followed by the
// convergence test, which ends the loop on the device (and always within
// max_iterations executions, see k_iisph_check).
template <typename Body>
// first_done: the first iteration already ran fused into the preceding
// phase (its scalars are accumulated); its test runs first, outside the loop.
// body(stream) enqueues one iteration and returns whether the convergence
// test (k_iisph_check, which follows it) may start as a programmatic
// dependent of the iteration's last kernel (launch_pdl).
fs_status enqueue_pressure_loop(fs_ctx* c, bool capture, bool two_d, bool fp64_test, Body&& body,
                                bool first_done = false) {
    const int max_it = c->prm.max_iterations;
    if (max_it <= 0) return FS_OK;
    cudaStream_t st = c->stream;
    auto check = [&](cudaStream_t s, cudaGraphConditionalHandle h, bool set, bool pdl = false) {
        c->launches++;
        if (c->scenes > 0)
            launch_pdl(pdl, k_iisph_check_scenes, 1, 256, 0, s, c->scalars, c->scenes, c->prm.min_iterations, max_it,
                       c->prm.max_density_error, (const int*)c->status, h, set);
        else
            launch_pdl(pdl, k_iisph_check, 1, 1, 0, s, c->scalars, c->prm.min_iterations, max_it,
                       c->prm.max_density_error, fp64_test, two_d, (const int*)c->status, h, set);
    };
    if (!capture) {
        auto all_done = [&]() -> fs_status {
            FS_CUDA(cudaGetLastError());
            FS_TRY(read_scalars(c));
            bool d = true;
            for (int i = 0; i < c->nsc(); i++) d = d && c->scalars_host[i].done;
            return d ? FS_ERR_STATE : FS_OK;   // FS_ERR_STATE here only means "stop"
        };
        if (first_done) {
            check(st, 0, false);
            if (all_done() != FS_OK) return FS_OK;
        }
        for (int it = first_done ? 1 : 0; it < max_it; it++) {
            const bool pdl = body(st);
            check(st, 0, false, pdl);
            if (all_done() != FS_OK) break;
        }
        return FS_OK;
    }
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t graph;
    FS_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps));
    cudaGraphConditionalHandle handle;
    FS_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    if (first_done) {
        // the fused first iteration's test sets the loop's initial condition
        check(st, handle, true);
        FS_CUDA(cudaGetLastError());
        FS_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps));
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    FS_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &cp));
    cudaGraph_t body_graph = cp.conditional.phGraph_out[0];
    FS_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    FS_CUDA(cudaStreamBeginCaptureToGraph(c->body_stream, body_graph, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    const bool pdl = body(c->body_stream);
    check(c->body_stream, handle, true, pdl);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(c->body_stream, nullptr);
    if (e != cudaSuccess || e2 != cudaSuccess) return fail(FS_ERR_CUDA, "capture of the pressure loop failed");
    return FS_OK;
}

// One pressure iteration on tile lists: the acceleration pass, then the
// update as its programmatic dependent (it reads what that pass does not
// write before it waits); the convergence test follows (enqueue_pressure_loop).
#define FSB_ACC_LAUNCH(...) __VA_ARGS__<<<tiles, threads, acc_smem, bs>>>(nf, s, T, L, k, c->scalars, c->status)
#define FSB_UPDATE_LAUNCH(...) \
    launch_pdl(true, __VA_ARGS__, tiles, threads, upd_smem, bs, nf, s, T, L, k, c->scalars, c->status)
void enqueue_tile_pressure_iteration(fs_ctx* c, cudaStream_t bs, unsigned tiles, int64_t nf, const State<float>& s,
                                     const TileLists& T, const Lists& L, const SolverConsts<float>& k) {
    const int tpo = c->tuning.pressure_tpo;
    const unsigned threads = (unsigned)(kTileOwners * tpo);
    const size_t acc_smem = tile_pass_smem(20, T.K, false, T.cap), upd_smem = tile_pass_smem(32, T.K, false, T.cap);
    FSB_PRESSURE_SWITCH(c->tuning.pressure_ahead, tpo, k_tile_iisph3d_pressure_acc, FSB_ACC_LAUNCH)
    FSB_PRESSURE_SWITCH(c->tuning.pressure_ahead, tpo, k_tile_iisph3d_pressure_update, FSB_UPDATE_LAUNCH)
}
#undef FSB_ACC_LAUNCH
#undef FSB_UPDATE_LAUNCH

// the IISPH 3D step on tile lists (fs_tiles.cuh)
fs_status step_iisph3d_tiled(fs_ctx* c, bool capture) {
    cudaStream_t st = c->stream;
    const int64_t n = c->n, nf = c->n_owners;
    const unsigned tiles = (unsigned)((nf + kTileOwners - 1) / kTileOwners);
    const unsigned rest = (unsigned)((n - nf + kPassThreads - 1) / kPassThreads);
    const SolverConsts<float> k = consts_of<float>(c);
    const Lists L = lists_of(c);
    const TileLists T = tile_lists_of(c);
    std::swap(c->rho[c->cur], c->rho_prev);
    State<float> s = state_of<float>(c);
    FS_TRY(mark(c, 1, st));
    c->launches++;
    FSB_AHEAD_SWITCH(c->tuning.l1_ahead, k_tile_iisph3d_l1,
                     <<<tiles + rest, kPassThreads, tile_pass_smem(36, T.K, !kL1GlobalEntries, T.cap), st>>>(
                         nf, n, tiles, s, T, L, k, c->scalars, c->status))
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 2, st));
    c->launches++;
    k_tile_iisph3d_l2<<<tiles, kPassThreads, tile_pass_smem(32, T.K, !kL2GlobalEntries, T.cap), st>>>(
        nf, s, T, L, k, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 3, st));
    // the second loop also ran the first pressure iteration (fs_tiles.cuh)
    FS_TRY(enqueue_pressure_loop(c, capture, false, true, [&](cudaStream_t bs) {
        c->launches += 2;
        enqueue_tile_pressure_iteration(c, bs, tiles, nf, s, T, L, k);
        return true;
    }, true));
    FS_TRY(mark(c, 4, st));
    c->launches++;
    k_cfl<<<1, 128, 0, st>>>(c->scalars, c->nsc(), c->prm.particle_size, cfl_default(c), c->prm.lambda_v,
                             c->prm.lambda_a, c->status);
    c->launches++;
    k_iisph3d_integrate<float><<<grid_for(n, c->tuning.block), c->tuning.block, 0, st>>>(n, s, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 5, st));
    return FS_OK;
}

template <typename R, bool KAHAN> fs_status step_iisph3d(fs_ctx* c, bool capture) {
    if constexpr (std::is_same<R, float>::value && KAHAN) {
        if (tiled_mode(c) && c->n_owners > 0) return step_iisph3d_tiled(c, capture);
    }
    cudaStream_t st = c->stream;
    const int64_t n = c->n, no = c->n_owners;
    const SolverConsts<R> k = consts_of<R>(c);
    const Lists L = lists_of(c);
    const bool split = c->reference_order;
    const bool fp32 = c->precision == FS_PRECISION_FP32;
    // density double buffer: the current density becomes rho_prev
    std::swap(c->rho[c->cur], c->rho_prev);
    State<R> s = state_of<R>(c);
    FS_TRY(mark(c, 1, st));
    if (split) {
    c->launches++;
        k_iisph3d_density<R, KAHAN><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->status);
    c->launches++;
        k_iisph3d_l1<R, KAHAN, true><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->scalars, c->status);
    } else {
    c->launches++;
        k_iisph3d_l1<R, KAHAN, false><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->scalars, c->status);
    }
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 2, st));
    if (fp32) {
    c->launches++;
        k_iisph3d_l2<R, KAHAN, true><<<grid_for(no), kBlock, 0, st>>>(no, s, L, k, c->scalars, c->status);
    } else {
    c->launches++;
        k_iisph3d_l2<R, KAHAN, false><<<grid_for(no), kBlock, 0, st>>>(no, s, L, k, c->scalars, c->status);
    }
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 3, st));
    FS_TRY(enqueue_pressure_loop(c, capture, false, !fp32, [&](cudaStream_t bs) {
        c->launches += 2;
        k_iisph3d_pressure_acc<R, KAHAN><<<grid_for(no), kBlock, 0, bs>>>(no, s, L, k, c->scalars, c->status);
        k_iisph3d_pressure_update<R, KAHAN><<<grid_for(no), kBlock, 0, bs>>>(no, s, L, k, c->scalars, c->status);
        return false;
    }));
    FS_TRY(mark(c, 4, st));
    c->launches++;
    k_cfl<<<1, 128, 0, st>>>(c->scalars, c->nsc(), c->prm.particle_size, cfl_default(c), c->prm.lambda_v,
                             c->prm.lambda_a, c->status);
    c->launches++;
    k_iisph3d_integrate<R><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 5, st));
    return FS_OK;
}

// 3D SESPH in the fast mode on tile lists (fs_tiles.cuh): the density and
// acceleration passes; maxima, CFL clamp and integration as in step_sesph
fs_status step_sesph3d_tiled(fs_ctx* c) {
    cudaStream_t st = c->stream;
    const int64_t n = c->n, nf = c->n_owners;
    const unsigned tiles = (unsigned)((nf + kTileOwners - 1) / kTileOwners);
    const SolverConsts<float> k = consts_of<float>(c);
    const Lists L = lists_of(c);
    const TileLists T = tile_lists_of(c);
    State<float> s = state_of<float>(c);
    FS_TRY(mark(c, 1, st));
    c->launches++;
    FSB_AHEAD_SWITCH(c->tuning.l1_ahead, k_tile_sesph3d_density,
                     <<<tiles, kPassThreads, tile_pass_smem(16, T.K, false, T.cap), st>>>(nf, s, T, L, k, c->status))
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 2, st));
    c->launches++;
    FSB_AHEAD_SWITCH(c->tuning.l1_ahead, k_tile_sesph3d_accel,
                     <<<tiles, kPassThreads, tile_pass_smem(36, T.K, false, T.cap), st>>>(nf, s, T, L, k, c->status))
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 3, st));
    c->launches++;
    k_sesph_maxima<float><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    c->launches++;
    k_sesph_maxima_final<<<1, 1, 0, st>>>(c->scalars);
    c->launches++;
    k_cfl<<<1, 128, 0, st>>>(c->scalars, c->nsc(), c->prm.particle_size, cfl_default(c), c->prm.lambda_v,
                             c->prm.lambda_a, c->status);
    FS_TRY(mark(c, 4, st));
    c->launches++;
    k_sesph_integrate<float><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 5, st));
    return FS_OK;
}

template <typename R, bool KAHAN> fs_status step_sesph(fs_ctx* c) {
    if constexpr (std::is_same<R, float>::value && KAHAN) {
        if (tiled_mode(c) && c->n_owners > 0) return step_sesph3d_tiled(c);
    }
    cudaStream_t st = c->stream;
    const int64_t n = c->n, no = c->n_owners;
    const SolverConsts<R> k = consts_of<R>(c);
    const Lists L = lists_of(c);
    State<R> s = state_of<R>(c);
    FS_TRY(mark(c, 1, st));
    c->launches++;
    k_sesph_density<R, KAHAN><<<grid_for(no), kBlock, 0, st>>>(no, s, L, k, c->status);
    FS_TRY(mark(c, 2, st));
    c->launches++;
    k_sesph_accel<R, KAHAN><<<grid_for(no), kBlock, 0, st>>>(no, s, L, k, c->status);
    FS_TRY(mark(c, 3, st));
    if (c->dim == 3) {
    c->launches++;
        k_sesph_maxima<R><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    c->launches++;
        k_sesph_maxima_final<<<1, 1, 0, st>>>(c->scalars);
    c->launches++;
        k_cfl<<<1, 128, 0, st>>>(c->scalars, c->nsc(), c->prm.particle_size, cfl_default(c), c->prm.lambda_v,
                                 c->prm.lambda_a, c->status);
    }
    FS_TRY(mark(c, 4, st));
    c->launches++;
    k_sesph_integrate<R><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 5, st));
    return FS_OK;
}

template <typename R, bool KAHAN> fs_status step_iisph2d(fs_ctx* c, bool capture) {
    cudaStream_t st = c->stream;
    const int64_t n = c->n, no = c->n_owners;
    const SolverConsts<R> k = consts_of<R>(c);
    const Lists L = lists_of(c);
    const bool split = c->reference_order;
    std::swap(c->rho[c->cur], c->rho_prev);
    State<R> s = state_of<R>(c);
    FS_TRY(mark(c, 1, st));
    if (split) {
    c->launches++;
        k_iisph2d_density<R, KAHAN><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->status);
    c->launches++;
        k_iisph2d_l1<R, KAHAN, true><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->scalars, c->status);
    } else {
    c->launches++;
        k_iisph2d_l1<R, KAHAN, false><<<grid_for(n), kBlock, 0, st>>>(n, s, L, k, c->scalars, c->status);
    }
    FS_TRY(mark(c, 2, st));
    c->launches++;
    k_iisph2d_l2<R, KAHAN><<<grid_for(no), kBlock, 0, st>>>(no, s, L, k, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 3, st));
    FS_TRY(enqueue_pressure_loop(c, capture, true, c->precision != FS_PRECISION_FP32,
                                 [&](cudaStream_t bs) {
        c->launches += 2;
        k_iisph2d_pressure_acc<R, KAHAN><<<grid_for(no), kBlock, 0, bs>>>(no, s, L, k, c->scalars, c->status);
        k_iisph2d_pressure_update<R, KAHAN><<<grid_for(no), kBlock, 0, bs>>>(no, s, L, k, c->scalars, c->status);
        return false;
    }));
    FS_TRY(mark(c, 4, st));
    c->launches++;
    k_iisph2d_integrate<R><<<grid_for(n), kBlock, 0, st>>>(n, s, c->scalars, c->status);
    FS_CUDA(cudaGetLastError());
    FS_TRY(mark(c, 5, st));
    return FS_OK;
}

template <typename R, bool KAHAN> fs_status step_dispatch(fs_ctx* c, bool capture) {
    switch (c->prm.solver) {
        case FS_SOLVER_IISPH_3D: return step_iisph3d<R, KAHAN>(c, capture);
        case FS_SOLVER_SESPH_2D:
        case FS_SOLVER_SESPH_3D: return step_sesph<R, KAHAN>(c);
        case FS_SOLVER_IISPH_2D: return step_iisph2d<R, KAHAN>(c, capture);
        default: return fail(FS_ERR_INVALID, "context has no solver");
    }
}

fs_status step_dispatch_any(fs_ctx* c, bool capture) {
    if (c->precision == FS_PRECISION_FP64) return step_dispatch<double, false>(c, capture);
    if (c->precision == FS_PRECISION_FP32) return step_dispatch<float, false>(c, capture);
    return step_dispatch<float, true>(c, capture);
}

fs_status search_dispatch(fs_ctx* c, bool solver_lists) {
    if (c->precision == FS_PRECISION_FP64) return search_impl<double>(c, solver_lists);
    return search_impl<float>(c, solver_lists);
}

// the statistics of scenes [0, entries) (the search's largest list is
// counted in scene 0's scalars for all scenes)
fs_status fill_stats(fs_ctx* c, fs_step_stats* stats, int st, int entries = 1) {
    if (!stats) return FS_OK;
    for (int i = 0; i < std::min(entries, c->nsc()); i++) {
        const StepScalars& h = c->scalars_host[i];
        fs_step_stats& o = stats[i];
        o.desired_dt = h.desired_dt;
        o.actual_dt = h.dt;
        o.iterations = h.iteration;
        o.avg_density_error = h.avg_err;
        o.avg_density_error_fp64 = h.avg_err64;
        o.max_density_error = h.max_err;
        o.max_velocity = std::sqrt(h.final_max_v2);
        o.max_acceleration = std::sqrt(h.final_max_a2);
        o.status = st;
        o.max_neighbors = c->scalars_host[0].max_neighbors;
    }
    return FS_OK;
}

// neighborhood search of a step (with solver lists). A list overflow stops
// every later kernel (they check the status word); with an automatic
// capacity the lists are grown and the search is repeated once.
fs_status search_for_step(fs_ctx* c, float dt) {
    for (int attempt = 0; attempt < 3; attempt++) {
        c->launches++;
        k_step_begin<<<grid_for(c->nsc(), 128), 128, 0, c->stream>>>(c->scalars, c->nsc(), dt, false);
        FS_CUDA(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
        cudaEventRecord(c->ev[0], c->stream);
        FS_TRY(search_dispatch(c, c->prm.solver != FS_SOLVER_NONE));
        int st = 0;
        FS_TRY(read_status(c, &st));
        if (st == FS_ERR_CAPACITY && attempt < 2 && c->prm.neighbor_capacity == 0 &&
            c->prm.solver != FS_SOLVER_NONE) {
            FS_TRY(read_scalars(c));
            int K = 32;
            while (K < c->scalars_host->max_neighbors) K *= 2;
            FS_TRY(ensure_lists(c, K));
            continue;
        }
        if (st != FS_OK)
            return fail((fs_status)st, st == FS_ERR_CAPACITY ? "neighbor list capacity exceeded"
                                                             : "device reported an error during the search");
        c->searched_dt = dt;
        return FS_OK;
    }
    return fail(FS_ERR_CAPACITY, "neighbor list capacity exceeded");
}

// Solver phases as one CUDA graph (the IISPH loop a conditional node in it),
// captured once per buffer assignment and reused. Capturing runs the same
// host code as the eager path, which also rotates the host-side buffer
// pointers; a replay applies the rotation recorded at capture time.
// with_search: the graph also holds the neighborhood search of the step (no
// host synchronisation inside the step; a list overflow is found afterwards
// in the status word, which the search sets and every solver kernel honours).
fs_status solve_graph(fs_ctx* c, float dt, bool with_search = false) {
    fs_ctx::SolveGraph key;
    key.cur = c->cur;
    key.rho0 = c->rho[0];
    key.rho1 = c->rho[1];
    key.rho_prev = c->rho_prev;
    key.K = c->nbr_capacity;
    key.n = c->n;
    key.n_owners = c->n_owners;
    key.dt = dt;
    key.with_search = with_search;
    key.cells = c->cells;
    key.dims0 = c->dims[0];
    key.dims1 = c->dims[1];
    for (auto& g : c->solve_graphs) {
        if (g.same_key(key)) {
            const int64_t per_launch = g.launches;
            FS_CUDA(cudaGraphLaunch(g.exec, c->stream));
            c->launches += per_launch;
            c->cur = g.post_cur;
            c->rho[0] = g.post_rho0;
            c->rho[1] = g.post_rho1;
            c->rho_prev = g.post_rho_prev;
            return FS_OK;
        }
    }
    const int64_t launches0 = c->launches;
    FS_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    fs_status r = FS_OK;
    if (with_search) {
        c->launches++;
        k_step_begin<<<grid_for(c->nsc(), 128), 128, 0, c->stream>>>(c->scalars, c->nsc(), dt, false);
        r = mark(c, 0, c->stream);
        if (r == FS_OK) r = search_dispatch(c, true);
    }
    if (r == FS_OK) r = begin_solver_phases(c, dt, c->stream);
    if (r == FS_OK) r = step_dispatch_any(c, true);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (r != FS_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        c->cur = key.cur;
        c->rho[0] = key.rho0;
        c->rho[1] = key.rho1;
        c->rho_prev = key.rho_prev;
        return r != FS_OK ? r : fail(FS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    fs_ctx::SolveGraph g = key;
    g.graph = graph;
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(FS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    g.launches = c->launches - launches0;
    g.post_cur = c->cur;
    g.post_rho0 = c->rho[0];
    g.post_rho1 = c->rho[1];
    g.post_rho_prev = c->rho_prev;
    c->solve_graphs.push_back(g);
    FS_CUDA(cudaGraphLaunch(g.exec, c->stream));
    return FS_OK;
}

// solver phases of a step on the lists of the last search
fs_status solve_after_search(fs_ctx* c, float dt, fs_step_stats* stats) {
    if (!c->have_lists) return fail(FS_ERR_STATE, "execute the neighborhood search first");
    const bool graphs = !(c->prm.flags & FS_FLAG_SYNC_EACH_ITERATION);
    if (graphs) {
        FS_TRY(solve_graph(c, dt));
    } else {
        FS_TRY(begin_solver_phases(c, dt, c->stream));
        FS_TRY(step_dispatch_any(c, false));
    }
    c->have_lists = false;  // positions moved: the lists belong to the old positions
    c->small_last = false;
    FS_TRY(read_scalars(c));
    int st = 0;
    FS_TRY(read_status(c, &st));
    for (int i = 0; i < 5; i++) cudaEventElapsedTime(&c->phase_ms[i], c->ev[i], c->ev[i + 1]);
    fill_stats(c, stats, st);
    if (st != FS_OK) return fail((fs_status)st, "device reported an error during the step");
    return FS_OK;
}

// Enqueues `steps` whole steps (search + solver) as CUDA-graph launches with
// no host synchronisation in between. The status word is cleared once: after
// a failure every later step skips its solver phases, leaving the state as
// the last successful step left it (up to the search's reordering).
// Whether whole steps of this context run in the small-scene kernel
// (fs_small.cuh): one scene of at most kSmallMax particles on the per-owner
// lists, with the dense cell grid.
bool small_eligible(const fs_ctx* c) {
    return (c->prm.flags & FS_FLAG_ONE_KERNEL_STEPS) && c->scenes == 0 && c->n > 0 && c->n <= kSmallMax && !tiled_mode(c) && !c->hash_table &&
           c->prm.solver != FS_SOLVER_NONE && !(c->prm.flags & FS_FLAG_SYNC_EACH_ITERATION) &&
           (int64_t)c->regions * (c->cells + 1) <= kSmallMaxTable;
}

template <typename R, bool KAHAN>
fs_status launch_small(fs_ctx* c, int32_t steps, float dt) {
    SmallStepArgs<R> a{};
    a.steps = steps;
    a.dim = c->dim;
    a.split = c->reference_order;
    a.fp32 = c->precision == FS_PRECISION_FP32;
    a.n = c->n;
    a.n_struct = c->n_struct;
    a.n_owners = c->n_owners;
    a.cur = c->cur;
    for (int b = 0; b < 2; b++)
        a.buf[b] = SmallBuffers{c->pos[b], c->vel[b], c->acc[b], c->ext[b], c->rho[b], c->p[b], c->type[b], c->hidx[b]};
    a.rho_prev = (R*)c->rho_prev;
    a.vstar = c->vstar;
    a.anp = c->anp;
    a.err = c->err;
    a.gbnd = c->gbnd;
    a.include_inactive = c->include_inactive;
    a.single_region = c->reference_order;
    a.trunc = c->truncate_cells;
    a.rows = !c->reference_order && c->dim == 3;
    a.sort_by_host = c->sort_lists_by_host;
    a.radius = c->search_radius;
    a.radius2 = c->radius2;
    a.key_bits = c->key_bits;
    a.regions = c->regions;
    a.cells = c->cells;
    a.grids = c->grids;
    a.bbox = c->bbox;
    for (int b = 0; b < 2; b++) {
        a.keys[b] = c->keys[b];
        a.keys64[b] = c->reference_order ? c->keys64[b] : nullptr;
        a.perm[b] = c->perm[b];
    }
    a.h2d_cell = c->h2d_cell;
    a.h2d_rank = c->h2d_rank;
    a.cell_start = c->cell_start;
    a.owner_mask = 1u << FS_TYPE_NORMAL;
    a.nbr = c->nbr;
    a.count = c->nbr_count;
    a.stride = c->nbr_stride;
    a.K = c->nbr_capacity;
    a.c = consts_of<R>(c);
    a.sc = c->scalars;
    a.status = c->status;
    a.desired_dt = dt;
    a.dynamic_generator = dynamic_timestep(c);
    a.particle_size = c->prm.particle_size;
    a.min_ts = c->prm.min_timestep;
    a.max_ts = c->prm.max_timestep;
    a.lambda_v = c->prm.lambda_v;
    a.lambda_a = c->prm.lambda_a;
    a.cfl_timestep = cfl_default(c);
    a.min_it = c->prm.min_iterations;
    a.max_it = c->prm.max_iterations;
    a.max_err = c->prm.max_density_error;
    a.stamps = c->small_stamps;
    cudaError_t e;
    switch (c->prm.solver) {
        case FS_SOLVER_IISPH_3D: e = launch_small_steps<R, KAHAN, kSmallIISPH3D>(a, c->stream, &c->small_blocks); break;
        case FS_SOLVER_IISPH_2D: e = launch_small_steps<R, KAHAN, kSmallIISPH2D>(a, c->stream, &c->small_blocks); break;
        default: e = launch_small_steps<R, KAHAN, kSmallSESPH>(a, c->stream, &c->small_blocks); break;
    }
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, std::string("small-scene steps: ") + cudaGetErrorString(e));
    c->launches++;
    // the buffer rotation the kernel applied, step by step: the search's
    // reordering, then (IISPH) the density double buffer
    const bool iisph = c->prm.solver == FS_SOLVER_IISPH_3D || c->prm.solver == FS_SOLVER_IISPH_2D;
    for (int32_t i = 0; i < steps; i++) {
        c->cur ^= 1;
        if (iisph) std::swap(c->rho[c->cur], c->rho_prev);
    }
    return FS_OK;
}

fs_status enqueue_small_steps(fs_ctx* c, int32_t steps, float dt) {
    if (c->precision == FS_PRECISION_FP64) return launch_small<double, false>(c, steps, dt);
    if (c->precision == FS_PRECISION_FP32) return launch_small<float, false>(c, steps, dt);
    return launch_small<float, true>(c, steps, dt);
}

fs_status enqueue_steps(fs_ctx* c, int32_t steps, float dt) {
    FS_CUDA(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    c->small_last = small_eligible(c);
    if (c->small_last) {
        if (steps > 0) FS_TRY(enqueue_small_steps(c, steps, dt));
    } else {
        for (int32_t i = 0; i < steps; i++) FS_TRY(solve_graph(c, dt, true));
    }
    c->have_lists = false;
    return FS_OK;
}

// the phase times of the last step (search, first loop, second loop,
// pressure iterations, integration): from the events of the step-by-step
// path or the small-scene kernel's timestamps
fs_status read_phase_times(fs_ctx* c) {
    if (!c->small_last) {
        for (int i = 0; i < 5; i++) cudaEventElapsedTime(&c->phase_ms[i], c->ev[i], c->ev[i + 1]);
        return FS_OK;
    }
    unsigned long long t[6];
    FS_CUDA(cudaMemcpy(t, c->small_stamps, sizeof(t), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 5; i++) c->phase_ms[i] = t[i + 1] >= t[i] ? (float)((double)(t[i + 1] - t[i]) * 1e-6) : 0.f;
    return FS_OK;
}

fs_status finish_steps(fs_ctx* c, fs_step_stats* stats, int* st) {
    FS_TRY(read_scalars(c));
    FS_TRY(read_status(c, st));
    FS_TRY(read_phase_times(c));
    fill_stats(c, stats, *st);
    return FS_OK;
}

fs_status one_step(fs_ctx* c, float desired_dt, fs_step_stats* stats) {
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->prm.solver == FS_SOLVER_NONE) return fail(FS_ERR_INVALID, "context has no solver");
    const float dt = desired_of(c, desired_dt);
    if (!(c->prm.flags & FS_FLAG_SYNC_EACH_ITERATION)) {
        FS_TRY(enqueue_steps(c, 1, dt));
        int st = 0;
        FS_TRY(finish_steps(c, stats, &st));
        if (st == FS_OK) return FS_OK;
        if (st != FS_ERR_CAPACITY || c->prm.neighbor_capacity != 0)
            return fail((fs_status)st, "device reported an error during the step");
        // the lists overflowed: the solver phases did not run; grow and redo
        int K = 32;
        while (K < c->scalars_host->max_neighbors) K *= 2;
        FS_TRY(ensure_lists(c, K));
    }
    FS_TRY(search_for_step(c, dt));
    return solve_after_search(c, dt, stats);
}

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

int32_t fs_abi_version(void) { return FS_ABI_VERSION; }

const char* fs_last_error(void) { return g_error.c_str(); }

void fs_params_default(fs_params* p, int32_t dim, int32_t solver, int32_t search) {
    std::memset(p, 0, sizeof(*p));
    p->dim = dim;
    p->solver = solver;
    p->search = search;
    p->precision = FS_PRECISION_FP32_KAHAN;
    p->rest_density = 1000.0f;   // IFluidSolver.hpp:19-21
    p->gravity = 9.81f;
    p->particle_size = 0.1f;
    p->stiffness = 100000.0f;    // SESPHSettings*.hpp
    p->viscosity = 5.0f;
    p->single_layer_boundary = 0;
    p->single_layer_gamma_1 = 1.1f;
    p->single_layer_gamma_2 = 1.1f;
    p->max_density_error = 0.001f;  // IISPHSettings*.hpp
    p->min_iterations = 2;
    p->max_iterations = 100;
    p->omega = 0.5f;
    p->gamma = 0.7f;
    p->timestep = 0.001f;        // ConstantTimestepGenerator.hpp:8-13
    p->lambda_v = 0.4f;
    p->lambda_a = 0.25f;
    p->timestep_generator = FS_TIMESTEP_CONSTANT;
    p->min_timestep = 0.0001f;   // DynamicCflTimestepGenerator.hpp:11-18
    p->max_timestep = 0.02f;
    p->max_particles = 0;
    p->neighbor_capacity = 0;
    p->device = 0;
}

// a context for one scene (scenes == 0) or for `scenes` batched scenes whose
// host particles are [offsets[s], offsets[s + 1])
static fs_status create_ctx(const fs_params* p, int32_t scenes, const int64_t* offsets, fs_ctx** out) {
    if (!out) return fail(FS_ERR_INVALID, "out is null");
    *out = nullptr;
    FS_TRY(check_params(p));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FS_ERR_NO_DEVICE, "no CUDA device");
    if (p->device < 0 || p->device >= ndev) return fail(FS_ERR_INVALID, "device ordinal out of range");
    FS_CUDA(cudaSetDevice(p->device));
    cudaDeviceProp prop;
    FS_CUDA(cudaGetDeviceProperties(&prop, p->device));
    if (prop.major < 10) return fail(FS_ERR_NO_DEVICE, "device is not sm_100 class");
    fs_ctx* c = new (std::nothrow) fs_ctx();
    if (!c) return fail(FS_ERR_INVALID, "out of host memory");
    c->prm = *p;
    c->device = p->device;
    derive(c);
    c->cap = p->max_particles;
    if (scenes > 0) {
        c->scenes = scenes;
        c->scene_offsets.assign(offsets, offsets + scenes + 1);
        c->cap = std::max<int64_t>(c->cap, offsets[scenes]);
    }
    auto bail = [&](fs_status s) {
        free_all(c);
        delete c;
        return s;
    };
#define FS_ALLOC(ptr, count)                      \
    do {                                          \
        fs_status s_ = dalloc(&(ptr), (count));   \
        if (s_ != FS_OK) return bail(s_);         \
    } while (0)
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(FS_ERR_CUDA, "cudaStreamCreate failed"));
    const size_t cap = (size_t)c->cap;
    const size_t v4 = c->real_size * 4, r1 = c->real_size;
    // scalar fields that the tile passes stage: readable up to a multiple of 4 entries
    const size_t cap4 = (cap + 3) & ~(size_t)3;
    for (int b = 0; b < 2; b++) {
        char** fields[] = {(char**)&c->pos[b], (char**)&c->vel[b], (char**)&c->acc[b], (char**)&c->ext[b]};
        for (char** f : fields) FS_ALLOC(*f, cap * v4);
        FS_ALLOC(*(char**)&c->rho[b], cap4 * r1);
        FS_ALLOC(*(char**)&c->p[b], cap4 * r1);
        FS_ALLOC(c->type[b], cap);
        FS_ALLOC(c->hidx[b], cap);
        FS_ALLOC(c->keys[b], cap);
        FS_ALLOC(c->perm[b], cap);
        if (c->reference_order || p->search == FS_SEARCH_COMPACT_2D) FS_ALLOC(c->keys64[b], cap);
    }
    if (p->search == FS_SEARCH_COMPACT_2D) {
        uint32_t slots = 64;
        while ((uint64_t)slots < 2 * (uint64_t)cap) slots <<= 1;
        FS_ALLOC(c->hash_table, slots);
        c->hash_mask = slots - 1;
    }
    if (c->truncate_cells) {
        FS_ALLOC(c->h2d_cell, cap);
        FS_ALLOC(c->h2d_rank, cap);
    }
    FS_ALLOC(*(char**)&c->rho_prev, cap4 * r1);
    FS_ALLOC(*(char**)&c->vstar, cap * v4);
    FS_ALLOC(*(char**)&c->anp, cap * v4);
    FS_ALLOC(*(char**)&c->err, cap * r1);
    FS_ALLOC(*(char**)&c->gbnd, cap * v4);
    const int S = c->nsc();
    FS_ALLOC(c->bbox, 6 * S);
    FS_ALLOC(c->grids, S);
    FS_ALLOC(c->status, 1);
    FS_ALLOC(c->small_stamps, 8);
    FS_ALLOC(c->scalars, S);
    if (scenes > 0) {
        FS_ALLOC(c->scene_of[0], cap);
        FS_ALLOC(c->scene_of[1], cap);
        FS_ALLOC(c->d_scene_offsets, scenes + 1);
        if (cudaMemcpy(c->d_scene_offsets, offsets, sizeof(int64_t) * (scenes + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess)
            return bail(fail(FS_ERR_CUDA, "copy of the scene offsets failed"));
    }
    FS_ALLOC(c->nbr_count, (cap + kTileOwners - 1) / kTileOwners * kTileOwners);   // whole tiles
    if (cudaMallocHost((void**)&c->scalars_host, sizeof(StepScalars) * S) != cudaSuccess)
        return bail(fail(FS_ERR_CUDA, "cudaMallocHost failed"));
    // the radix sort's per-tile digit counts for the largest sort
    FS_ALLOC(c->sort_hist, (size_t)sort_hist_entries((int64_t)cap));
    if (prepare_small_sort() != cudaSuccess) return bail(fail(FS_ERR_CUDA, "small-sort shared memory"));
    int K = p->neighbor_capacity > 0 ? p->neighbor_capacity : (p->dim == 2 ? 32 : 64);
    if (contract_capacity(p->search) > 0) K = std::min(K, contract_capacity(p->search) + 1);
    {
        fs_status s_ = ensure_lists(c, K);
        if (s_ != FS_OK) return bail(s_);
    }
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(FS_ERR_CUDA, "cudaEventCreate failed"));
    if (cudaMemsetAsync(c->status, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return bail(fail(FS_ERR_CUDA, "initialisation failed"));
#undef FS_ALLOC
    *out = c;
    return FS_OK;
}

fs_status fs_create(const fs_params* p, fs_ctx** out) { return create_ctx(p, 0, nullptr, out); }

fs_status fs_destroy(fs_ctx* c) {
    if (!c) return FS_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return FS_OK;
}

fs_status fs_set_params(fs_ctx* c, const fs_params* p) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    FS_TRY(check_params(p));
    if (p->dim != c->prm.dim || p->solver != c->prm.solver || p->search != c->prm.search ||
        p->precision != c->prm.precision || p->flags != c->prm.flags || p->max_particles != c->prm.max_particles)
        return fail(FS_ERR_INVALID, "layout-defining parameters cannot change; create a new context");
    if (std::memcmp(&c->prm, p, sizeof(fs_params)) == 0) return FS_OK;
    FS_CUDA(cudaSetDevice(c->device));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    clear_graphs(c);
    c->prm = *p;
    derive(c);
    return FS_OK;
}

fs_status fs_upload(fs_ctx* c, const fs_particles* in) {
    if (!c || !in) return fail(FS_ERR_INVALID, "null argument");
    if (in->n < 0 || in->n > c->cap) return fail(FS_ERR_INVALID, "particle count exceeds the context capacity");
    if (in->n > 0 && !in->position) return fail(FS_ERR_INVALID, "position is required for upload");
    if (c->scenes > 0 && in->n != c->scene_offsets[c->scenes])
        return fail(FS_ERR_INVALID, "a batched upload holds exactly the particles of every scene");
    FS_CUDA(cudaSetDevice(c->device));
    StagedUpload d;
    UploadCensus h;
    std::vector<int> boxes;
    FS_TRY(stage_upload(c, in, d, h, boxes));
    if (h.counts[3]) return fail(FS_ERR_INVALID, "particle type must be 0, 1 or 2");
    const int64_t n_before = c->n, owners_before = c->n_owners;
    set_layout(c, in->n, (int64_t)h.counts[0], (int64_t)h.counts[1], (int64_t)h.counts[2]);
    if (c->n != n_before || c->n_owners != owners_before) clear_graphs(c);
    FS_TRY(choose_grids(c, boxes.data(), boxes.data() + 3 * c->nsc()));
    FS_TRY(ensure_cells(c));
    fs_status r = c->precision == FS_PRECISION_FP64 ? pack_upload<double>(c, d, in->n) : pack_upload<float>(c, d, in->n);
    if (r != FS_OK) return r;
    // The 2D hashed grid's history lives as long as the context, like the
    // reference's search object, whose grid survives changes of the
    // collection's contents; a different particle count starts it afresh.
    if (c->h2d_rank && c->h2d_n != in->n) {
        FS_CUDA(cudaMemsetAsync(c->h2d_rank, 0xff, sizeof(uint32_t) * (size_t)c->cap, c->stream));
        c->h2d_n = in->n;
    }
    c->have_state = true;
    c->have_lists = false;
    c->have_cells = false;
    return FS_OK;
}

fs_status fs_download(fs_ctx* c, fs_particles* out) {
    if (!c || !out) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    FS_CUDA(cudaSetDevice(c->device));
    if (c->precision == FS_PRECISION_FP64) return download_impl<double>(c, out);
    return download_impl<float>(c, out);
}

fs_status fs_find_neighbors(fs_ctx* c) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    FS_CUDA(cudaSetDevice(c->device));
    FS_TRY(search_for_step(c, c->prm.timestep));
    cudaEventRecord(c->ev[1], c->stream);
    FS_CUDA(cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->phase_ms[0], c->ev[0], c->ev[1]);
    return FS_OK;
}

fs_status fs_solve_step(fs_ctx* c, float desired_dt, fs_step_stats* stats) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->prm.solver == FS_SOLVER_NONE) return fail(FS_ERR_INVALID, "context has no solver");
    FS_CUDA(cudaSetDevice(c->device));
    const float dt = desired_of(c, desired_dt);
    return solve_after_search(c, dt, stats);
}

fs_status fs_get_neighbors_csr(fs_ctx* c, int64_t* offsets, int64_t* indices, int64_t* total) {
    if (!c || !offsets) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    FS_CUDA(cudaSetDevice(c->device));
    const int64_t n = c->n;
    const int64_t ns = c->n_struct;
    cudaStream_t st = c->stream;
    if (n == 0) {
        offsets[0] = 0;
        if (total) *total = 0;
        return FS_OK;
    }
    if (c->csr_capacity < n + 1) {
        if (c->csr_offsets) cudaFree(c->csr_offsets);
        if (c->csr_counts) cudaFree(c->csr_counts);
        c->csr_offsets = nullptr;
        c->csr_counts = nullptr;
        FS_TRY(dalloc(&c->csr_offsets, (size_t)n + 1));
        FS_TRY(dalloc(&c->csr_counts, (size_t)n + 1));
        c->csr_capacity = n + 1;
    }
    WalkParams w = walk_of(c, false);
    const uint32_t mask = contract_owner_mask(c->prm.search);
    FS_CUDA(cudaMemsetAsync(c->csr_counts, 0, sizeof(uint32_t) * (n + 1), st));
    if (c->precision == FS_PRECISION_FP64) {
        State<double> s = state_of<double>(c);
    c->launches++;
        k_csr_count<double><<<grid_for(ns), kBlock, 0, st>>>(ns, s.pos, s.type, c->cell_start, w, mask,
                                                             c->csr_counts);
    } else {
        State<float> s = state_of<float>(c);
    c->launches++;
        k_csr_count<float><<<grid_for(ns), kBlock, 0, st>>>(ns, s.pos, s.type, c->cell_start, w, mask,
                                                            c->csr_counts);
    }
    FS_CUDA(cudaGetLastError());
    c->launches++;
    k_scan_exclusive<uint32_t, int64_t><<<1, 1024, 0, st>>>(c->csr_counts, c->csr_offsets, n + 1);
    FS_CUDA(cudaGetLastError());
    int64_t tot = 0;
    FS_CUDA(cudaMemcpyAsync(&tot, c->csr_offsets + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    FS_CUDA(cudaStreamSynchronize(st));
    if (total) *total = tot;
    // per-list capacity of the contract (the reference throws beyond it)
    const int cap = contract_capacity(c->prm.search);
    std::vector<uint32_t> counts((size_t)n);
    FS_CUDA(cudaMemcpy(counts.data(), c->csr_counts, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> hidx((size_t)n);
    FS_CUDA(cudaMemcpy(hidx.data(), c->hidx[c->cur], sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    bool over = false;
    std::vector<int64_t> cnt_host((size_t)n, 0);
    for (int64_t k = 0; k < n; k++) {
        cnt_host[hidx[k]] = counts[k];
        if (cap > 0 && (int64_t)counts[k] > cap) over = true;
    }
    offsets[0] = 0;
    for (int64_t h = 0; h < n; h++) offsets[h + 1] = offsets[h] + cnt_host[h];
    if (over) {
        g_error = "a neighbor list exceeds the contract's capacity";
        if (!indices) return FS_ERR_CAPACITY;
    }
    if (!indices) return over ? FS_ERR_CAPACITY : FS_OK;
    uint32_t* d_idx = nullptr;
    FS_TRY(dalloc(&d_idx, (size_t)std::max<int64_t>(tot, 1)));
    if (c->precision == FS_PRECISION_FP64) {
        State<double> s = state_of<double>(c);
    c->launches++;
        k_csr_fill<double><<<grid_for(ns), kBlock, 0, st>>>(ns, s.pos, s.type, c->cell_start, w, mask,
                                                            c->csr_offsets, d_idx);
    } else {
        State<float> s = state_of<float>(c);
    c->launches++;
        k_csr_fill<float><<<grid_for(ns), kBlock, 0, st>>>(ns, s.pos, s.type, c->cell_start, w, mask,
                                                           c->csr_offsets, d_idx);
    }
    std::vector<uint32_t> idx((size_t)tot);
    std::vector<int64_t> off_sorted((size_t)n + 1);
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaMemcpyAsync(idx.data(), d_idx, sizeof(uint32_t) * tot, cudaMemcpyDeviceToHost, st);
    cudaError_t e3 = cudaMemcpyAsync(off_sorted.data(), c->csr_offsets, sizeof(int64_t) * (n + 1),
                                     cudaMemcpyDeviceToHost, st);
    cudaError_t e4 = cudaStreamSynchronize(st);
    cudaFree(d_idx);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess)
        return fail(FS_ERR_CUDA, "CSR export failed");
    for (int64_t k = 0; k < n; k++) {
        const int64_t h = hidx[k];
        int64_t o = offsets[h];
        for (int64_t q = off_sorted[k]; q < off_sorted[k + 1]; q++) indices[o++] = hidx[idx[q]];
        std::sort(indices + offsets[h], indices + offsets[h + 1]);
    }
    return over ? FS_ERR_CAPACITY : FS_OK;
}

fs_status fs_get_solver_lists_csr(fs_ctx* c, int64_t* offsets, int64_t* indices, int64_t* total) {
    if (!c || !offsets) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (!c->have_lists) return fail(FS_ERR_STATE, "no solver lists: execute the neighborhood search first");
    FS_CUDA(cudaSetDevice(c->device));
    const int64_t n = c->n, no = c->n_owners;
    cudaStream_t st = c->stream;
    const bool tiled = tiled_mode(c) && no > 0;
    std::vector<uint32_t> counts((size_t)std::max<int64_t>(no, 1), 0);
    std::vector<int64_t> off_sorted((size_t)no + 1, 0);
    uint32_t* d_counts = nullptr;
    int64_t* d_off = nullptr;
    uint32_t* d_idx = nullptr;
    auto release = [&] {
        if (d_counts) cudaFree(d_counts);
        if (d_off) cudaFree(d_off);
        if (d_idx) cudaFree(d_idx);
    };
    if (no > 0) {
        if (dalloc(&d_counts, (size_t)no) != FS_OK || dalloc(&d_off, (size_t)no + 1) != FS_OK) {
            release();
            return fail(FS_ERR_CUDA, "allocation for the list export failed");
        }
        c->launches++;
        k_export_solver_lists<<<grid_for(no), kBlock, 0, st>>>(no, tiled, tile_lists_of(c), lists_of(c), nullptr,
                                                               d_counts, nullptr);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(counts.data(), d_counts, sizeof(uint32_t) * no, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            release();
            return fail(FS_ERR_CUDA, "list export failed");
        }
        for (int64_t k = 0; k < no; k++) off_sorted[k + 1] = off_sorted[k] + counts[k];
    }
    std::vector<uint32_t> hidx((size_t)std::max<int64_t>(n, 1));
    if (n > 0 && cudaMemcpy(hidx.data(), c->hidx[c->cur], sizeof(uint32_t) * n, cudaMemcpyDeviceToHost) !=
                     cudaSuccess) {
        release();
        return fail(FS_ERR_CUDA, "list export failed");
    }
    std::vector<int64_t> cnt_host((size_t)n + 1, 0);
    for (int64_t k = 0; k < no; k++) cnt_host[hidx[k]] = counts[k];
    offsets[0] = 0;
    for (int64_t h = 0; h < n; h++) offsets[h + 1] = offsets[h] + cnt_host[h];
    const int64_t tot = off_sorted[no];
    if (total) *total = tot;
    if (!indices || tot == 0) {
        release();
        return FS_OK;
    }
    std::vector<uint32_t> idx((size_t)tot);
    if (dalloc(&d_idx, (size_t)tot) != FS_OK ||
        cudaMemcpyAsync(d_off, off_sorted.data(), sizeof(int64_t) * (no + 1), cudaMemcpyHostToDevice, st) !=
            cudaSuccess) {
        release();
        return fail(FS_ERR_CUDA, "list export failed");
    }
    c->launches++;
    k_export_solver_lists<<<grid_for(no), kBlock, 0, st>>>(no, tiled, tile_lists_of(c), lists_of(c), d_off, nullptr,
                                                           d_idx);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(idx.data(), d_idx, sizeof(uint32_t) * tot, cudaMemcpyDeviceToHost, st) ==
                        cudaSuccess &&
                    cudaStreamSynchronize(st) == cudaSuccess;
    release();
    if (!ok) return fail(FS_ERR_CUDA, "list export failed");
    for (int64_t k = 0; k < no; k++) {
        const int64_t h = hidx[k];
        int64_t o = offsets[h];
        for (int64_t q = off_sorted[k]; q < off_sorted[k + 1]; q++) {
            if (idx[q] >= (uint32_t)n) {
                // report the entry and its tile's ranges
                std::string msg = "solver list entry " + std::to_string(q - off_sorted[k]) + " of sorted owner " +
                                  std::to_string(k) + " (of " + std::to_string(counts[k]) + ") maps to no particle";
                if (tiled && (idx[q] >> 28) == 0xfu) {
                    TileDesc dd;
                    if (cudaMemcpy(&dd, c->tile_desc + k / kTileOwners, sizeof(dd), cudaMemcpyDeviceToHost) ==
                        cudaSuccess) {
                        msg += ": slot " + std::to_string(idx[q] & 0xffffu) + ", tile " +
                               std::to_string(k / kTileOwners) + " with " + std::to_string(dd.h.nranges) +
                               " ranges, " + std::to_string(dd.h.staged & 0xffffu) + " staged:";
                        for (uint32_t r = 0; r < dd.h.nranges && r < (uint32_t)kTileRanges; r++)
                            msg += " [" + std::to_string(dd.start[r]) + "+" +
                                   std::to_string(dd.len_base[r] & kRangeLen) + "@" +
                                   std::to_string(dd.len_base[r] >> 16) + "]";
                    }
                }
                return fail(FS_ERR_CUDA, msg);
            }
            indices[o++] = hidx[idx[q]];
        }
        std::sort(indices + offsets[h], indices + offsets[h + 1]);
    }
    return FS_OK;
}

fs_status fs_boundary_preprocess(fs_ctx* c) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->dim != 3) return fail(FS_ERR_INVALID, "the boundary preprocessor needs 3D particles (MovementData3D)");
    if (c->scenes > 0) return fail(FS_ERR_INVALID, "not available on batched contexts");
    // the neighbor sets of the current positions: a search since the last step
    if (c->prm.solver != FS_SOLVER_NONE ? !c->have_lists : !c->have_cells)
        return fail(FS_ERR_STATE, "execute the neighborhood search first");
    FS_CUDA(cudaSetDevice(c->device));
    if (c->n == 0) return FS_OK;
    const WalkParams w = walk_of(c, false);
    c->launches++;
    if (c->precision == FS_PRECISION_FP64) {
        const SolverConsts<double> k = consts_of<double>(c);
        k_boundary_mass<double><<<grid_for(c->n), kBlock, 0, c->stream>>>(
            c->n, state_of<double>(c), c->cell_start, w, k.kern, (double)c->prm.rest_density,
            (double)c->prm.particle_size);
    } else {
        const SolverConsts<float> k = consts_of<float>(c);
        k_boundary_mass<float><<<grid_for(c->n), kBlock, 0, c->stream>>>(
            c->n, state_of<float>(c), c->cell_start, w, k.kern, c->prm.rest_density, c->prm.particle_size);
    }
    FS_CUDA(cudaGetLastError());
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

static_assert(sizeof(StatsOut) == sizeof(fs_global_stats), "StatsOut mirrors fs_global_stats");

fs_status fs_global_statistics(fs_ctx* c, float zero_height, fs_global_stats* out) {
    if (!c || !out) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    FS_CUDA(cudaSetDevice(c->device));
    if (!c->stats_parts) {
        FS_TRY(dalloc(&c->stats_parts, (size_t)kStatsBlocks));
        FS_TRY(dalloc(&c->stats_out, (size_t)1));
    }
    const int blocks = (int)std::min<int64_t>(kStatsBlocks, std::max<int64_t>(1, (c->n + kStatsThreads - 1) / kStatsThreads));
    c->launches += 2;
    if (c->precision == FS_PRECISION_FP64)
        k_stats_partial<double><<<blocks, kStatsThreads, 0, c->stream>>>(c->n, state_of<double>(c), c->prm.gravity,
                                                                          zero_height, c->stats_parts);
    else
        k_stats_partial<float><<<blocks, kStatsThreads, 0, c->stream>>>(c->n, state_of<float>(c), c->prm.gravity,
                                                                         zero_height, c->stats_parts);
    k_stats_finish<<<1, kStatsThreads, 0, c->stream>>>(c->stats_parts, blocks, c->stats_out);
    FS_CUDA(cudaGetLastError());
    FS_CUDA(cudaMemcpyAsync(out, c->stats_out, sizeof(fs_global_stats), cudaMemcpyDeviceToHost, c->stream));
    FS_CUDA(cudaStreamSynchronize(c->stream));
    return FS_OK;
}

fs_status fs_particles_file_info(const char* path, int32_t* dim, int64_t* n, uint32_t* components) {
    if (!path) return fail(FS_ERR_INVALID, "path is null");
    fsio::ParticleFile f;
    const std::string e = fsio::read_particle_file(path, f);
    if (!e.empty()) return fail(FS_ERR_INVALID, e);
    if (dim) *dim = f.dim;
    if (n) *n = (int64_t)f.n;
    if (components) *components = f.components;
    return FS_OK;
}

fs_status fs_particles_file_read(const char* path, fs_particles* out) {
    if (!path || !out) return fail(FS_ERR_INVALID, "null argument");
    fsio::ParticleFile f;
    const std::string e = fsio::read_particle_file(path, f);
    if (!e.empty()) return fail(FS_ERR_INVALID, e);
    if (out->n != (int64_t)f.n)
        return fail(FS_ERR_INVALID, "out->n is " + std::to_string(out->n) + ", the file holds " + std::to_string(f.n));
    const size_t n = (size_t)f.n, d = (size_t)f.dim;
    auto copy = [&](float* dst, const std::vector<float>& src, size_t per) {
        if (!dst) return;
        if (src.empty()) std::memset(dst, 0, sizeof(float) * n * per);
        else std::memcpy(dst, src.data(), sizeof(float) * n * per);
    };
    copy(out->position, f.position, d);
    copy(out->velocity, f.velocity, d);
    copy(out->acceleration, f.acceleration, d);
    copy(out->external, f.external, d);
    copy(out->mass, f.mass, 1);
    copy(out->density, f.density, 1);
    copy(out->pressure, f.pressure, 1);
    if (out->type) {
        if (f.type.empty()) std::memset(out->type, 0, n);
        else std::memcpy(out->type, f.type.data(), n);
    }
    if (out->tag)
        for (size_t i = 0; i < n; i++) out->tag[i] = f.tag.empty() ? (uint32_t)i : f.tag[i];
    return FS_OK;
}

fs_status fs_particles_file_write(const char* path, int32_t dim, const fs_particles* in) {
    if (!path || !in) return fail(FS_ERR_INVALID, "null argument");
    if (dim != 2 && dim != 3) return fail(FS_ERR_INVALID, "dim must be 2 or 3");
    if (in->n < 0) return fail(FS_ERR_INVALID, "negative particle count");
    fsio::ParticleFile f;
    f.dim = dim;
    f.n = (uint64_t)in->n;
    const size_t n = (size_t)in->n;
    auto take = [&](std::vector<float>& dst, const float* src, size_t per) {
        if (src) dst.assign(src, src + n * per);
    };
    take(f.position, in->position, dim);
    if (in->position) {
        f.velocity.assign(n * dim, 0.0f);
        f.acceleration.assign(n * dim, 0.0f);
        take(f.velocity, in->velocity, dim);
        take(f.acceleration, in->acceleration, dim);
    }
    take(f.external, in->external, dim);
    if (in->mass || in->density || in->pressure) {
        f.mass.assign(n, 0.0f);
        f.density.assign(n, 0.0f);
        f.pressure.assign(n, 0.0f);
        take(f.mass, in->mass, 1);
        take(f.density, in->density, 1);
        take(f.pressure, in->pressure, 1);
    }
    if (in->type || in->tag) {
        f.type.assign(n, 0);
        f.tag.resize(n);
        for (size_t i = 0; i < n; i++) {
            f.type[i] = in->type ? in->type[i] : (uint8_t)FS_TYPE_NORMAL;
            f.tag[i] = in->tag ? in->tag[i] : (uint32_t)i;
        }
    }
    const std::string e = fsio::write_particle_file(path, f);
    if (!e.empty()) return fail(FS_ERR_INVALID, e);
    return FS_OK;
}

fs_status fs_dump(fs_ctx* c, const char* path) {
    if (!c || !path) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    const size_t n = (size_t)c->n, d = (size_t)c->dim;
    std::vector<float> pos(n * d), vel(n * d), acc(n * d), ext(n * d), mass(n), rho(n), p(n);
    std::vector<uint8_t> type(n);
    std::vector<uint32_t> tag(n);
    fs_particles v{};
    v.n = (int64_t)n;
    v.position = pos.data();
    v.velocity = vel.data();
    v.acceleration = acc.data();
    v.external = ext.data();
    v.mass = mass.data();
    v.density = rho.data();
    v.pressure = p.data();
    v.type = type.data();
    v.tag = tag.data();
    FS_TRY(fs_download(c, &v));
    return fs_particles_file_write(path, c->dim, &v);
}

fs_status fs_query_position(fs_ctx* c, const float* position, int64_t* out, int64_t cap, int64_t* count) {
    if (!c || !position) return fail(FS_ERR_INVALID, "null argument");
    if (cap > 0 && !out) return fail(FS_ERR_INVALID, "out is null");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->scenes > 0) return fail(FS_ERR_INVALID, "a position query names no scene: not available on batched contexts");
    const int search = c->prm.search;
    if (search == FS_SEARCH_COMPACT_2D)
        return fail(FS_ERR_INVALID, "the compact-hashing contract has no position query (it throws \"Not implemented\")");
    // the quadratic contracts test every particle; the others walk the cells
    // of the last search (stale cells, current positions, as the reference)
    const bool all = search == FS_SEARCH_QUADRATIC_2D || search == FS_SEARCH_QUADRATIC_3D;
    if (!all && !c->have_cells) return fail(FS_ERR_STATE, "position queries need a neighborhood search after the upload");
    if (count) *count = 0;
    if (c->n == 0) return FS_OK;
    FS_CUDA(cudaSetDevice(c->device));
    WalkParams w = walk_of(c, false);
    w.length_test = search != FS_SEARCH_COMPRESSED_3D;
    const bool skip = search == FS_SEARCH_HASHED_3D;
    uint32_t* d_out = nullptr;
    unsigned long long* d_cnt = nullptr;
    const int64_t room = std::max<int64_t>(cap, 0);
    FS_TRY(dalloc(&d_out, (size_t)std::max<int64_t>(room, 1)));
    if (dalloc(&d_cnt, 1) != FS_OK) {
        cudaFree(d_out);
        return FS_ERR_CUDA;
    }
    cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), c->stream);
    const float z = c->dim == 3 ? position[2] : 0.0f;
    const int gq = (int)std::min<int64_t>((c->n + kBlock - 1) / kBlock, 1184);
    if (c->precision == FS_PRECISION_FP64) {
        State<double> s = state_of<double>(c);
        const V3<double> x = v3<double>(position[0], position[1], z);
        c->launches++;
        if (all) k_query_all<double><<<gq, kBlock, 0, c->stream>>>(x, c->n, s.pos, w, d_out, room, d_cnt);
        else k_query_position<double><<<1, 32, 0, c->stream>>>(x, s.pos, s.type, s.hidx, c->cell_start, w,
                                                               skip, d_out, room, d_cnt);
    } else {
        State<float> s = state_of<float>(c);
        const V3<float> x = v3<float>(position[0], position[1], z);
        c->launches++;
        if (all) k_query_all<float><<<gq, kBlock, 0, c->stream>>>(x, c->n, s.pos, w, d_out, room, d_cnt);
        else k_query_position<float><<<1, 32, 0, c->stream>>>(x, s.pos, s.type, s.hidx, c->cell_start, w,
                                                              skip, d_out, room, d_cnt);
    }
    cudaError_t e = cudaGetLastError();
    unsigned long long cnt = 0;
    std::vector<uint32_t> tmp((size_t)room);
    std::vector<uint32_t> hidx((size_t)c->n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && room)
        e = cudaMemcpyAsync(tmp.data(), d_out, sizeof(uint32_t) * room, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hidx.data(), c->hidx[c->cur], sizeof(uint32_t) * c->n, cudaMemcpyDeviceToHost, c->stream);
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    cudaFree(d_out);
    cudaFree(d_cnt);
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(FS_ERR_CUDA, cudaGetErrorString(e2));
    const int64_t m = std::min<int64_t>((int64_t)cnt, room);
    for (int64_t q = 0; q < m; q++) out[q] = hidx[tmp[q]];
    std::sort(out, out + m);
    if (count) *count = (int64_t)cnt;
    return FS_OK;
}

fs_status fs_step(fs_ctx* c, float desired_dt, fs_step_stats* stats) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    FS_CUDA(cudaSetDevice(c->device));
    return one_step(c, desired_dt, stats);
}

fs_status fs_run(fs_ctx* c, int32_t steps, float desired_dt, fs_step_stats* stats) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    if (steps < 0) return fail(FS_ERR_INVALID, "steps must be >= 0");
    FS_CUDA(cudaSetDevice(c->device));
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->prm.solver == FS_SOLVER_NONE) return fail(FS_ERR_INVALID, "context has no solver");
    if (steps == 0) return FS_OK;
    if (c->prm.flags & FS_FLAG_SYNC_EACH_ITERATION) {
        for (int32_t i = 0; i < steps; i++) FS_TRY(one_step(c, desired_dt, stats));
        return FS_OK;
    }
    // one step first: it settles the list capacity (and captures the graph)
    FS_TRY(one_step(c, desired_dt, stats));
    const float dt = desired_of(c, desired_dt);
    FS_TRY(enqueue_steps(c, steps - 1, dt));
    int st = 0;
    FS_TRY(finish_steps(c, stats, &st));
    if (st != FS_OK) return fail((fs_status)st, "device reported an error during fs_run");
    return FS_OK;
}

// mean whole-step time of `steps` steps after `warm` (graphs re-captured);
// the step is the sum of the five phase times the events measure
static fs_status time_steps(fs_ctx* t, int warm, int steps, double& step_ms, double& l1_ms, double& iter_ms,
                            int& iter_samples) {
    fs_step_stats st{};
    clear_graphs(t);
    for (int i = 0; i < warm; i++) FS_TRY(one_step(t, 0.0f, &st));
    step_ms = l1_ms = iter_ms = 0.0;
    iter_samples = 0;
    for (int i = 0; i < steps; i++) {
        FS_TRY(one_step(t, 0.0f, &st));
        double sum = 0.0;
        for (int q = 0; q < 5; q++) sum += t->phase_ms[q];
        step_ms += sum / steps;
        l1_ms += t->phase_ms[1] / steps;
        if (st.iterations > 1) {
            iter_ms += t->phase_ms[3] / (st.iterations - 1);
            iter_samples++;
        }
    }
    if (iter_samples) iter_ms /= iter_samples;
    return FS_OK;
}

// fraction of the tiles of the last search that fell back to 32-bit lists
static fs_status fallback_fraction(fs_ctx* t, float& frac) {
    const int64_t tiles = (t->n_owners + kTileOwners - 1) / kTileOwners;
    frac = 0.f;
    if (tiles == 0) return FS_OK;
    std::vector<TileDesc> d((size_t)tiles);
    FS_CUDA(cudaMemcpy(d.data(), t->tile_desc, sizeof(TileDesc) * tiles, cudaMemcpyDeviceToHost));
    int64_t fb = 0;
    for (const TileDesc& x : d) fb += x.h.nranges == kTileFallback ? 1 : 0;
    frac = (float)fb / (float)tiles;
    return FS_OK;
}

// The fast mode's launch shapes, chosen by timing whole steps on a copy of
// the context: the same parameters and the same particles (downloaded from
// the context, uploaded into the copy before every trial), so the caller's
// state and step count stay as they were. A coordinate search, one axis
// after the other, each trial 2 steps to capture its graph and settle, then
// 4 timed steps:
//   1. prefetch depths, trials (pressure, first loop) (1,1), (2,2), (3,1),
//      (4,2); the first loop is rated by its phase time, the pressure passes
//      per loop iteration (the first iteration runs inside the second loop),
//      each depth by the mean over the trials that used it;
//   2. the staging cap per tile, 1024 / 1536 / 2048 / 3072, by whole steps;
//   3. the per-particle kernels' block size, 128 / 256 / 512, by whole steps.
fs_status fs_autotune(fs_ctx* c, fs_tuning* out) {
    if (!c || !out) return fail(FS_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (c->scenes > 0)
        return fail(FS_ERR_INVALID, "tune a single-scene context and hand its result to fs_set_tuning");
    *out = fs_tuning{};
    out->first_loop_prefetch = c->tuning.l1_ahead;
    out->pressure_prefetch = c->tuning.pressure_ahead;
    out->tile_cap = c->tuning.cap;
    out->block_size = c->tuning.block;
    out->pressure_threads_per_owner = c->tuning.pressure_tpo;
    // nothing tunable unless the IISPH passes are tiled
    if (!tiled_mode(c) || c->prm.solver != FS_SOLVER_IISPH_3D || c->n_fluid == 0) return FS_OK;
    FS_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)c->n, d = (size_t)c->dim;
    std::vector<float> pos(n * d), vel(n * d), acc(n * d), ext(n * d), mass(n), rho(n), p(n);
    std::vector<uint8_t> type(n);
    std::vector<uint32_t> tag(n);
    fs_particles v{};
    v.n = (int64_t)n;
    v.position = pos.data();
    v.velocity = vel.data();
    v.acceleration = acc.data();
    v.external = ext.data();
    v.mass = mass.data();
    v.density = rho.data();
    v.pressure = p.data();
    v.type = type.data();
    v.tag = tag.data();
    FS_TRY(fs_download(c, &v));
    fs_ctx* t = nullptr;
    FS_TRY(create_ctx(&c->prm, 0, nullptr, &t));
    struct Guard {
        fs_ctx* t;
        ~Guard() { fs_destroy(t); }
    } guard{t};
    t->tuning = c->tuning;
    double step_ms, l1_ms, iter_ms;
    int samples;
    // 1. prefetch depths
    const int trials[4][2] = {{1, 1}, {2, 2}, {3, 1}, {kMaxAhead, 2}};
    double l1_sum[kMaxAhead + 1] = {}, pi_sum[kMaxAhead + 1] = {};
    int l1_cnt[kMaxAhead + 1] = {}, pi_cnt[kMaxAhead + 1] = {};
    for (const auto& tr : trials) {
        FS_TRY(fs_upload(t, &v));
        t->tuning.pressure_ahead = tr[0];
        t->tuning.l1_ahead = tr[1];
        FS_TRY(time_steps(t, 2, 4, step_ms, l1_ms, iter_ms, samples));
        l1_sum[tr[1]] += l1_ms;
        l1_cnt[tr[1]]++;
        if (samples) {
            pi_sum[tr[0]] += iter_ms;
            pi_cnt[tr[0]]++;
        }
    }
    int best_l1 = c->tuning.l1_ahead, best_pi = c->tuning.pressure_ahead;
    double t_l1 = 1e30, t_pi = 1e30;
    for (int a = 1; a <= kMaxAhead; a++) {
        if (l1_cnt[a]) {
            out->first_loop_ms[a - 1] = (float)(l1_sum[a] / l1_cnt[a]);
            if (l1_sum[a] / l1_cnt[a] < t_l1) t_l1 = l1_sum[a] / l1_cnt[a], best_l1 = a;
        }
        if (pi_cnt[a]) {
            out->pressure_iteration_ms[a - 1] = (float)(pi_sum[a] / pi_cnt[a]);
            if (pi_sum[a] / pi_cnt[a] < t_pi) t_pi = pi_sum[a] / pi_cnt[a], best_pi = a;
        }
    }
    t->tuning.l1_ahead = best_l1;
    t->tuning.pressure_ahead = best_pi;
    // 2. threads per owner in the pressure passes, at the chosen depth
    const int tpos[3] = {1, 2, 4};
    double t_tpo = 1e30;
    int best_tpo = t->tuning.pressure_tpo;
    for (int q = 0; q < 3; q++) {
        FS_TRY(fs_upload(t, &v));
        t->tuning.pressure_tpo = tpos[q];
        FS_TRY(time_steps(t, 2, 4, step_ms, l1_ms, iter_ms, samples));
        if (!samples) continue;
        out->pressure_iteration_ms_by_threads[q] = (float)iter_ms;
        if (iter_ms < t_tpo) t_tpo = iter_ms, best_tpo = tpos[q];
    }
    t->tuning.pressure_tpo = best_tpo;
    // 3. staging cap
    const int caps[4] = {1024, 1536, 2048, 3072};
    double best = 1e30;
    int best_cap = t->tuning.cap;
    for (int q = 0; q < 4; q++) {
        FS_TRY(fs_upload(t, &v));
        t->tuning.cap = caps[q];
        FS_TRY(time_steps(t, 2, 4, step_ms, l1_ms, iter_ms, samples));
        out->step_ms_by_tile_cap[q] = (float)step_ms;
        FS_TRY(fallback_fraction(t, out->fallback_tiles_by_tile_cap[q]));
        if (step_ms < best) best = step_ms, best_cap = caps[q];
    }
    t->tuning.cap = best_cap;
    // 4. block size of the per-particle kernels
    const int blocks[3] = {128, 256, 512};
    best = 1e30;
    int best_block = t->tuning.block;
    for (int q = 0; q < 3; q++) {
        FS_TRY(fs_upload(t, &v));
        t->tuning.block = blocks[q];
        FS_TRY(time_steps(t, 2, 4, step_ms, l1_ms, iter_ms, samples));
        out->step_ms_by_block_size[q] = (float)step_ms;
        if (step_ms < best) best = step_ms, best_block = blocks[q];
    }
    out->tuned = 1;
    out->first_loop_prefetch = best_l1;
    out->pressure_prefetch = best_pi;
    out->tile_cap = best_cap;
    out->block_size = best_block;
    out->pressure_threads_per_owner = best_tpo;
    return fs_set_tuning(c, out);
}

fs_status fs_set_tile_wait_limit(fs_ctx* c, int32_t tries) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    FS_CUDA(cudaSetDevice(c->device));
    const int v = tries < 0 ? kTileWaitTries : tries;
    FS_CUDA(cudaStreamSynchronize(c->stream));
    FS_CUDA(cudaMemcpyToSymbol(g_tile_wait_tries, &v, sizeof(int)));
    return FS_OK;
}

extern "C++" {
namespace {
// the search's sort on caller keys (fs_sort_keys): device buffers for both
// ping-pong halves, values = input positions, sort_pairs as the search runs it
template <typename K>
fs_status sort_keys_impl(int32_t device, const K* keys, int64_t n, int32_t bits, K* sorted, uint32_t* order) {
    for (int64_t i = 0; i < n; i++)
        if (bits < (int)(8 * sizeof(K)) && (keys[i] >> bits) != 0)
            return fail(FS_ERR_INVALID, "key " + std::to_string(i) + " has bits at or above `bits`");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FS_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(FS_ERR_INVALID, "device ordinal out of range");
    FS_CUDA(cudaSetDevice(device));
    if (n == 0) return FS_OK;
    std::vector<uint32_t> iota((size_t)n);
    for (int64_t i = 0; i < n; i++) iota[(size_t)i] = (uint32_t)i;
    K* dk = nullptr;
    uint32_t *dv = nullptr, *hist = nullptr;
    cudaStream_t st = nullptr;
    auto release = [&](fs_status s) {
        cudaFree(dk);
        cudaFree(dv);
        cudaFree(hist);
        if (st) cudaStreamDestroy(st);
        return s;
    };
    if (dalloc(&dk, (size_t)(2 * n)) != FS_OK || dalloc(&dv, (size_t)(2 * n)) != FS_OK ||
        dalloc(&hist, (size_t)sort_hist_entries(n)) != FS_OK)
        return release(FS_ERR_CUDA);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = prepare_small_sort();
    if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys, sizeof(K) * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, iota.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, st);
    int64_t launches = 0;
    int res = 0;
    if (e == cudaSuccess) {
        K* const kb[2] = {dk, dk + n};
        uint32_t* const vb[2] = {dv, dv + n};
        res = sort_pairs<K>(n, bits, kb, vb, hist, st, launches);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && sorted)
        e = cudaMemcpyAsync(sorted, dk + res * n, sizeof(K) * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && order)
        e = cudaMemcpyAsync(order, dv + res * n, 4 * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return release(fail(FS_ERR_CUDA, std::string("fs_sort_keys: ") + cudaGetErrorString(e)));
    return release(FS_OK);
}
}  // namespace
}  // extern "C++"

fs_status fs_sort_keys(int32_t device, const void* keys, int32_t key_bytes, int64_t n, int32_t bits, void* sorted,
                       uint32_t* order) {
    if ((!keys && n > 0) || n < 0) return fail(FS_ERR_INVALID, "null keys or negative count");
    if (n > (int64_t)0xffffffffu) return fail(FS_ERR_INVALID, "more keys than 32-bit positions hold");
    if (key_bytes == 4) {
        if (bits < 1 || bits > 32) return fail(FS_ERR_INVALID, "bits must be in 1..32 for 4-byte keys");
        return sort_keys_impl<uint32_t>(device, static_cast<const uint32_t*>(keys), n, bits,
                                        static_cast<uint32_t*>(sorted), order);
    }
    if (key_bytes == 8) {
        if (bits < 1 || bits > 64) return fail(FS_ERR_INVALID, "bits must be in 1..64 for 8-byte keys");
        return sort_keys_impl<unsigned long long>(device, static_cast<const unsigned long long*>(keys), n, bits,
                                                  static_cast<unsigned long long*>(sorted), order);
    }
    return fail(FS_ERR_INVALID, "key_bytes must be 4 or 8");
}

fs_status fs_set_tuning(fs_ctx* c, const fs_tuning* in) {
    if (!c || !in) return fail(FS_ERR_INVALID, "null argument");
    if (in->first_loop_prefetch < 1 || in->first_loop_prefetch > kMaxAhead || in->pressure_prefetch < 1 ||
        in->pressure_prefetch > kMaxAhead)
        return fail(FS_ERR_INVALID, "prefetch depths must be in 1.." + std::to_string(kMaxAhead));
    if (in->tile_cap != 0 && (in->tile_cap < 256 || in->tile_cap > kTileCapMax || in->tile_cap % 4 != 0))
        return fail(FS_ERR_INVALID, "tile_cap must be 0 or a multiple of 4 in 256.." + std::to_string(kTileCapMax));
    if (in->block_size != 0 && (in->block_size < 32 || in->block_size > 1024 || in->block_size % 32 != 0))
        return fail(FS_ERR_INVALID, "block_size must be 0 or a multiple of 32 in 32..1024");
    const int tpo = in->pressure_threads_per_owner;
    if (tpo != 0 && tpo != 1 && tpo != 2 && tpo != 4)
        return fail(FS_ERR_INVALID, "pressure_threads_per_owner must be 0, 1, 2 or 4");
    TileTuning next = c->tuning;
    next.l1_ahead = in->first_loop_prefetch;
    next.pressure_ahead = in->pressure_prefetch;
    if (in->tile_cap) next.cap = in->tile_cap;
    if (in->block_size) next.block = in->block_size;
    if (tpo) next.pressure_tpo = tpo;
    if (next.l1_ahead != c->tuning.l1_ahead || next.pressure_ahead != c->tuning.pressure_ahead ||
        next.cap != c->tuning.cap || next.block != c->tuning.block || next.pressure_tpo != c->tuning.pressure_tpo) {
        FS_CUDA(cudaSetDevice(c->device));
        if (c->stream) FS_CUDA(cudaStreamSynchronize(c->stream));
        clear_graphs(c);   // the captured steps launch the old instantiations and shapes
        c->tuning = next;
        c->have_lists = false;   // tile lists are built for one cap: search again before solving
    }
    return FS_OK;
}

// the render scene of a 3D single-scene context: a fresh search (the cell
// tables of the current positions) and the particles' box
static fs_status render_scene_of(fs_ctx* c, float surface_fraction, RenderScene& rs) {
    if (c->dim != 3) return fail(FS_ERR_INVALID, "the ray tracer renders 3D particles (MovementData3D)");
    if (c->scenes > 0) return fail(FS_ERR_INVALID, "not available on batched contexts");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (!(surface_fraction > 0.0f)) return fail(FS_ERR_INVALID, "the surface density fraction must be positive");
    FS_CUDA(cudaSetDevice(c->device));
    FS_TRY(search_for_step(c, c->prm.timestep));
    int* d_box = nullptr;
    FS_TRY(dalloc(&d_box, 6));
    const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    int box[6];
    cudaError_t e = cudaMemcpyAsync(d_box, init, sizeof(init), cudaMemcpyHostToDevice, c->stream);
    c->launches++;
    if (e == cudaSuccess) {
        if (c->precision == FS_PRECISION_FP64)
            k_particle_box<double><<<grid_for(c->n), kBlock, 0, c->stream>>>(c->n, state_of<double>(c), d_box);
        else
            k_particle_box<float><<<grid_for(c->n), kBlock, 0, c->stream>>>(c->n, state_of<float>(c), d_box);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(box, d_box, sizeof(box), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_box);
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, std::string("particle box: ") + cudaGetErrorString(e));
    auto unord = [](int i) {
        const int b = i >= 0 ? i : i ^ 0x7fffffff;
        float f;
        std::memcpy(&f, &b, sizeof(f));
        return f;
    };
    const float ext = c->prm.particle_size * 2.0f;   // extended_in_all_directions_by(size * support factor)
    for (int a = 0; a < 3; a++) {
        rs.box_min[a] = box[a] == INT_MAX ? 0.0f : unord(box[a]) - ext;
        rs.box_max[a] = box[3 + a] == INT_MIN ? -1.0f : unord(box[3 + a]) + ext;
    }
    rs.step = c->prm.particle_size / 2.0f;
    rs.iso = surface_fraction * c->prm.rest_density;
    rs.kern.h = c->kernel_h;
    rs.kern.alpha = c->kernel_alpha;
    rs.kern.inv_h = 1.0f / c->kernel_h;
    rs.kern.alpha_h = c->kernel_alpha * c->kernel_h;
    rs.w = walk_of(c, false);
    return FS_OK;
}

fs_status fs_trace_rays(fs_ctx* c, float surface_fraction, int64_t n, const float* origins, const float* directions,
                        int32_t* hit, float* point, float* normal, float* length) {
    if (!c || (n > 0 && (!origins || !directions || !hit || !point || !normal || !length)))
        return fail(FS_ERR_INVALID, "null argument");
    if (n < 0) return fail(FS_ERR_INVALID, "negative ray count");
    RenderScene rs;
    FS_TRY(render_scene_of(c, surface_fraction, rs));
    if (n == 0) return FS_OK;
    float *d_in = nullptr, *d_out = nullptr;
    int32_t* d_hit = nullptr;
    FS_TRY(dalloc(&d_in, (size_t)n * 6));
    if (dalloc(&d_out, (size_t)n * 7) != FS_OK || dalloc(&d_hit, (size_t)n) != FS_OK) {
        cudaFree(d_in);
        cudaFree(d_out);
        return fail(FS_ERR_CUDA, "allocation for the rays failed");
    }
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemcpyAsync(d_in, origins, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_in + 3 * n, directions, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        c->launches++;
        if (c->precision == FS_PRECISION_FP64)
            k_trace_rays<double><<<grid_for(n), kBlock, 0, st>>>(n, d_in, d_in + 3 * n, state_of<double>(c),
                                                                 c->cell_start, rs, d_hit, d_out, d_out + 3 * n,
                                                                 d_out + 6 * n);
        else
            k_trace_rays<float><<<grid_for(n), kBlock, 0, st>>>(n, d_in, d_in + 3 * n, state_of<float>(c),
                                                                c->cell_start, rs, d_hit, d_out, d_out + 3 * n,
                                                                d_out + 6 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit, d_hit, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(point, d_out, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(normal, d_out + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(length, d_out + 6 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_hit);
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, std::string("ray tracing: ") + cudaGetErrorString(e));
    return FS_OK;
}

void fs_render_settings_default(fs_render_settings* r) {
    if (!r) return;
    *r = fs_render_settings{};
    r->samples_per_pixel = 50;         // Camera::SampleSettings (Camera.hpp:23-26)
    r->maximum_recursion_depth = 10;   // FluidRaytracer3D::Settings (FluidRaytracer3D.hpp:22-25)
    r->output_normals_of_first_hit = 0;
    r->surface_density_fraction = 0.8f;   // ParticleIntersectionAccelerator.hpp:20
    r->exposure = 0.2f;                   // ToneMapper::ToneMapperSettings (ToneMapper.hpp:11-20)
    r->gamma = 2.2f;
    r->seed = 1;
    r->tone_mapper = 0;                   // ToneMapperFunction::Exponential
    r->gamma_correction = 1;
}

// ToneMapper's mapping of one radiance value to a byte colour
// (ToneMapper.cpp:7-102), in the reference's float operations: exposure,
// the exponential 1 - exp(-v) or the ACES filmic curve (with its clamp),
// the clamp to [0, 1], the gamma correction pow(v, 1 / gamma), and the
// byte (clamp(v) * 255, truncated).
static float tone_clamp(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }
static void tone_map_pixels(const float* radiance, int64_t np, const fs_render_settings* r, uint8_t* rgba) {
    const float gpow = 1.0f / r->gamma;
    for (int64_t i = 0; i < np; i++) {
        for (int a = 0; a < 3; a++) {
            float v = radiance[3 * i + a] * r->exposure;
            if (r->tone_mapper == 1) {
                const float ka = 2.51f, kb = 0.03f, kc = 2.43f, kd = 0.59f, ke = 0.14f;
                v = tone_clamp((v * (ka * v + kb)) / (v * (kc * v + kd) + ke));
            } else {
                v = 1.0f - std::exp(-v);
            }
            v = tone_clamp(v);
            if (r->gamma_correction) v = std::pow(v, gpow);
            rgba[4 * i + a] = (uint8_t)(tone_clamp(v) * 255.0f);
        }
        rgba[4 * i + 3] = 255;
    }
}

fs_status fs_tone_map(const float* radiance, int64_t pixels, const fs_render_settings* r, uint8_t* rgba) {
    if (!radiance || !r || !rgba || pixels < 0) return fail(FS_ERR_INVALID, "null argument or negative size");
    if (r->tone_mapper != 0 && r->tone_mapper != 1) return fail(FS_ERR_INVALID, "tone_mapper must be 0 or 1");
    tone_map_pixels(radiance, pixels, r, rgba);
    return FS_OK;
}

fs_status fs_render(fs_ctx* c, const fs_camera* cam, const fs_render_settings* r, float* radiance, uint8_t* rgba) {
    if (!c || !cam || !r || !radiance) return fail(FS_ERR_INVALID, "null argument");
    if (r->tone_mapper != 0 && r->tone_mapper != 1) return fail(FS_ERR_INVALID, "tone_mapper must be 0 or 1");
    if (cam->width <= 0 || cam->height <= 0 || (int64_t)cam->width * cam->height > (int64_t)1 << 26)
        return fail(FS_ERR_INVALID, "image size out of range");
    if (r->samples_per_pixel <= 0 || r->maximum_recursion_depth < 0) return fail(FS_ERR_INVALID, "bad settings");
    RenderScene rs;
    FS_TRY(render_scene_of(c, r->surface_density_fraction, rs));
    // the camera: glm::lookAt's basis (Camera.cpp:41-44); the ray direction is the inverse view
    // rotation applied to the pixel's view-space direction
    RenderCamera rc{};
    const float* f0 = cam->view_direction;
    const float fl = std::sqrt(f0[0] * f0[0] + f0[1] * f0[1] + f0[2] * f0[2]);
    const float f[3] = {f0[0] / fl, f0[1] / fl, f0[2] / fl};
    const float* up = cam->view_up;
    float sv[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    const float sl = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    if (!(sl > 0.0f) || !(fl > 0.0f)) return fail(FS_ERR_INVALID, "view direction and up vector must span a plane");
    for (int a = 0; a < 3; a++) sv[a] /= sl;
    const float uv[3] = {sv[1] * f[2] - sv[2] * f[1], sv[2] * f[0] - sv[0] * f[2], sv[0] * f[1] - sv[1] * f[0]};
    for (int a = 0; a < 3; a++) {
        rc.pos[a] = cam->position[a];
        rc.right[a] = sv[a];
        rc.up[a] = uv[a];
        rc.back[a] = -f[a];
    }
    rc.tan_half_fov = std::tan(cam->field_of_view_x / 2.0f);
    rc.width = cam->width;
    rc.height = cam->height;
    rc.flip_y = cam->flip_y;
    RenderShading sh{};
    const float pi = 3.14159265358979323846f;
    const float fc[3] = {0.1f, 0.15f, 0.5f}, bc[3] = {0.0f, 0.42f, 0.063f};   // FluidRaytracer3D.cpp:183-184
    for (int a = 0; a < 3; a++) {
        sh.fluid[a] = std::pow(fc[a], 2.2f) * (1.0f / pi);
        sh.boundary[a] = std::pow(bc[a], 2.2f) * (1.0f / pi);
    }
    sh.samples = r->samples_per_pixel;
    sh.max_depth = r->maximum_recursion_depth;
    sh.normals_only = r->output_normals_of_first_hit != 0;
    sh.seed = r->seed;
    const int64_t np = (int64_t)cam->width * cam->height;
    float* d_rad = nullptr;
    FS_TRY(dalloc(&d_rad, (size_t)np * 3));
    c->launches++;
    if (c->precision == FS_PRECISION_FP64)
        k_render<double><<<grid_for(np), kBlock, 0, c->stream>>>(state_of<double>(c), c->cell_start, rs, rc, sh, d_rad);
    else
        k_render<float><<<grid_for(np), kBlock, 0, c->stream>>>(state_of<float>(c), c->cell_start, rs, rc, sh, d_rad);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(radiance, d_rad, sizeof(float) * 3 * np, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_rad);
    if (e != cudaSuccess) return fail(FS_ERR_CUDA, std::string("rendering: ") + cudaGetErrorString(e));
    if (rgba) tone_map_pixels(radiance, np, r, rgba);   // ToneMapper::map_render_target_to_image
    return FS_OK;
}

fs_status fs_last_phase_times(fs_ctx* c, float* ms5) {
    if (!c || !ms5) return fail(FS_ERR_INVALID, "null argument");
    for (int i = 0; i < 5; i++) ms5[i] = c->phase_ms[i];
    return FS_OK;
}

void* fs_stream(fs_ctx* c) { return c ? (void*)c->stream : nullptr; }

int64_t fs_launch_count(fs_ctx* c) { return c ? c->launches : 0; }

int32_t fs_small_blocks(fs_ctx* c) { return c && c->small_last ? c->small_blocks : 0; }

fs_status fs_batch_create(const fs_params* p, int32_t scenes, const int64_t* offsets, fs_ctx** out) {
    if (out) *out = nullptr;
    if (!p || !offsets || !out) return fail(FS_ERR_INVALID, "null argument");
    if (scenes < 1 || scenes > 65535) return fail(FS_ERR_INVALID, "scenes must be 1..65535");
    if (offsets[0] != 0) return fail(FS_ERR_INVALID, "offsets[0] must be 0");
    for (int32_t i = 0; i < scenes; i++)
        if (offsets[i + 1] < offsets[i]) return fail(FS_ERR_INVALID, "offsets must not decrease");
    if (p->solver != FS_SOLVER_IISPH_3D || p->search != FS_SEARCH_HASHED_3D ||
        p->precision != FS_PRECISION_FP32_KAHAN || (p->flags & FS_FLAG_REFERENCE_ORDER))
        return fail(FS_ERR_INVALID,
                    "batched scenes run the 3D IISPH solver with the hashed-3d contract in FP32 + Kahan, device order");
    return create_ctx(p, scenes, offsets, out);
}

fs_status fs_batch_run(fs_ctx* c, int32_t steps, float desired_dt, fs_step_stats* stats) {
    if (!c) return fail(FS_ERR_INVALID, "ctx is null");
    if (c->scenes == 0) return fail(FS_ERR_INVALID, "not a batched context (fs_batch_create)");
    if (steps < 0) return fail(FS_ERR_INVALID, "steps must be >= 0");
    FS_CUDA(cudaSetDevice(c->device));
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles uploaded");
    if (steps == 0) return FS_OK;
    FS_TRY(one_step(c, desired_dt, nullptr));
    if (steps > 1) {
        const float dt = desired_of(c, desired_dt);
        FS_TRY(enqueue_steps(c, steps - 1, dt));
        int st = 0;
        FS_TRY(finish_steps(c, nullptr, &st));
        if (st != FS_OK) return fail((fs_status)st, "device reported an error during fs_batch_run");
    }
    return fill_stats(c, stats, FS_OK, c->scenes);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Position query that allocates nothing (fs_query_position_noalloc).
//
// Who cannot allocate: code that asks for neighbors while a simulation is
// running -- an entity or sensor hook between two steps, a render or
// telemetry callback on its own thread. cudaFree waits for the whole device,
// so it stalls a step queued on any stream, and cudaMalloc can do the same;
// on a device whose memory is budgeted to the particle buffers a fresh
// allocation can also just fail halfway through a run; and a host heap call
// adds unbounded latency to a callback with a frame deadline. So this path
// works from one fixed device array per device, compiled into the library,
// and copies straight into the caller's buffer. It uses no cudaMalloc,
// cudaFree or host-side allocation; even its error messages fit the error
// string's inline storage.
//
// Shared state: one array per device, used by every context on it. Calls
// that overlap in time on one device race on the array (the count and the
// results). Set-up: the first call on a device, with that device current,
// resolves the array's address with cudaGetSymbolAddress and keeps it; that
// first call should come before any stream capture begins.
// ---------------------------------------------------------------------------

// [0]: neighbor count (zeroed before every launch); [1 ..]: host indices
static __device__ __align__(256) unsigned long long g_query_scratch[1 + FS_QUERY_NOALLOC_MAX];

namespace {

constexpr int kNoAllocDevices = 64;
std::mutex g_query_scratch_mutex;
unsigned long long* g_query_scratch_ptr[kNoAllocDevices] = {};

// k_query_position writing host indices into the fixed array
template <typename R>
__global__ void k_query_cells_noalloc(V3<R> x, const V4<R>* __restrict__ pos, const uint8_t* __restrict__ type,
                                      const uint32_t* __restrict__ hidx, const uint32_t* __restrict__ cell_start,
                                      WalkParams w, bool skip_cell_min,
                                      unsigned long long* __restrict__ scratch, int64_t cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long c = 0;
    const int ci[3] = {cell_coord<R>(x.x, w.r, w.trunc), cell_coord<R>(x.y, w.r, w.trunc), cell_coord<R>(x.z, w.r, w.trunc)};
    const int zr = w.dim == 2 ? 0 : 1;
    int ordinal = 0;
    for (int dx = -1; dx <= 1; dx++) {
        for (int dy = -1; dy <= 1; dy++) {
            for (int dz = -zr; dz <= zr; dz++, ordinal++) {
                const int c0 = ci[0] + dx, c1 = ci[1] + dy, c2 = ci[2] + dz;
                bool cl = false;
                const SceneGrid& gr = w.grids[0];
                const int l0 = local_cell(c0, gr.o0, gr.d0, cl);
                const int l1 = local_cell(c1, gr.o1, gr.d1, cl);
                const int l2 = local_cell(c2, gr.o2, gr.d2, cl);
                const int64_t lc = gr.base + ((int64_t)l2 * gr.d1 + l1) * gr.d0 + l0;
                auto members = [&](auto&& f) {
                    for (int g = 0; g < w.regions; g++) {
                        const uint32_t* cs = cell_start + g * (w.cells + 1);
                        for (uint32_t j = cs[lc], e = cs[lc + 1]; j < e; j++) {
                            const V4<R> pj = pos[j];
                            if (cl && (cell_coord<R>(pj.x, w.r, w.trunc) != c0 ||
                                       cell_coord<R>(pj.y, w.r, w.trunc) != c1 ||
                                       cell_coord<R>(pj.z, w.r, w.trunc) != c2))
                                continue;
                            if (!w.candidates_inactive && type[j] == FS_TYPE_INACTIVE) continue;
                            f(j, pj);
                        }
                    }
                };
                uint32_t skip = 0xffffffffu;
                if (skip_cell_min && ordinal > 0) members([&](uint32_t j, const V4<R>&) { skip = min(skip, hidx[j]); });
                members([&](uint32_t j, const V4<R>& pj) {
                    if (hidx[j] == skip || !within<R>(x - xyz<R>(pj), w)) return;
                    if ((int64_t)c < cap) scratch[1 + c] = hidx[j];
                    c++;
                });
            }
        }
    }
    scratch[0] = c;
}

// k_query_all writing host indices into the fixed array; scratch[0] must be
// zero at the launch
template <typename R>
__global__ void k_query_all_noalloc(V3<R> x, int64_t n, const V4<R>* __restrict__ pos,
                                    const uint32_t* __restrict__ hidx, WalkParams w,
                                    unsigned long long* __restrict__ scratch, int64_t cap) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        if (!within<R>(x - xyz<R>(pos[j]), w)) continue;
        const unsigned long long slot = atomicAdd(&scratch[0], 1ull);
        if ((int64_t)slot < cap) scratch[1 + slot] = hidx[j];
    }
}

// the fixed array of the current device (resolved once per device)
fs_status query_scratch(int device, unsigned long long** out) {
    if (device < 0 || device >= kNoAllocDevices) return fail(FS_ERR_INVALID, "bad device");
    std::lock_guard<std::mutex> lock(g_query_scratch_mutex);
    if (!g_query_scratch_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_query_scratch) != cudaSuccess || !p) return fail(FS_ERR_CUDA, "CUDA symbol");
        g_query_scratch_ptr[device] = (unsigned long long*)p;
    }
    *out = g_query_scratch_ptr[device];
    return FS_OK;
}

template <typename R>
bool launch_query_noalloc(fs_ctx* c, const float* position, const WalkParams& w, bool all, bool skip,
                          unsigned long long* scratch, int64_t cap) {
    const State<R> s = state_of<R>(c);
    const V3<R> x = v3<R>(position[0], position[1], c->dim == 3 ? position[2] : 0.0f);
    c->launches++;
    if (all) {
        const int g = (int)std::min<int64_t>((c->n + kBlock - 1) / kBlock, 1184);
        k_query_all_noalloc<R><<<g, kBlock, 0, c->stream>>>(x, c->n, s.pos, s.hidx, w, scratch, cap);
    } else {
        k_query_cells_noalloc<R><<<1, 32, 0, c->stream>>>(x, s.pos, s.type, s.hidx, c->cell_start, w, skip,
                                                          scratch, cap);
    }
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace

extern "C" fs_status fs_query_position_noalloc(fs_ctx* c, const float* position, int64_t* out, int64_t cap,
                                               int64_t* count) {
    // every message below fits std::string's inline buffer: no heap use
    if (!c || !position || (cap > 0 && !out)) return fail(FS_ERR_INVALID, "null argument");
    if (cap < 0) return fail(FS_ERR_INVALID, "cap < 0");
    if (cap > FS_QUERY_NOALLOC_MAX) return fail(FS_ERR_INVALID, "cap > 65536");
    if (!c->have_state) return fail(FS_ERR_STATE, "no particles");
    if (c->scenes > 0) return fail(FS_ERR_INVALID, "batched ctx");
    const int search = c->prm.search;
    if (search == FS_SEARCH_COMPACT_2D) return fail(FS_ERR_INVALID, "not supported");
    const bool all = search == FS_SEARCH_QUADRATIC_2D || search == FS_SEARCH_QUADRATIC_3D;
    if (!all && !c->have_cells) return fail(FS_ERR_STATE, "search first");
    if (count) *count = 0;
    if (c->n == 0) return FS_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(FS_ERR_CUDA, "CUDA device");
    unsigned long long* scratch = nullptr;
    FS_TRY(query_scratch(c->device, &scratch));
    WalkParams w = walk_of(c, false);
    w.length_test = search != FS_SEARCH_COMPRESSED_3D;
    const bool skip = search == FS_SEARCH_HASHED_3D;
    if (cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), c->stream) != cudaSuccess)
        return fail(FS_ERR_CUDA, "CUDA memset");
    const bool launched = c->precision == FS_PRECISION_FP64
                              ? launch_query_noalloc<double>(c, position, w, all, skip, scratch, cap)
                              : launch_query_noalloc<float>(c, position, w, all, skip, scratch, cap);
    if (!launched) return fail(FS_ERR_CUDA, "CUDA launch");
    unsigned long long cnt = 0;
    if (cudaMemcpyAsync(&cnt, scratch, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return fail(FS_ERR_CUDA, "CUDA copy");
    const int64_t m = std::min<int64_t>((int64_t)cnt, cap);
    if (m > 0 && (cudaMemcpyAsync(out, scratch + 1, sizeof(int64_t) * (size_t)m, cudaMemcpyDeviceToHost,
                                  c->stream) != cudaSuccess ||
                  cudaStreamSynchronize(c->stream) != cudaSuccess))
        return fail(FS_ERR_CUDA, "CUDA copy");
    std::sort(out, out + m);
    if (count) *count = (int64_t)cnt;
    return FS_OK;
}
