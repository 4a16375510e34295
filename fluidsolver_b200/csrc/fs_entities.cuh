// Entities and sensors of the Simulator that read the whole particle
// collection, run where the state lives: libFluid's BoundaryPreprocessor
// (entities/BoundaryPreprocessor.cpp) and its global particle statistics
// (sensors/ParticleStatistics.cpp).
#pragma once

#include "fs_common.cuh"
#include "fs_search.cuh"
#include "fs_solvers.cuh"

namespace fsb {

// ---------------------------------------------------------------------------
// BoundaryPreprocessor::execute_simulation_step (BoundaryPreprocessor.cpp:7-48).
// For every boundary particle i, over the boundary particles b of its
// neighbor list (the contract's walk, i itself included), in list order:
//   mass_i = min(rho0 size^3, rho0 gamma_1 / sum_b W(x_i - x_b))
// gamma_1 = size^3 * sum W over a perfectly sampled plane, x = 0 and
// y, z in -2..2 spacings, y outer (calculate_ideal_volume_reciprocal and
// calculate_gamma_1_from_ideal_volume_reciprocal, :104-119); rho0 size^3 is
// calculate_max_allowed_mass (:120-122). Math::min is fmin.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_boundary_mass(int64_t n, State<R> s, const uint32_t* __restrict__ cell_start, WalkParams w,
                                SplineKernel<R> kern, R rest_density, R particle_size) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || s.type[k] != FS_TYPE_BOUNDARY) return;
    R ideal = R(0);
    for (int y = -2; y <= 2; y++)
        for (int z = -2; z <= 2; z++)
            ideal += kern.W(v3<R>(R(0) * particle_size, (R)y * particle_size, (R)z * particle_size));
    const R size3 = (particle_size * particle_size) * particle_size;
    const R gamma_1 = size3 * ideal;
    const R max_mass = rest_density * size3;
    const V3<R> xi = xyz<R>(s.pos[k]);
    R volume_reciprocal = R(0);
    walk_cells<R>(xi, s.pos, s.type, cell_start, w.grid_of(k), w, [&](uint32_t j, uint8_t tj) {
        if (tj != FS_TYPE_BOUNDARY) return;
        volume_reciprocal += kern.W(xi - xyz<R>(s.pos[j]));
    });
    const R corrected = rest_density * gamma_1 / volume_reciprocal;
    s.pos[k].w = fmin(max_mass, corrected);
}

// ---------------------------------------------------------------------------
// Global statistics (ParticleStatistics.cpp:17-201) in two deterministic
// passes: per-block partial results, then one block folds them in block
// order. Per normal particle, in float as the reference: density, pressure,
// |v| (glm::length), the kinetic term (0.5 m) |v| |v| and the potential term
// (g m) (y - zero_height); sums in FP64.
// ---------------------------------------------------------------------------
struct StatsPart {
    double sum[5];               // density, pressure, |v|, kinetic, potential
    float mx[3], mn[3];          // density, pressure, |v|
    unsigned long long cnt[3];   // normal, boundary, inactive particles
};
constexpr int kStatsBlocks = 592;   // 4 blocks of 256 threads per SM of a B200
constexpr int kStatsThreads = 256;

struct StatsOut {   // the layout of fs_global_stats
    float density_max, density_min, density_avg;
    float pressure_max, pressure_min, pressure_avg;
    float velocity_max, velocity_min, velocity_avg;
    float kinetic_energy, potential_energy;
    int32_t reserved;
    long long normal, boundary, inactive;
};

__device__ __forceinline__ void fold_part(StatsPart& a, const StatsPart& b) {
    for (int i = 0; i < 5; i++) a.sum[i] += b.sum[i];
    for (int i = 0; i < 3; i++) {
        a.mx[i] = fmaxf(a.mx[i], b.mx[i]);
        a.mn[i] = fminf(a.mn[i], b.mn[i]);
        a.cnt[i] += b.cnt[i];
    }
}

__device__ __forceinline__ StatsPart empty_part() {
    StatsPart p;
    for (int i = 0; i < 5; i++) p.sum[i] = 0.0;
    for (int i = 0; i < 3; i++) {
        p.mx[i] = 1.17549435e-38f;   // std::numeric_limits<float>::min(), MaxMinAvgSensorData's start
        p.mn[i] = 3.40282347e+38f;   // std::numeric_limits<float>::max()
        p.cnt[i] = 0;
    }
    return p;
}

// block-wide fold of one StatsPart per thread into thread 0's
__device__ __forceinline__ StatsPart fold_block(StatsPart p) {
    __shared__ StatsPart sh[kStatsThreads];
    sh[threadIdx.x] = p;
    __syncthreads();
    for (int step = kStatsThreads / 2; step > 0; step >>= 1) {
        if ((int)threadIdx.x < step) fold_part(sh[threadIdx.x], sh[threadIdx.x + step]);
        __syncthreads();
    }
    return sh[0];
}

template <typename R>
__global__ void __launch_bounds__(kStatsThreads) k_stats_partial(int64_t n, State<R> s, float gravity,
                                                                  float zero_height, StatsPart* __restrict__ parts) {
    StatsPart p = empty_part();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t t = s.type[k];
        if (t == FS_TYPE_BOUNDARY) {
            p.cnt[1]++;
        } else if (t == FS_TYPE_INACTIVE) {
            p.cnt[2]++;
        } else if (t == FS_TYPE_NORMAL) {
            p.cnt[0]++;
            const V4<R> x = s.pos[k], v = s.vel[k];
            const float mass = (float)x.w, rho = (float)s.rho[k], pr = (float)s.p[k];
            const float vx = (float)v.x, vy = (float)v.y, vz = (float)v.z;
            const float speed = sqrtf((vx * vx + vy * vy) + vz * vz);
            const float vals[3] = {rho, pr, speed};
            for (int i = 0; i < 3; i++) {
                p.sum[i] += (double)vals[i];
                p.mx[i] = fmaxf(p.mx[i], vals[i]);
                p.mn[i] = fminf(p.mn[i], vals[i]);
            }
            p.sum[3] += (double)(((0.5f * mass) * speed) * speed);
            p.sum[4] += (double)((gravity * mass) * ((float)x.y - zero_height));
        }
    }
    p = fold_block(p);
    if (threadIdx.x == 0) parts[blockIdx.x] = p;
}

__global__ void __launch_bounds__(kStatsThreads) k_stats_finish(const StatsPart* __restrict__ parts, int nparts,
                                                                 StatsOut* __restrict__ out) {
    StatsPart p = empty_part();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) fold_part(p, parts[i]);
    p = fold_block(p);
    if (threadIdx.x != 0) return;
    const double cnt = (double)p.cnt[0];
    StatsOut o;
    o.density_max = p.mx[0];
    o.density_min = p.mn[0];
    o.density_avg = p.cnt[0] ? (float)(p.sum[0] / cnt) : 0.0f;
    o.pressure_max = p.mx[1];
    o.pressure_min = p.mn[1];
    o.pressure_avg = p.cnt[0] ? (float)(p.sum[1] / cnt) : 0.0f;
    o.velocity_max = p.mx[2];
    o.velocity_min = p.mn[2];
    o.velocity_avg = p.cnt[0] ? (float)(p.sum[2] / cnt) : 0.0f;
    o.kinetic_energy = (float)p.sum[3];
    o.potential_energy = (float)p.sum[4];
    o.reserved = 0;
    o.normal = (long long)p.cnt[0];
    o.boundary = (long long)p.cnt[1];
    o.inactive = (long long)p.cnt[2];
    *out = o;
}

}  // namespace fsb
