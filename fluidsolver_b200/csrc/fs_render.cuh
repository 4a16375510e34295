// The fluid path tracer of libFluid's visualizer (visualizer/raytracer/) on
// the device state: rays marched through the SPH density of the particles
// (ParticleIntersectionAccelerator.cpp), a stochastic path tracer over the
// surfaces they find (FluidRaytracer3D.cpp:70-200) with a white sky (the
// Skybox without an image, Skybox.cpp:27-31), and the pinhole camera of
// Camera.cpp:10-39. One thread per ray (fs_trace_rays) or per pixel
// (fs_render); the density at a march point is a walk over the 27 cells of
// the search grid around it.
#pragma once

#include "fs_common.cuh"
#include "fs_search.cuh"
#include "fs_solvers.cuh"

namespace fsb {

// ParticleIntersectionAccelerator::VolumeEvaluationResult (.hpp:40-54)
struct VolumeEval {
    float density = 0.f, fluid_density = 0.f, boundary_density = 0.f;
    V3<float> fluid_normal = v3<float>(0.f, 0.f, 0.f), boundary_normal = v3<float>(0.f, 0.f, 0.f);
    V3<float> position = v3<float>(0.f, 0.f, 0.f);
};

struct RenderScene {
    float box_min[3], box_max[3];   // the particles' box, extended by the kernel support
    float step;                     // the march step, particle_size / 2
    float iso;                      // surface density: fraction * rest density
    SplineKernel<float> kern;
    WalkParams w;
};

__device__ __forceinline__ V3<float> lerp3(V3<float> a, V3<float> b, float f) {
    return v3<float>((1.0f - f) * a.x + b.x * f, (1.0f - f) * a.y + b.y * f, (1.0f - f) * a.z + b.z * f);
}

// Math::safe_normalize (LibFluidMath.hpp:36-42): zero where normalize gives NaN
__device__ __forceinline__ V3<float> safe_normalize(V3<float> v) {
    const float l = sqrtf(dot(v, v));
    const V3<float> r = v3<float>(v.x / l, v.y / l, v.z / l);
    if (isnan(r.x) || isnan(r.y) || isnan(r.z)) return v3<float>(0.f, 0.f, 0.f);
    return r;
}

// evaluate_volume_at_position (:76-126): sums over the non-inactive particles
// within the search radius of x; the normals sum m_j GetKernelDerivativeValue(x - x_j)
template <typename R>
__device__ VolumeEval evaluate_volume(V3<float> x, const State<R>& s, const uint32_t* __restrict__ cell_start,
                                      const RenderScene& rs) {
    VolumeEval e;
    e.position = x;
    walk_cells<R>(v3<R>((R)x.x, (R)x.y, (R)x.z), s.pos, s.type, cell_start, rs.w.grid_of(0), rs.w,
                  [&](uint32_t j, uint8_t tj) {
                      if (tj == FS_TYPE_INACTIVE) return;
                      const V4<R> pj = s.pos[j];
                      const V3<float> d = v3<float>(x.x - (float)pj.x, x.y - (float)pj.y, x.z - (float)pj.z);
                      const float m = (float)pj.w;
                      const float c = m * rs.kern.W(d);
                      const V3<float> g = rs.kern.gradW(d);   // -GetKernelDerivativeValue(d)
                      e.density += c;
                      if (tj == FS_TYPE_NORMAL) {
                          e.fluid_density += c;
                          e.fluid_normal = v3<float>(e.fluid_normal.x - m * g.x, e.fluid_normal.y - m * g.y,
                                                     e.fluid_normal.z - m * g.z);
                      } else if (tj == FS_TYPE_BOUNDARY) {
                          e.boundary_density += c;
                          e.boundary_normal = v3<float>(e.boundary_normal.x - m * g.x,
                                                        e.boundary_normal.y - m * g.y,
                                                        e.boundary_normal.z - m * g.z);
                      }
                  });
    return e;
}

// get_volume_state (:181-193): 0 outside, 1 fluid, 2 boundary
__device__ __forceinline__ int volume_state(const VolumeEval& e, float iso) {
    if (e.density < iso) return 0;
    return e.fluid_density > e.boundary_density ? 1 : 2;
}

// is_surface_intersected (:128-179). type: 0 the fluid surface reached from
// outside, 1 from inside, 2 a boundary surface
__device__ bool surface_crossed(const VolumeEval& last, const VolumeEval& cur, float iso, int& type,
                                V3<float>& point, V3<float>& normal) {
    const int ls = volume_state(last, iso), cs = volume_state(cur, iso);
    if (ls == cs || ls == 2) return false;
    if (ls == 0) {
        const float f = (iso - last.density) / (cur.density - last.density);
        point = lerp3(last.position, cur.position, f);
        if (cs == 1) {
            type = 0;
            normal = safe_normalize(lerp3(last.fluid_normal, cur.fluid_normal, f));
        } else {
            type = 2;
            normal = safe_normalize(lerp3(last.boundary_normal, cur.boundary_normal, f));
        }
    } else if (cs == 0) {
        type = 1;
        const float f = (last.density - iso) / (last.density - cur.density);
        point = lerp3(last.position, cur.position, f);
        normal = safe_normalize(lerp3(last.fluid_normal, cur.fluid_normal, f));
    } else {
        type = 2;
        const float f = (last.boundary_density - last.fluid_density) /
                        (cur.fluid_density - last.fluid_density - cur.boundary_density + last.boundary_density);
        point = lerp3(last.position, cur.position, f);
        normal = safe_normalize(lerp3(last.boundary_normal, cur.boundary_normal, f));
    }
    return true;
}

// AABB::is_ray_intersecting (AABB.cpp:7-37), the slab test with Math::min/max
__device__ __forceinline__ bool box_hit(const RenderScene& rs, V3<float> o, V3<float> d) {
    const float tx1 = (rs.box_min[0] - o.x) / d.x, tx2 = (rs.box_max[0] - o.x) / d.x;
    const float txn = fminf(tx1, tx2), txf = fmaxf(tx1, tx2);
    const float ty1 = (rs.box_min[1] - o.y) / d.y, ty2 = (rs.box_max[1] - o.y) / d.y;
    const float tyn = fminf(ty1, ty2), tyf = fmaxf(ty1, ty2);
    if (txn > tyf || tyn > txf) return false;
    const float tn = fmaxf(txn, tyn), tf = fminf(txf, tyf);
    const float tz1 = (rs.box_min[2] - o.z) / d.z, tz2 = (rs.box_max[2] - o.z) / d.z;
    const float tzn = fminf(tz1, tz2), tzf = fmaxf(tz1, tz2);
    return !(tn > tzf || tzn > tf);
}

__device__ __forceinline__ bool box_contains(const RenderScene& rs, V3<float> p) {
    return !(p.x < rs.box_min[0] || p.x > rs.box_max[0] || p.y < rs.box_min[1] || p.y > rs.box_max[1] ||
             p.z < rs.box_min[2] || p.z > rs.box_max[2]);
}

// is_intersecting_with_particles (:20-74): march points x + (step t + offset) d,
// t = 1 .. 10^6 - 1, the surface is where the volume state changes. Points
// outside the box are skipped until the ray has entered it and end the march
// once it has left. Only the t whose points the box can hold are visited
// (the slab range, widened by two steps); the others would be skipped.
template <typename R>
__device__ bool trace_ray(V3<float> o, V3<float> d, float offset, const State<R>& s,
                          const uint32_t* __restrict__ cell_start, const RenderScene& rs, int& type,
                          V3<float>& point, V3<float>& normal, float& length) {
    if (!box_hit(rs, o, d)) return false;
    constexpr long long kMaxSteps = 1000000;
    long long t0 = 1, t1 = kMaxSteps - 1;
    {
        float near = -INFINITY, far = INFINITY;
        const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            const float u = (rs.box_min[a] - oo[a]) / dd[a], v = (rs.box_max[a] - oo[a]) / dd[a];
            if (isnan(u) || isnan(v)) ok = false;
            near = fmaxf(near, fminf(u, v));
            far = fminf(far, fmaxf(u, v));
        }
        if (ok) {
            if (far < 0.f) return false;   // the box lies behind the ray: every point is skipped
            const double lo = floor(((double)near - offset) / rs.step) - 2.0;
            const double hi = ceil(((double)far - offset) / rs.step) + 2.0;
            t0 = lo > 1.0 ? (long long)lo : 1;
            t1 = hi < (double)(kMaxSteps - 1) ? (long long)hi : kMaxSteps - 1;
        }
    }
    const float hs = rs.step / 2.0f;
    VolumeEval last = evaluate_volume<R>(v3<float>(o.x + hs * d.x, o.y + hs * d.y, o.z + hs * d.z), s, cell_start, rs);
    bool within = false;
    for (long long t = t0; t <= t1; t++) {
        const float a = rs.step * (float)t + offset;
        const V3<float> p = v3<float>(o.x + a * d.x, o.y + a * d.y, o.z + a * d.z);
        if (!box_contains(rs, p)) {
            if (within) break;
            continue;
        }
        within = true;
        const VolumeEval cur = evaluate_volume<R>(p, s, cell_start, rs);
        if (surface_crossed(last, cur, rs.iso, type, point, normal)) {
            length = rs.step * (float)t;
            return true;
        }
        last = cur;
    }
    return false;
}

template <typename R>
__global__ void k_trace_rays(int64_t nrays, const float* __restrict__ origins, const float* __restrict__ dirs,
                             State<R> s, const uint32_t* __restrict__ cell_start, RenderScene rs,
                             int32_t* __restrict__ hit, float* __restrict__ point, float* __restrict__ normal,
                             float* __restrict__ length) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nrays) return;
    const V3<float> o = v3<float>(origins[3 * r], origins[3 * r + 1], origins[3 * r + 2]);
    const V3<float> d = v3<float>(dirs[3 * r], dirs[3 * r + 1], dirs[3 * r + 2]);
    int type = -1;
    V3<float> p = v3<float>(0.f, 0.f, 0.f), n = p;
    float len = -1.0f;
    const bool h = trace_ray<R>(o, d, 0.0f, s, cell_start, rs, type, p, n, len);
    hit[r] = h ? type : -1;
    point[3 * r] = p.x;
    point[3 * r + 1] = p.y;
    point[3 * r + 2] = p.z;
    normal[3 * r] = n.x;
    normal[3 * r + 1] = n.y;
    normal[3 * r + 2] = n.z;
    length[r] = h ? len : -1.0f;
}

// the particles' box (calculate_aabb, :54-74), as ordered integer bits
__device__ __forceinline__ int ordered(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float unordered(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

template <typename R>
__global__ void k_particle_box(int64_t n, State<R> s, int* __restrict__ box) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n || s.type[k] == FS_TYPE_INACTIVE) return;
    const V4<R> p = s.pos[k];
    const float c[3] = {(float)p.x, (float)p.y, (float)p.z};
    for (int a = 0; a < 3; a++) {
        atomicMin(&box[a], ordered(c[a]));
        atomicMax(&box[3 + a], ordered(c[a]));
    }
}

// ---------------------------------------------------------------------------
// the path tracer (FluidRaytracer3D::evaluate_ray, :70-165)
// ---------------------------------------------------------------------------
struct RenderCamera {
    float pos[3];
    float right[3], up[3], back[3];   // the inverse view rotation's columns
    float tan_half_fov;
    int width, height, flip_y;
};
struct RenderShading {
    float fluid[3], boundary[3];      // bsdf: the colours (gamma 2.2 decoded) over pi
    int samples, max_depth, normals_only;
    unsigned long long seed;
};

// a counter-based stream of uniform floats in [0, 1) per pixel
struct PixelRng {
    unsigned long long key;
    unsigned int n = 0;
    __device__ float next() {
        unsigned long long z = key + 0x9E3779B97F4A7C15ull * (unsigned long long)(++n);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (float)(z >> 40) * (1.0f / 16777216.0f);
    }
};

// CosineWeightedHemisphereDistribution::sample_ray (CosineWeightedHemisphereDistribution.cpp:7-65)
__device__ void cosine_sample(float z1, float z2, V3<float> up, V3<float>& dir, float& solid_angle) {
    const float pi = 3.14159265358979323846f;
    const float x = cosf(2.0f * pi * z2) * sqrtf(z1), y = sinf(2.0f * pi * z2) * sqrtf(z1), z = sqrtf(1.0f - z1);
    V3<float> t;
    if (fabsf(up.x) > kFltEps) t = v3<float>((-up.y - up.z) / up.x, 1.0f, 1.0f);
    else if (fabsf(up.y) > kFltEps) t = v3<float>(1.0f, (-up.x - up.z) / up.y, 1.0f);
    else t = v3<float>(1.0f, 1.0f, (-up.x - up.y) / up.z);
    const float tl = sqrtf(dot(t, t));
    t = v3<float>(t.x / tl, t.y / tl, t.z / tl);
    V3<float> b = v3<float>(up.y * t.z - up.z * t.y, up.z * t.x - up.x * t.z, up.x * t.y - up.y * t.x);
    const float bl = sqrtf(dot(b, b));
    b = v3<float>(b.x / bl, b.y / bl, b.z / bl);
    dir = v3<float>(t.x * x + b.x * y + up.x * z, t.y * x + b.y * y + up.y * z, t.z * x + b.z * y + up.z * z);
    const float probability = cosf(asinf(sqrtf(z1))) / pi;
    solid_angle = 1.0f / probability;
}

template <typename R>
__global__ void k_render(State<R> s, const uint32_t* __restrict__ cell_start, RenderScene rs, RenderCamera cam,
                         RenderShading sh, float* __restrict__ radiance) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = cam.width, h = cam.height;
    if (px >= w * h) return;
    const int x = px % w, y = px / w;
    PixelRng rng{sh.seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(px + 1))};
    // Camera::generate_ray_for_sample_position (Camera.cpp:10-39); its aspect ratio is width / width
    float rx = ((float)x + 0.5f) / (float)w * 2.0f - 1.0f, ry = ((float)y + 0.5f) / (float)h * 2.0f - 1.0f;
    if (!cam.flip_y) ry = -ry;
    V3<float> pv = v3<float>(rx * cam.tan_half_fov, ry * cam.tan_half_fov, -1.0f);
    const float pl = sqrtf(dot(pv, pv));
    pv = v3<float>(pv.x / pl, pv.y / pl, pv.z / pl);
    V3<float> dir = v3<float>(cam.right[0] * pv.x + cam.up[0] * pv.y + cam.back[0] * pv.z,
                              cam.right[1] * pv.x + cam.up[1] * pv.y + cam.back[1] * pv.z,
                              cam.right[2] * pv.x + cam.up[2] * pv.y + cam.back[2] * pv.z);
    const float dl = sqrtf(dot(dir, dir));
    dir = v3<float>(dir.x / dl, dir.y / dl, dir.z / dl);
    const V3<float> origin = v3<float>(cam.pos[0], cam.pos[1], cam.pos[2]);
    auto bsdf = [&](int type) {
        const float* c = type == 2 ? sh.boundary : sh.fluid;
        return v3<float>(c[0], c[1], c[2]);
    };
    V3<float> sum = v3<float>(0.f, 0.f, 0.f);
    for (int smp = 0; smp < sh.samples; smp++) {
        int type;
        V3<float> p, n;
        float len;
        V3<float> out = v3<float>(0.f, 0.f, 0.f);
        if (!trace_ray<R>(origin, dir, rng.next() * rs.step, s, cell_start, rs, type, p, n, len)) {
            out = sh.normals_only ? v3<float>(-dir.x / 2.0f + 0.5f, -dir.y / 2.0f + 0.5f, -dir.z / 2.0f + 0.5f)
                                  : v3<float>(1.f, 1.f, 1.f);   // the sky
        } else if (sh.normals_only) {
            out = v3<float>(n.x / 2.0f + 0.5f, n.y / 2.0f + 0.5f, n.z / 2.0f + 0.5f);
        } else {
            V3<float> wgt = v3<float>(1.f, 1.f, 1.f);
            for (int depth = 0; depth < sh.max_depth; depth++) {
                if (fabsf(wgt.x) <= kFltEps && fabsf(wgt.y) <= kFltEps && fabsf(wgt.z) <= kFltEps) break;
                const V3<float> f = bsdf(type);
                {   // sample the sky: a cosine-weighted direction, unless occluded
                    V3<float> sd;
                    float sa;
                    const float z1 = rng.next(), z2 = rng.next();
                    cosine_sample(z1, z2, n, sd, sa);
                    int t2;
                    V3<float> p2, n2;
                    float l2;
                    if (!trace_ray<R>(p, sd, rng.next() * rs.step, s, cell_start, rs, t2, p2, n2, l2)) {
                        const float c = sa * fminf(fmaxf(dot(n, sd), 0.0f), 1.0f);
                        out = v3<float>(out.x + c * f.x * wgt.x, out.y + c * f.y * wgt.y, out.z + c * f.z * wgt.z);
                    }
                }
                V3<float> nd;
                float na;
                const float z1 = rng.next(), z2 = rng.next();
                cosine_sample(z1, z2, n, nd, na);
                int t3;
                V3<float> p3, n3;
                float l3;
                if (!trace_ray<R>(p, nd, rng.next() * rs.step, s, cell_start, rs, t3, p3, n3, l3)) break;
                const float c = na * fminf(fmaxf(dot(n, nd), 0.0f), 1.0f);
                wgt = v3<float>(wgt.x * c * f.x, wgt.y * c * f.y, wgt.z * c * f.z);
                type = t3;
                p = p3;
                n = n3;
            }
        }
        sum = v3<float>(sum.x + out.x, sum.y + out.y, sum.z + out.z);
    }
    const float inv = 1.0f / (float)sh.samples;
    radiance[3 * px] = sum.x * inv;
    radiance[3 * px + 1] = sum.y * inv;
    radiance[3 * px + 2] = sum.z * inv;
}

}  // namespace fsb
