/*
 * TEST INFRASTRUCTURE -- CPU restatement of libFluid's per-timestep hot path
 * (the oracle). Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it, as the checker; the product never links it.
 *
 * Plain C, serial, float arithmetic in the reference's operation order
 * (compile with -O2 -ffp-contract=off so no FMA is formed). Each function
 * names the reference file:line it restates (paths within the FluidSolver
 * repository, src/libFluid/...). Its outputs are pinned bit-for-bit against the
 * reference's own sources compiled in oracle/_ref (tests/golden holds the
 * fixtures generated from them, see tests/golden/make_golden.py).
 *
 * Layout: positions etc. are dense arrays with `dim` floats per particle in
 * input order; types are 0 normal, 1 boundary, 2 inactive (Particle.hpp:7-12).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define T_NORMAL 0
#define T_BOUNDARY 1
#define T_INACTIVE 2

/* ------------------------------------------------------------------------ */
/* vector helpers in glm's scalar order                                      */
/* ------------------------------------------------------------------------ */
typedef struct {
    float x, y, z;
} v3;

static v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 scl(float s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
/* glm::dot: (x*x' + y*y') + z*z'; in 2D z == 0 and the extra +0 is exact */
static float dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

static v3 load(const float* a, int dim, int64_t i) {
    if (!a) return mk(0.f, 0.f, 0.f);
    return dim == 2 ? mk(a[2 * i], a[2 * i + 1], 0.f) : mk(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
}
static void store(float* a, int dim, int64_t i, v3 v) {
    a[dim * i] = v.x;
    a[dim * i + 1] = v.y;
    if (dim == 3) a[3 * i + 2] = v.z;
}

/* ------------------------------------------------------------------------ */
/* cubic spline kernel: CubicSplineKernel.cpp:9-80, CubicSplineKernel3D.cpp:7-71 */
/* ------------------------------------------------------------------------ */
typedef struct {
    float h, alpha;
} kern_t;

static kern_t kern_make(int dim, float support) {
    kern_t k;
    const float pi = 3.14159265358979323846f;
    k.h = support / 2.0f;
    if (dim == 2) k.alpha = 5.0f / (14.0f * pi * (k.h * k.h));
    else k.alpha = 1.0f / (4.0f * pi * ((k.h * k.h) * k.h));
    return k;
}

/* GetKernelValue(x) */
static float kW(const kern_t* k, v3 x) {
    float q = sqrtf(dot3(x, x)) / k->h;
    float ret = 0.0f;
    if (q < 1.0f) {
        float a = 2.0f - q, b = 1.0f - q;
        ret = ((a * a) * a) - 4.0f * ((b * b) * b);
    } else if (q < 2.0f) {
        float a = 2.0f - q;
        ret = (a * a) * a;
    }
    return k->alpha * ret;
}

/* GetKernelDerivativeValue(x): (alpha * (pre * poly)) * -1 */
static v3 kdW(const kern_t* k, v3 x) {
    float len = sqrtf(dot3(x, x));
    float q = len / k->h;
    v3 pre = mk(0.f, 0.f, 0.f);
    if (len > FLT_EPSILON) pre = mk((k->h * x.x) / len, (k->h * x.y) / len, (k->h * x.z) / len);
    v3 ret = mk(0.f, 0.f, 0.f);
    if (q < 1.0f) {
        float a = 2.0f - q, b = 1.0f - q;
        float poly = -3.0f * (a * a) + 12.0f * (b * b);
        ret = mk(pre.x * poly, pre.y * poly, pre.z * poly);
    } else if (q < 2.0f) {
        float a = 2.0f - q;
        float poly = -3.0f * (a * a);
        ret = mk(pre.x * poly, pre.y * poly, pre.z * poly);
    }
    return mk((k->alpha * ret.x) * -1.0f, (k->alpha * ret.y) * -1.0f, (k->alpha * ret.z) * -1.0f);
}

/* GetKernelDerivativeReversedValue(nb, pos) = kdW(pos - nb) * -1 */
static v3 kdWr(const kern_t* k, v3 nb, v3 pos) {
    v3 g = kdW(k, sub(pos, nb));
    return mk(g.x * -1.0f, g.y * -1.0f, g.z * -1.0f);
}

void oracle_kernel_eval(int dim, float support, int64_t n, const float* x, float* W, float* dW) {
    kern_t k = kern_make(dim, support);
    for (int64_t i = 0; i < n; i++) {
        v3 v = load(x, dim, i);
        W[i] = kW(&k, v);
        store(dW, dim, i, kdW(&k, v));
    }
}

/* ConstantTimestepGenerator::get_non_cfl_validating_timestep (ConstantTimestepGenerator.cpp:17-41).
 * sqrt(size / a) is the C double sqrt there; the product with lambda_a is in double. */
float oracle_cfl(float timestep, float lambda_v, float lambda_a, float particle_size, float max_acc, float max_vel) {
    float dta = timestep, dtv = timestep;
    if (max_acc > 0.0f) dta = (float)(sqrt((double)(particle_size / max_acc)) * (double)lambda_a);
    if (max_vel > 0.0f) dtv = particle_size / max_vel * lambda_v;
    float nt = fminf(dta, dtv);
    return fmaxf(nt, 0.000001f);
}

/* DynamicCflTimestepGenerator (DynamicCflTimestepGenerator.cpp:6-61, 82-107):
 * the largest |v| and |a| (glm::length: sqrt of ((x x + y y) + z z) in float)
 * over the particles that are not inactive, then
 *   dt = min_ts, or max(min_ts, min(max_ts, cfl)) when both maxima exceed
 *   FLT_EPSILON, cfl = max(min(sqrt(size / a) lambda_a, size / v lambda_v), 1e-6)
 * with max_ts in place of a bound whose maximum is 0, and sqrt in double as in
 * oracle_cfl. vel, acc: dim floats per particle. */
float oracle_dynamic_timestep(int dim, int64_t n, const float* vel, const float* acc, const uint8_t* type,
                              float particle_size, float min_ts, float max_ts, float lambda_v, float lambda_a) {
    float max_v = 0.0f, max_a = 0.0f;
    for (int64_t i = 0; i < n; i++) {
        if (type[i] == T_INACTIVE) continue;
        const v3 v = load(vel, dim, i), a = load(acc, dim, i);
        const float lv = sqrtf(dot3(v, v)), la = sqrtf(dot3(a, a));
        max_v = fmaxf(max_v, lv);
        max_a = fmaxf(max_a, la);
    }
    float ts = min_ts;
    if (max_v > FLT_EPSILON && max_a > FLT_EPSILON) {
        float dta = max_ts, dtv = max_ts;
        if (max_a > 0.0f) dta = (float)(sqrt((double)(particle_size / max_a)) * (double)lambda_a);
        if (max_v > 0.0f) dtv = particle_size / max_v * lambda_v;
        const float allowed = fmaxf(fminf(dta, dtv), 0.000001f);
        ts = fmaxf(ts, fminf(max_ts, allowed));
    }
    return ts;
}

/* BoundaryPreprocessor::execute_simulation_step (BoundaryPreprocessor.cpp:7-48)
 * on 3D particles with the given neighbor lists (CSR, in the interface's list
 * order; pass the reference's order for bit-identical sums): every boundary
 * particle's mass becomes fmin(rho0 size^3, (rho0 gamma_1) / sum W(x_i - x_b))
 * over its boundary neighbors b, gamma_1 = size^3 * (sum W over the plane x = 0,
 * y, z in -2..2 spacings, y outer) (:104-122). Other masses are copied. */
void oracle_boundary_masses(int64_t n, const float* pos, const float* mass, const uint8_t* type, float particle_size,
                            float rest_density, const int64_t* offsets, const int64_t* idx, float* out) {
    kern_t k = kern_make(3, particle_size * 2.0f);
    float ideal = 0.0f;
    for (int y = -2; y <= 2; y++)
        for (int z = -2; z <= 2; z++)
            ideal += kW(&k, mk(0.0f * particle_size, (float)y * particle_size, (float)z * particle_size));
    const float size3 = (particle_size * particle_size) * particle_size;
    const float gamma_1 = size3 * ideal;
    const float max_mass = rest_density * size3;
    for (int64_t i = 0; i < n; i++) {
        out[i] = mass[i];
        if (type[i] != T_BOUNDARY) continue;
        const v3 xi = load(pos, 3, i);
        float vr = 0.0f;
        for (int64_t q = offsets[i]; q < offsets[i + 1]; q++) {
            const int64_t j = idx[q];
            if (type[j] != T_BOUNDARY) continue;
            vr += kW(&k, sub(xi, load(pos, 3, j)));
        }
        const float corrected = rest_density * gamma_1 / vr;
        out[i] = fminf(max_mass, corrected);
    }
}

/* The global sensors of ParticleStatistics.cpp:17-201, as the reference
 * computes them: serial float sums in collection order, maxima from FLT_MIN,
 * minima from FLT_MAX (MaxMinAvgSensorData), average = sum / count in float.
 * out: density max, min, avg; pressure max, min, avg; |v| max, min, avg;
 * kinetic, potential energy. counts: normal, boundary, inactive. */
void oracle_global_stats(int dim, int64_t n, const float* pos, const float* vel, const float* mass,
                         const float* density, const float* pressure, const uint8_t* type, float gravity,
                         float zero_height, float* out, int64_t* counts) {
    float mx[3] = {FLT_MIN, FLT_MIN, FLT_MIN}, mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, avg[3] = {0.f, 0.f, 0.f};
    float kin = 0.0f, pot = 0.0f;
    int64_t cnt[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; i++) {
        if (type[i] == T_BOUNDARY) { cnt[1]++; continue; }
        if (type[i] == T_INACTIVE) { cnt[2]++; continue; }
        if (type[i] != T_NORMAL) continue;
        cnt[0]++;
        const v3 v = load(vel, dim, i);
        const float speed = sqrtf(dot3(v, v));
        const float vals[3] = {density[i], pressure[i], speed};
        for (int q = 0; q < 3; q++) {
            avg[q] += vals[q];
            mn[q] = vals[q] < mn[q] ? vals[q] : mn[q];   /* std::min(d.minimum, value) */
            mx[q] = mx[q] < vals[q] ? vals[q] : mx[q];   /* std::max(d.maximum, value) */
        }
        const float h = load(pos, dim, i).y - zero_height;
        kin += ((0.5f * mass[i]) * speed) * speed;
        pot += (gravity * mass[i]) * h;
    }
    for (int q = 0; q < 3; q++) {
        if (cnt[0] > 0) avg[q] = avg[q] / (float)cnt[0];
        out[3 * q] = mx[q];
        out[3 * q + 1] = mn[q];
        out[3 * q + 2] = avg[q];
    }
    out[9] = kin;
    out[10] = pot;
    for (int q = 0; q < 3; q++) counts[q] = cnt[q];
}

/* ------------------------------------------------------------------------ */
/* neighborhood search                                                       */
/* ------------------------------------------------------------------------ */
enum {
    NS_QUADRATIC_2D = 0, /* QuadraticNeighborhoodSearchDynamicAllocated.cpp:11-38 */
    NS_HASHED_2D = 1,    /* HashedNeighborhoodSearch.cpp:9-73                     */
    NS_COMPACT_2D = 2,   /* CompactHashingNeighborhoodSearch.cpp:14-84, 210-247   */
    NS_QUADRATIC_3D = 3, /* QuadraticNeighborhoodSearch3D.cpp:32-69               */
    NS_HASHED_3D = 4,    /* HashedNeighborhoodSearch3D.cpp:134-185               */
    NS_COMPRESSED_3D = 5 /* CompressedNeighbors.cpp:536-595                       */
};

static int ns_dim(int kind) { return kind <= NS_COMPACT_2D ? 2 : 3; }

static int ns_owner(int kind, uint8_t t) {
    if (kind == NS_QUADRATIC_2D) return 1;
    if (kind == NS_HASHED_2D) return t == T_NORMAL;
    return t != T_INACTIVE;
}
static int ns_candidate(int kind, uint8_t t) {
    if (kind == NS_QUADRATIC_2D || kind == NS_HASHED_2D) return 1;
    return t != T_INACTIVE;
}

/* the contract's predicate; d = x_i - x_j */
static int ns_within(int dim, v3 d, float r, float r2) {
    if (dim == 2) return sqrtf(d.x * d.x + d.y * d.y) <= r;
    return dot3(d, d) <= r2;
}

/* Candidates sorted by (cell z, y, x, index): a cell's particles are one
 * ascending run found by binary search, for any extent of the domain. */
typedef struct {
    int c[3];
    int64_t i;
    int64_t ord;   /* order within the cell: the index, or the hashed-2d insertion sequence */
} cell_entry;

typedef struct {
    int64_t m;           /* number of candidates */
    cell_entry* e;
} grid_t;

static int cellc(float x, float r) { return (int)floorf(x / r); }
/* HashedNeighborhoodSearch (2D) truncates toward zero (HashedNeighborhoodSearch.cpp:108-115) */
static int g_truncate_cells = 0;
static int cellk(float x, float r) { return g_truncate_cells ? (int)(x / r) : (int)floorf(x / r); }

/* The 2D hashed grid's history (HashedNeighborhoodSearch::UpdateGrid,
 * HashedNeighborhoodSearch.cpp:117-151). Its cells are std::lists that the
 * reference updates incrementally: for i ascending, a particle whose cell
 * changed is removed from the old list and appended to the new one. So the
 * order within a cell is the order of arrival: by the sequence number of
 * the particle's last insertion, which a running counter hands out in that
 * loop. cell[2 i], cell[2 i + 1] hold particle i's current cell (INT32_MAX
 * before the first search, like currentStatus), seq[i] its sequence number;
 * *counter is the next one. Without a history (NULL) the order is the first
 * call's: ascending index. */
typedef struct {
    int32_t* cell;
    int64_t* seq;
    int64_t* counter;
} h2d_history_t;
static h2d_history_t g_h2d = {0, 0, 0};

static int cell_cmp3(const int* a, const int* b) {
    for (int k = 2; k >= 0; k--) {
        if (a[k] < b[k]) return -1;
        if (a[k] > b[k]) return 1;
    }
    return 0;
}
static int entry_cmp(const void* pa, const void* pb) {
    const cell_entry* a = (const cell_entry*)pa;
    const cell_entry* b = (const cell_entry*)pb;
    int c = cell_cmp3(a->c, b->c);
    if (c) return c;
    return a->ord < b->ord ? -1 : (a->ord > b->ord ? 1 : 0);
}

static void grid_build(grid_t* g, int dim, int64_t n, const float* pos, const uint8_t* type, int kind, float r) {
    g->e = (cell_entry*)malloc(sizeof(cell_entry) * (size_t)(n ? n : 1));
    g->m = 0;
    for (int64_t i = 0; i < n; i++) {
        if (!ns_candidate(kind, type ? type[i] : 0)) continue;
        v3 p = load(pos, dim, i);
        cell_entry* e = &g->e[g->m++];
        e->c[0] = cellk(p.x, r);
        e->c[1] = cellk(p.y, r);
        e->c[2] = dim == 3 ? cellk(p.z, r) : 0;
        e->i = i;
        e->ord = i;
        if (kind == NS_HASHED_2D && g_h2d.cell) {
            int32_t* hc = g_h2d.cell + 2 * i;
            if (hc[0] != e->c[0] || hc[1] != e->c[1]) {
                hc[0] = e->c[0];
                hc[1] = e->c[1];
                g_h2d.seq[i] = (*g_h2d.counter)++;
            }
            e->ord = g_h2d.seq[i];
        }
    }
    qsort(g->e, (size_t)g->m, sizeof(cell_entry), entry_cmp);
}

/* first entry of cell c (or m) */
static int64_t grid_lower(const grid_t* g, const int* c) {
    int64_t lo = 0, hi = g->m;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (cell_cmp3(g->e[mid].c, c) < 0) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static void grid_free(grid_t* g) { free(g->e); }

/* Neighbors of particle i in the list order of the contract:
 *   quadratic: ascending index over all particles;
 *   hashed / compact / compressed: cells dx, dy (, dz) ascending with dx
 *   outermost, ascending index within a cell (HashedNeighborhoodSearch3D.cpp:321-341;
 *   HashedNeighborhoodSearch.cpp:33-41 on its first call). Compressed lists are
 *   strictly ascending in the reference's own (re-sorted) index space; their
 *   set is the same. Returns the count; writes up to cap indices. */
static int64_t ns_one(int kind, const grid_t* g, int64_t n, const float* pos, const uint8_t* type, v3 xi, float r,
                      float r2, int64_t* out, int64_t cap) {
    const int dim = ns_dim(kind);
    int64_t c = 0;
    if (kind == NS_QUADRATIC_2D || kind == NS_QUADRATIC_3D) {
        for (int64_t j = 0; j < n; j++) {
            if (!ns_candidate(kind, type ? type[j] : 0)) continue;
            if (ns_within(dim, sub(xi, load(pos, dim, j)), r, r2)) {
                if (c < cap) out[c] = j;
                c++;
            }
        }
        return c;
    }
    int ci[3] = {cellk(xi.x, r), cellk(xi.y, r), dim == 3 ? cellk(xi.z, r) : 0};
    int zr = dim == 3 ? 1 : 0;
    for (int dx = -1; dx <= 1; dx++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dz = -zr; dz <= zr; dz++) {
                int cc[3] = {ci[0] + dx, ci[1] + dy, ci[2] + dz};
                for (int64_t q = grid_lower(g, cc); q < g->m && cell_cmp3(g->e[q].c, cc) == 0; q++) {
                    int64_t j = g->e[q].i;
                    if (ns_within(dim, sub(xi, load(pos, dim, j)), r, r2)) {
                        if (c < cap) out[c] = j;
                        c++;
                    }
                }
            }
    return c;
}

/* Full search: offsets (n+1) and, if idx != NULL, the lists. Returns the
 * total, or -1 when a list exceeds the contract's capacity (97 compressed,
 * 40 compact; the reference throws). */
int64_t oracle_ns(int kind, int64_t n, const float* pos, const uint8_t* type, float radius, int64_t* offsets,
                  int64_t* idx) {
    const int dim = ns_dim(kind);
    const float r2 = radius * radius;
    g_truncate_cells = kind == NS_HASHED_2D;
    grid_t g;
    grid_build(&g, dim, n, pos, type, kind, radius);
    int64_t tot = 0, over = 0;
    const int64_t cap_contract = kind == NS_COMPRESSED_3D ? 97 : (kind == NS_COMPACT_2D ? 40 : 0);
    if (kind == NS_QUADRATIC_2D || kind == NS_QUADRATIC_3D) {
        for (int64_t i = 0; i < n; i++) {
            offsets[i] = tot;
            if (!ns_owner(kind, type ? type[i] : 0)) continue;
            int64_t c = ns_one(kind, &g, n, pos, type, load(pos, dim, i), radius, r2, idx ? idx + tot : NULL,
                               idx ? (int64_t)1 << 62 : 0);
            if (cap_contract && c > cap_contract) over = 1;
            tot += c;
        }
        offsets[n] = tot;
        grid_free(&g);
        return over ? -1 : tot;
    }
    /* cell-ordered searches: the 27 (9 in 2D) neighbor-cell runs are found
     * once per occupied cell; pass 0 counts, pass 1 fills */
    int64_t* count = (int64_t*)calloc((size_t)(n ? n : 1), sizeof(int64_t));
    const int zr = dim == 3 ? 1 : 0;
    for (int pass = 0; pass < (idx ? 2 : 1); pass++) {
        if (pass == 1) {
            int64_t acc = 0;
            for (int64_t i = 0; i < n; i++) {
                offsets[i] = acc;
                acc += count[i];
            }
        }
        int64_t a = 0;
        while (a < g.m) {
            int64_t b = a;
            while (b < g.m && cell_cmp3(g.e[b].c, g.e[a].c) == 0) b++;
            int64_t rs[27], re[27];
            int nr = 0;
            for (int dx = -1; dx <= 1; dx++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dz = -zr; dz <= zr; dz++) {
                        int cc[3] = {g.e[a].c[0] + dx, g.e[a].c[1] + dy, g.e[a].c[2] + dz};
                        int64_t q = grid_lower(&g, cc), e = q;
                        while (e < g.m && cell_cmp3(g.e[e].c, cc) == 0) e++;
                        rs[nr] = q;
                        re[nr++] = e;
                    }
            for (int64_t p = a; p < b; p++) {
                const int64_t i = g.e[p].i;
                if (!ns_owner(kind, type ? type[i] : 0)) continue;
                const v3 xi = load(pos, dim, i);
                int64_t c = 0;
                for (int k = 0; k < nr; k++)
                    for (int64_t q = rs[k]; q < re[k]; q++) {
                        const int64_t j = g.e[q].i;
                        if (ns_within(dim, sub(xi, load(pos, dim, j)), radius, r2)) {
                            if (pass == 1) idx[offsets[i] + c] = j;
                            c++;
                        }
                    }
                count[i] = c;
            }
            a = b;
        }
    }
    for (int64_t i = 0; i < n; i++) {
        if (!idx) offsets[i] = tot;
        if (cap_contract && count[i] > cap_contract) over = 1;
        tot += count[i];
    }
    offsets[n] = tot;
    free(count);
    grid_free(&g);
    return over ? -1 : tot;
}

/* ------------------------------------------------------------------------ */
/* solver state                                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t n;
    int dim;
    float *pos, *vel, *acc, *ext; /* dim per particle */
    float *mass, *density, *pressure;
    uint8_t* type;
    /* IISPH data (IISPHParticleData3D, IISPHFluidSolver3D.hpp:13-19) */
    float *vstar, *anp; /* dim per particle */
    float *source, *diag, *err;
} state_t;

typedef struct {
    int solver;      /* 0 sesph-2d, 1 sesph-3d, 2 iisph-2d, 3 iisph-3d */
    int ns_kind;     /* NS_* above; fixes the list order */
    float rest_density, gravity, particle_size;
    float stiffness, viscosity;
    int single_layer;
    float gamma1, gamma2;
    float max_err;
    int min_it, max_it;
    float omega, gamma;
    float timestep, lambda_v, lambda_a;
} cfg_t;

typedef struct {
    int64_t* off;
    int64_t* idx;
} lists_t;

static lists_t build_lists(const cfg_t* c, const state_t* s) {
    lists_t L;
    L.off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(s->n + 1));
    int64_t tot = oracle_ns(c->ns_kind, s->n, s->pos, s->type, c->particle_size * 2.0f, L.off, NULL);
    if (tot < 0) tot = L.off[s->n];
    L.idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(tot ? tot : 1));
    oracle_ns(c->ns_kind, s->n, s->pos, s->type, c->particle_size * 2.0f, L.off, L.idx);
    return L;
}

#define FOR_NB(L, i, j)                                                        \
    for (int64_t q_ = (L).off[i], j; q_ < (L).off[(i) + 1] && (j = (L).idx[q_], 1); q_++)

/* viscosity (IISPHFluidSolver3D.hpp:43-76 and its copies in the other solvers) */
static v3 viscosity(const cfg_t* c, const kern_t* k, const state_t* s, lists_t L, int64_t i, const float* rho) {
    const int d = s->dim;
    v3 xi = load(s->pos, d, i), vi = load(s->vel, d, i);
    v3 tmp = mk(0.f, 0.f, 0.f);
    FOR_NB(L, i, j) {
        if (s->type[j] == T_INACTIVE) continue;
        v3 xj = load(s->pos, d, j), vj = load(s->vel, d, j);
        float mj = s->mass[j], rj = rho[j];
        if (rj == 0.0f) continue;
        v3 vij = sub(vi, vj), xij = sub(xi, xj);
        float f = (mj / rj) * (dot3(vij, xij) / (dot3(xij, xij) + 0.01f * c->particle_size * c->particle_size));
        tmp = add(tmp, scl(f, kdWr(k, xj, xi)));
    }
    return scl(2.0f * c->viscosity, tmp);
}

/* one IISPH-3D step (IISPHFluidSolver3D.hpp:120-562); returns actual dt */
static float step_iisph3d(const cfg_t* c, state_t* s, float desired, int* iterations, float* avg_out) {
    const int d = 3;
    const int64_t n = s->n;
    kern_t k = kern_make(3, c->particle_size * 2.0f);
    lists_t L = build_lists(c, s);
    float dt = desired;
    const float r2 = c->rest_density * c->rest_density;
    /* L1 (:141-212), serial: density is overwritten while later particles read it */
    for (int64_t i = 0; i < n; i++) {
        uint8_t t = s->type[i];
        if (t == T_INACTIVE) continue;
        s->pressure[i] = 0.0f;
        v3 npa = load(s->ext, d, i);
        if (t != T_BOUNDARY) {
            npa = add(npa, mk(0.0f, -c->gravity, 0.0f));
            npa = add(npa, viscosity(c, &k, s, L, i, s->density));
        }
        v3 vs = add(load(s->vel, d, i), scl(dt, npa));
        store(s->vstar, d, i, vs);
        store(s->anp, d, i, npa);
        store(s->ext, d, i, mk(0.f, 0.f, 0.f));
        if (t == T_BOUNDARY) continue;
        float rho = 0.0f;
        v3 xi = load(s->pos, d, i);
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            if (tj == T_INACTIVE) continue;
            float m = s->mass[j];
            if (c->single_layer && tj == T_BOUNDARY) m *= c->gamma1;
            rho += m * kW(&k, sub(xi, load(s->pos, d, j)));
        }
        s->density[i] = rho;
    }
    /* L2 (:216-339) */
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] != T_NORMAL) continue;
        v3 xi = load(s->pos, d, i), vsi = load(s->vstar, d, i);
        float contrib = 0.0f;
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            v3 g = kdWr(&k, load(s->pos, d, j), xi);
            if (tj == T_NORMAL) contrib += s->mass[j] * dot3(sub(vsi, load(s->vstar, d, j)), g);
            else if (tj == T_BOUNDARY) contrib += s->mass[j] * dot3(vsi, g);
        }
        s->source[i] = c->rest_density - s->density[i] - dt * contrib;
        v3 in = mk(0.f, 0.f, 0.f);
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            v3 g = kdWr(&k, load(s->pos, d, j), xi);
            if (tj == T_NORMAL) in = sub(in, scl(s->mass[j] / r2, g));
            else if (tj == T_BOUNDARY) {
                if (c->single_layer) in = sub(in, scl(2.0f * c->gamma * s->mass[j] / r2, g));
                else in = sub(in, scl(2.0f * s->mass[j] / r2, g));
            }
        }
        float diag = 0.0f;
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            v3 xj = load(s->pos, d, j);
            v3 g = kdWr(&k, xj, xi);
            if (tj == T_NORMAL) {
                diag += s->mass[j] * dot3(in, g);
                diag += s->mass[j] * dot3(scl(s->mass[i] / r2, kdWr(&k, xi, xj)), g);
            } else if (tj == T_BOUNDARY) {
                diag += s->mass[j] * dot3(in, g);
            }
        }
        diag *= dt * dt;
        s->diag[i] = diag;
    }
    /* iterations (:346-523) */
    float max_v2 = 0.0f, max_a2 = 0.0f;
    for (int it = 0; it < c->max_it; it++) {
        for (int64_t i = 0; i < n; i++) {
            if (s->type[i] != T_NORMAL) continue;
            v3 xi = load(s->pos, d, i);
            float pi = s->pressure[i];
            v3 pa = mk(0.f, 0.f, 0.f);
            FOR_NB(L, i, j) {
                uint8_t tj = s->type[j];
                v3 g = kdWr(&k, load(s->pos, d, j), xi);
                if (tj == T_NORMAL) pa = sub(pa, scl(s->mass[j] * (pi / r2 + s->pressure[j] / r2), g));
                else if (tj == T_BOUNDARY) {
                    if (c->single_layer) pa = sub(pa, scl(c->gamma * s->mass[j] * 2.0f * pi / r2, g));
                    else pa = sub(pa, scl(s->mass[j] * 2.0f * pi / r2, g));
                }
            }
            store(s->acc, d, i, pa);
        }
        for (int64_t i = 0; i < n; i++) {
            if (s->type[i] != T_NORMAL) continue;
            v3 xi = load(s->pos, d, i), ai = load(s->acc, d, i);
            float ap = 0.0f;
            FOR_NB(L, i, j) {
                uint8_t tj = s->type[j];
                v3 g = kdWr(&k, load(s->pos, d, j), xi);
                if (tj == T_NORMAL) ap += s->mass[j] * dot3(sub(ai, load(s->acc, d, j)), g);
                else if (tj == T_BOUNDARY) ap += s->mass[j] * dot3(ai, g);
            }
            ap *= dt * dt;
            if (fabsf(s->diag[i]) > FLT_EPSILON)
                s->pressure[i] = fmaxf(0.0f, s->pressure[i] + c->omega * ((s->source[i] - ap) / s->diag[i]));
            else
                s->pressure[i] = 0.0f;
            float e = fabsf(s->source[i] - ap);
            if (fabsf(s->diag[i]) > FLT_EPSILON) {
                if (fabsf(s->pressure[i]) <= FLT_EPSILON) e = 0.0f;
                s->err[i] = e;
            }
        }
        *iterations = it + 1;
        float maxe = 0.0f, avg = 0.0f;
        int64_t cnt = 0;
        max_v2 = 0.0f;
        max_a2 = 0.0f;
        for (int64_t i = 0; i < n; i++) {
            if (s->type[i] != T_NORMAL) continue;
            v3 a = load(s->acc, d, i);
            max_a2 = fmaxf(max_a2, dot3(a, a));
            v3 v = add(load(s->vstar, d, i), scl(dt, a));
            max_v2 = fmaxf(max_v2, dot3(v, v));
            if (fabsf(s->diag[i]) > FLT_EPSILON) {
                maxe = fmaxf(maxe, s->err[i]);
                avg += s->err[i];
                cnt++;
            }
        }
        if (cnt > 0) avg = avg / (float)cnt;
        *avg_out = avg;
        if (c->min_it >= 1 && it >= c->min_it - 1 && avg <= c->max_err) break;
    }
    float old = dt;
    float corrected = oracle_cfl(c->timestep, c->lambda_v, c->lambda_a, c->particle_size, sqrtf(max_a2), sqrtf(max_v2));
    corrected = fminf(corrected, desired);
    dt = corrected;
    /* integration (:539-561) */
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] == T_INACTIVE) continue;
        v3 vs = load(s->vstar, d, i);
        if (old != dt) {
            v3 a = load(s->anp, d, i);
            vs = add(sub(vs, scl(old, a)), scl(dt, a));
        }
        v3 v = add(vs, scl(dt, load(s->acc, d, i)));
        store(s->vel, d, i, v);
        store(s->pos, d, i, add(load(s->pos, d, i), scl(dt, v)));
    }
    free(L.off);
    free(L.idx);
    return dt;
}

/* one SESPH step, 2D (SESPHFluidSolver.hpp:49-111) or 3D (SESPHFluidSolver3D.hpp:49-130) */
static float step_sesph(const cfg_t* c, state_t* s, float desired) {
    const int d = s->dim;
    const int three = d == 3;
    const int64_t n = s->n;
    kern_t k = kern_make(d, c->particle_size * 2.0f);
    lists_t L = build_lists(c, s);
    float dt = desired;
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] != T_NORMAL) continue;
        v3 xi = load(s->pos, d, i);
        float rho = 0.0f;
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            if (tj == T_INACTIVE) continue;
            float w = kW(&k, sub(xi, load(s->pos, d, j)));
            if (three && tj == T_BOUNDARY && c->single_layer) rho += c->gamma1 * s->mass[j] * w;
            else rho += s->mass[j] * w;
        }
        s->density[i] = rho;
        float p = c->stiffness * (rho / c->rest_density - 1.0f);
        s->pressure[i] = p < 0.0f ? 0.0f : p;
    }
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] != T_NORMAL) continue;
        v3 xi = load(s->pos, d, i);
        v3 npa = mk(0.f, 0.f, 0.f);
        npa = add(npa, mk(0.0f, -c->gravity, 0.0f));
        npa = add(npa, viscosity(c, &k, s, L, i, s->density));
        float rho = s->density[i], pr = s->pressure[i], m = s->mass[i];
        float pdd = rho == 0.0f ? 0.0f : pr / (rho * rho);
        v3 pa = mk(0.f, 0.f, 0.f);
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            if (tj == T_INACTIVE) continue;
            v3 g = kdWr(&k, load(s->pos, d, j), xi);
            if (tj == T_BOUNDARY) {
                v3 t = scl(-m * (pdd + pdd), g);
                if (three && c->single_layer) t = mk(t.x * c->gamma2, t.y * c->gamma2, t.z * c->gamma2);
                pa = add(pa, t);
            } else {
                float rj = s->density[j];
                float pddj = rj == 0.0f ? 0.0f : s->pressure[j] / (rj * rj);
                pa = add(pa, scl(-s->mass[j] * (pdd + pddj), g));
            }
        }
        store(s->acc, d, i, add(pa, npa));
    }
    if (three) {
        float ma2 = 0.0f, mv2 = 0.0f;
        for (int64_t i = 0; i < n; i++) {
            v3 a = load(s->acc, d, i);
            ma2 = fmaxf(ma2, dot3(a, a));
            v3 v = add(load(s->vel, d, i), scl(dt, a));
            mv2 = fmaxf(mv2, dot3(v, v));
        }
        float corrected = oracle_cfl(c->timestep, c->lambda_v, c->lambda_a, c->particle_size, sqrtf(ma2), sqrtf(mv2));
        dt = fminf(corrected, desired);
    }
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] == T_INACTIVE) continue;
        v3 v = add(load(s->vel, d, i), scl(dt, load(s->acc, d, i)));
        store(s->vel, d, i, v);
        store(s->pos, d, i, add(load(s->pos, d, i), scl(dt, v)));
    }
    free(L.off);
    free(L.idx);
    return dt;
}

/* one IISPH-2D step (IISPHFluidSolver.hpp:139-525). The reference's
 * convergence test reads `abs(predictedDensityError)`; abs_int selects the
 * integer abs (truncating) when set. */
static float step_iisph2d(const cfg_t* c, state_t* s, float desired, int* iterations, float* avg_out, int abs_int) {
    const int d = 2;
    const int64_t n = s->n;
    kern_t k = kern_make(2, c->particle_size * 2.0f);
    lists_t L = build_lists(c, s);
    const float dt = desired;
    const float r0 = c->rest_density;
    for (int64_t i = 0; i < n; i++) {
        uint8_t t = s->type[i];
        if (t == T_INACTIVE) continue;
        if (t != T_BOUNDARY) {
            v3 xi = load(s->pos, d, i);
            float rho = 0.0f;
            FOR_NB(L, i, j) {
                if (s->type[j] == T_INACTIVE) continue;
                rho += s->mass[j] * kW(&k, sub(xi, load(s->pos, d, j)));
            }
            s->density[i] = rho;
        }
        v3 npa = load(s->ext, d, i);
        if (t != T_BOUNDARY) {
            npa = add(npa, mk(0.0f, -c->gravity, 0.0f));
            npa = add(npa, viscosity(c, &k, s, L, i, s->density));
        }
        store(s->vstar, d, i, add(load(s->vel, d, i), scl(dt, npa)));
        store(s->ext, d, i, mk(0.f, 0.f, 0.f));
    }
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] != T_NORMAL) continue;
        v3 xi = load(s->pos, d, i), vsi = load(s->vstar, d, i);
        float sum = 0.0f;
        FOR_NB(L, i, j) {
            if (s->type[j] == T_INACTIVE) continue;
            sum += s->mass[j] * dot3(sub(vsi, load(s->vstar, d, j)), kdWr(&k, load(s->pos, d, j), xi));
        }
        s->source[i] = r0 - s->density[i] - dt * sum;
        /* the inner sum is the same for every outer neighbor in the reference's
         * O(n^2) loop (:318-350); it is computed once */
        v3 internal = mk(0.f, 0.f, 0.f);
        FOR_NB(L, i, j) {
            uint8_t tj = s->type[j];
            v3 g = kdWr(&k, load(s->pos, d, j), xi);
            if (tj == T_NORMAL) internal = add(internal, scl(s->mass[j] / r0 / r0, g));
            else if (tj == T_BOUNDARY) internal = add(internal, scl(2.0f * c->gamma * s->mass[j] / r0 / r0, g));
        }
        float dsum = 0.0f;
        v3 neg = mk(-internal.x, -internal.y, -internal.z);
        FOR_NB(L, i, j) {
            if (s->type[j] == T_INACTIVE) continue;
            dsum += s->mass[j] * dot3(neg, kdWr(&k, load(s->pos, d, j), xi));
        }
        FOR_NB(L, i, j) {
            if (s->type[j] != T_NORMAL) continue;
            v3 xj = load(s->pos, d, j);
            dsum += s->mass[j] * dot3(scl(s->mass[i] / r0 / r0, kdWr(&k, xi, xj)), kdWr(&k, xj, xi));
        }
        s->diag[i] = dt * dt * dsum;
        s->pressure[i] = 0.0f;
    }
    int it = 0;
    float err = 0.0f;
    while ((it < c->min_it || (abs_int ? (float)abs((int)err) : fabsf(err)) > c->max_err) && it < c->max_it) {
        err = 0.0f;
        int64_t cnt = 0;
        for (int64_t i = 0; i < n; i++) {
            if (s->type[i] != T_NORMAL) continue;
            v3 xi = load(s->pos, d, i);
            float pi = s->pressure[i];
            v3 sum = mk(0.f, 0.f, 0.f);
            FOR_NB(L, i, j) {
                uint8_t tj = s->type[j];
                v3 g = kdWr(&k, load(s->pos, d, j), xi);
                if (tj == T_NORMAL) sum = add(sum, scl(s->mass[j] * (pi / r0 / r0 + s->pressure[j] / r0 / r0), g));
                else if (tj == T_BOUNDARY) sum = add(sum, scl(c->gamma * s->mass[j] * 2.0f * (pi / r0 / r0), g));
            }
            store(s->acc, d, i, mk(-sum.x, -sum.y, -sum.z));
        }
        for (int64_t i = 0; i < n; i++) {
            if (s->type[i] != T_NORMAL) continue;
            v3 xi = load(s->pos, d, i), ai = load(s->acc, d, i);
            float sum = 0.0f;
            FOR_NB(L, i, j) {
                uint8_t tj = s->type[j];
                v3 g = kdWr(&k, load(s->pos, d, j), xi);
                if (tj == T_NORMAL) sum += s->mass[j] * dot3(sub(ai, load(s->acc, d, j)), g);
                else if (tj == T_BOUNDARY) sum += s->mass[j] * dot3(ai, g);
            }
            float Ap = dt * dt * sum;
            float aii = s->diag[i], src = s->source[i];
            if (fabsf(aii) > FLT_EPSILON) s->pressure[i] = fmaxf(0.0f, s->pressure[i] + c->omega * ((src - Ap) / aii));
            else s->pressure[i] = 0.0f;
            float e = fabsf(src - Ap);
            if (fabsf(aii) > FLT_EPSILON) {
                if (fabsf(s->pressure[i]) <= FLT_EPSILON) e = 0.0f;
                err += e;
                cnt++;
            }
        }
        err = cnt != 0 ? err / (float)cnt : 0.0f;
        it++;
    }
    *iterations = it;
    *avg_out = err;
    for (int64_t i = 0; i < n; i++) {
        if (s->type[i] == T_INACTIVE) continue;
        v3 v = add(load(s->vstar, d, i), scl(dt, load(s->acc, d, i)));
        store(s->vel, d, i, v);
        store(s->pos, d, i, add(load(s->pos, d, i), scl(dt, v)));
    }
    free(L.off);
    free(L.idx);
    return dt;
}

/* Runs `steps` steps of solver c on the state arrays in place (input order;
 * vstar/anp: dim floats per particle, source/diag/err one float; any of the
 * IISPH arrays may be NULL). stats receives per step
 * {desired dt, actual dt, iterations, avg density error}. h2d_cell / h2d_seq /
 * h2d_counter: the 2D hashed grid's history (h2d_history_t), kept by the
 * caller across calls like the reference's search object keeps its grid
 * across steps; NULL for a fresh grid at every step. */
int oracle_run(const float* cfg, int64_t n, int dim, float* pos, float* vel, float* acc, float* ext, float* mass,
               float* density, float* pressure, uint8_t* type, float* vstar, float* anp, float* source, float* diag,
               float* err, int steps, float* stats, int abs_int, int32_t* h2d_cell, int64_t* h2d_seq,
               int64_t* h2d_counter) {
    cfg_t c;
    c.solver = (int)cfg[0];
    c.ns_kind = (int)cfg[1];
    c.rest_density = cfg[2];
    c.gravity = cfg[3];
    c.particle_size = cfg[4];
    c.stiffness = cfg[5];
    c.viscosity = cfg[6];
    c.single_layer = cfg[7] != 0.0f;
    c.gamma1 = cfg[8];
    c.gamma2 = cfg[9];
    c.max_err = cfg[10];
    c.min_it = (int)cfg[11];
    c.max_it = (int)cfg[12];
    c.omega = cfg[13];
    c.gamma = cfg[14];
    c.timestep = cfg[15];
    c.lambda_v = cfg[16];
    c.lambda_a = cfg[17];
    state_t s;
    s.n = n;
    s.dim = dim;
    s.pos = pos;
    s.vel = vel;
    s.acc = acc;
    s.ext = ext;
    s.mass = mass;
    s.density = density;
    s.pressure = pressure;
    s.type = type;
    float* own[5] = {0};
    s.vstar = vstar ? vstar : (own[0] = (float*)calloc((size_t)n * dim, sizeof(float)));
    s.anp = anp ? anp : (own[1] = (float*)calloc((size_t)n * dim, sizeof(float)));
    s.source = source ? source : (own[2] = (float*)calloc((size_t)n, sizeof(float)));
    s.diag = diag ? diag : (own[3] = (float*)calloc((size_t)n, sizeof(float)));
    s.err = err ? err : (own[4] = (float*)calloc((size_t)n, sizeof(float)));
    g_h2d.cell = h2d_cell;
    g_h2d.seq = h2d_seq;
    g_h2d.counter = h2d_counter;
    for (int st = 0; st < steps; st++) {
        int its = 0;
        float avg = 0.0f, dt = 0.0f;
        const float desired = c.timestep;
        switch (c.solver) {
            case 0:
            case 1: dt = step_sesph(&c, &s, desired); break;
            case 2: dt = step_iisph2d(&c, &s, desired, &its, &avg, abs_int); break;
            case 3: dt = step_iisph3d(&c, &s, desired, &its, &avg); break;
            default: return -1;
        }
        if (stats) {
            stats[4 * st + 0] = desired;
            stats[4 * st + 1] = dt;
            stats[4 * st + 2] = (float)its;
            stats[4 * st + 3] = avg;
        }
    }
    for (int q = 0; q < 5; q++) free(own[q]);
    g_h2d.cell = 0;
    g_h2d.seq = 0;
    g_h2d.counter = 0;
    return 0;
}
