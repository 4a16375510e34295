// Neighborhood search: cell keys -> radix sort -> reordering of the particle
// SoA -> per-region cell-start table -> neighbor lists.
//
// One device search serves every reference contract. What the contract fixes
// (and the reference line it follows):
//   predicate   2D: sqrt(dot(d,d)) <= r   (HashedNeighborhoodSearch.cpp:56,
//                    QuadraticNeighborhoodSearchDynamicAllocated.cpp:32,
//                    CompactHashingNeighborhoodSearch.cpp:235)
//               3D: dot(d,d) <= r*r       (HashedNeighborhoodSearch3D.cpp:334,
//                    QuadraticNeighborhoodSearch3D.cpp:60, CompressedNeighbors.cpp:576)
//   owners / candidates: see fs_search_kind in the public header.
// The cell grid (cell edge = search radius, cell = floor(x / r) as in
// HashedNeighborhoodSearch3D.cpp:224-228) is ours; every candidate is tested
// with the contract's exact float predicate, so the neighbor SETS do not
// depend on it.
//
// Layout. Cells are numbered linearly, x fastest, relative to a grid origin
// that follows the particles' bounding box. Sorting by (region, cell) makes
// the three cells x-1, x, x+1 of every (y, z) row one contiguous particle
// range, so a particle's 27 neighbor cells are 9 ranges. Regions keep fluid,
// boundary and listed-inactive particles in separate blocks (one block in the
// reference-order mode). cell_start[g][c] is the first sorted index of region
// g whose cell is >= c (an exclusive scan of the per-cell counts).
//
// Scenes. A context holds one scene or many independent ones (batched mode).
// Every scene has its own grid (SceneGrid: dims, this step's origin, and the
// offset `base` of its cells in the concatenated cell tables), so particles
// of different scenes never share a cell and never meet in a walk.
//
// A grid smaller than the bounding box is clamped: such particles go to border
// cells. Particles in or next to border cells take a slow path that checks
// every candidate's own cell; for all others no check is needed, because a
// clamped particle lies at least two cells away from them (farther than r).
#pragma once

#include "fs_common.cuh"

namespace fsb {

// Sort keys: region (0 fluid, 1 boundary, 2 listed inactive, 3 excluded
// inactive) in the two bits above the linear cell index, which takes
// key_bits bits (the fewest that hold the grid's cells), so the radix sort
// runs over key_bits + 2 bits only.
__host__ __device__ __forceinline__ uint32_t inactive_key(int key_bits) { return 0xffffffffu >> (30 - key_bits); }

// cell coordinate of a position: (int)floor(x / r), or the truncation toward
// zero of HashedNeighborhoodSearch (2D) (HashedNeighborhoodSearch.cpp:108-115)
// when its list order is reproduced
template <typename R> __device__ __forceinline__ int cell_coord(R x, float r, bool trunc) {
    return trunc ? (int)((float)x / r) : (int)floor((float)x / r);
}

// ---------------------------------------------------------------------------
// per-scene bounding box of the cells of the particles in the structure
// ---------------------------------------------------------------------------
// bbox[3 s .. 3 s + 2]: min xyz of scene s; bbox[3 scenes + 3 s ..]: its
// max xyz (two memsets reset the table). scene: per-particle
// scene ids (null: one scene). A block whose particles all belong to one
// scene reduces first and issues one atomic per bound; a mixed block (a scene
// boundary inside it) issues one per particle.
template <typename R>
__global__ void k_bbox(int64_t n, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                       const uint16_t* FSB_R scene, int scenes, bool include_inactive, float r, bool trunc,
                       int* FSB_R bbox) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    const int sk = (k < n && scene) ? scene[k] : 0;
    // one scene: a grid-stride loop (a grid of a few blocks per SM); scenes:
    // one particle per thread
    const int64_t stride = scene ? n : (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = k; i < n; i += stride) {
        if (!include_inactive && type[i] == FS_TYPE_INACTIVE) continue;
        const V4<R> p = pos[i];
        const int c[3] = {cell_coord<R>(p.x, r, trunc), cell_coord<R>(p.y, r, trunc), cell_coord<R>(p.z, r, trunc)};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            mn[a] = min(mn[a], c[a]);
            mx[a] = max(mx[a], c[a]);
        }
    }
    __shared__ int s_first;
    if (threadIdx.x == 0) s_first = sk;
    __syncthreads();
    const int s0 = s_first;
    if (!__syncthreads_and(k >= n || sk == s0)) {
        if (mn[0] != INT_MAX) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                atomicMin(&bbox[3 * sk + a], mn[a]);
                atomicMax(&bbox[3 * scenes + 3 * sk + a], mx[a]);
            }
        }
        return;
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    __shared__ int s_b[6][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            s_b[a][wid] = mn[a];
            s_b[3 + a][wid] = mx[a];
        }
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            int lo = lane < nw ? s_b[a][lane] : INT_MAX, hi = lane < nw ? s_b[3 + a][lane] : INT_MIN;
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (lane == 0) {
                if (lo != INT_MAX) atomicMin(&bbox[3 * s0 + a], lo);
                if (hi != INT_MIN) atomicMax(&bbox[3 * scenes + 3 * s0 + a], hi);
            }
        }
    }
}

// Grid origin of every scene for this step: the bbox minimum, shifted so that
// the box is centred in the scene's dims when it is smaller.
__device__ __forceinline__ void grid_origin_at(int sidx, const int* FSB_R bbox, SceneGrid* FSB_R grids, int scenes) {
    SceneGrid& g = grids[sidx];
    const int d[3] = {g.d0, g.d1, g.d2};
    int o[3];
    for (int a = 0; a < 3; a++) {
        int lo = bbox[3 * sidx + a], hi = bbox[3 * scenes + 3 * sidx + a];
        if (lo > hi) { lo = 0; hi = 0; }
        long long ext = (long long)hi - lo + 1;
        long long slack = (long long)d[a] - ext;
        o[a] = (int)(slack > 0 ? (long long)lo - slack / 2 : (long long)lo);
    }
    g.o0 = o[0];
    g.o1 = o[1];
    g.o2 = o[2];
}
static __global__ void k_origin(const int* FSB_R bbox, SceneGrid* FSB_R grids, int scenes) {
    const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= scenes) return;
    grid_origin_at(sidx, bbox, grids, scenes);
}

// clamped local cell of a cell coordinate; *clamped set when outside the grid
__device__ __forceinline__ int local_cell(int c, int origin, int dim, bool& clamped) {
    long long l = (long long)c - origin;
    if (l < 0) { clamped = true; return 0; }
    if (l >= dim) { clamped = true; return dim - 1; }
    return (int)l;
}

// region of a particle in the sorted layout (0 fluid, 1 boundary, 2 listed inactive)
__device__ __forceinline__ uint32_t region_of(uint8_t t, bool single_region) {
    if (single_region) return 0;
    return t == FS_TYPE_NORMAL ? 0u : (t == FS_TYPE_BOUNDARY ? 1u : 2u);
}

// Sort keys of every particle. keys64 (the reference-order mode) appends a
// 32-bit order within the cell: the host index, or, with the 2D hashed grid's
// history (h2d_cell / h2d_rank per host index, null otherwise), the arrival
// order of HashedNeighborhoodSearch::UpdateGrid (HashedNeighborhoodSearch.cpp:117-151):
// a particle that stays in its cell keeps its rank from the last search, and
// one that arrives goes after every stayer, arrivals by ascending index (the
// reference appends them to the cell's std::list in its i-ascending loop).
template <typename R>
__device__ __forceinline__ void keys_at(int64_t k, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                                        const uint32_t* FSB_R hidx, bool include_inactive, bool single_region,
                                        float r, bool trunc, const SceneGrid* FSB_R grids,
                                        const uint16_t* FSB_R scene, int key_bits, uint32_t* FSB_R keys,
                                        unsigned long long* FSB_R keys64, uint32_t* FSB_R perm,
                                        int2* FSB_R h2d_cell, const uint32_t* FSB_R h2d_rank,
                                        int* FSB_R status) {
    uint8_t t = type[k];
    uint32_t key;
    uint32_t order = keys64 ? hidx[k] : 0u;
    if (!include_inactive && t == FS_TYPE_INACTIVE) {
        key = inactive_key(key_bits);
    } else {
        V4<R> p = pos[k];
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) {
            // a position that is NaN or infinite ends the step with FS_ERR_NAN
            // (and stays out of the cell structure, which the rest of the
            // step then no longer builds on)
            raise_status(status, FS_ERR_NAN);
            p.x = p.y = p.z = R(0);
        }
        const SceneGrid g = grids[scene ? scene[k] : 0];
        bool cl = false;
        const int cx = cell_coord<R>(p.x, r, trunc), cy = cell_coord<R>(p.y, r, trunc);
        int lx = local_cell(cx, g.o0, g.d0, cl);
        int ly = local_cell(cy, g.o1, g.d1, cl);
        int lz = local_cell(cell_coord<R>(p.z, r, trunc), g.o2, g.d2, cl);
        const uint32_t lin = (uint32_t)(g.base + ((int64_t)lz * g.d1 + ly) * g.d0 + lx);
        key = (region_of(t, single_region) << key_bits) | lin;
        if (h2d_cell) {
            const uint32_t h = order;
            const int2 was = h2d_cell[h];
            const uint32_t rank = h2d_rank[h];
            if (rank != 0xffffffffu && was.x == cx && was.y == cy) {
                order = rank;
            } else {
                order = 0x80000000u | h;
                h2d_cell[h] = make_int2(cx, cy);
            }
        }
    }
    if (keys64) keys64[k] = ((unsigned long long)key << 32) | order;
    else keys[k] = key;
    perm[k] = (uint32_t)k;
}
template <typename R>
__global__ void k_keys(int64_t n, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                       const uint32_t* FSB_R hidx, bool include_inactive, bool single_region, float r,
                       bool trunc, const SceneGrid* FSB_R grids, const uint16_t* FSB_R scene,
                       int key_bits, uint32_t* FSB_R keys,
                       unsigned long long* FSB_R keys64, uint32_t* FSB_R perm,
                       int2* FSB_R h2d_cell, const uint32_t* FSB_R h2d_rank,
                       int* FSB_R status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    keys_at<R>(k, pos, type, hidx, include_inactive, single_region, r, trunc, grids, scene, key_bits, keys, keys64,
               perm, h2d_cell, h2d_rank, status);
}

// The 2D hashed grid's history after a sort (see k_keys): every particle's
// rank within its cell of the new sorted order, stored by host index. Ranks
// are relative to the device cell, which may hold several true cells of a
// clamped grid; within each true cell they order its members as the
// reference's list does, which is all the walks need.
// (key_shift: where the cell key starts in the 64-bit sort key)
__device__ __forceinline__ void h2d_rank_at(int64_t k, const unsigned long long* FSB_R keys64, int64_t cells,
                                            int key_bits, const uint32_t* FSB_R cell_start,
                                            const uint32_t* FSB_R hidx, uint32_t* FSB_R h2d_rank,
                                            int key_shift = 32) {
    const uint32_t key = (uint32_t)(keys64[k] >> key_shift);
    const uint32_t first = cell_start[(int64_t)(key >> key_bits) * (cells + 1) + (key & ((1u << key_bits) - 1u))];
    h2d_rank[hidx[k]] = (uint32_t)k - first;
}
static __global__ void k_h2d_rank(int64_t n_struct, const unsigned long long* FSB_R keys64, int64_t cells,
                           int key_bits, const uint32_t* FSB_R cell_start, const uint32_t* FSB_R hidx,
                           uint32_t* FSB_R h2d_rank) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_struct) return;
    h2d_rank_at(k, keys64, cells, key_bits, cell_start, hidx, h2d_rank);
}

// new[k] = old[perm[k]] for every persistent field
template <typename R>
__device__ __forceinline__ void reorder_at(int64_t k, const uint32_t* FSB_R perm, const V4<R>* FSB_R pos0,
                                           V4<R>* FSB_R pos1, const V4<R>* FSB_R vel0, V4<R>* FSB_R vel1,
                                           const V4<R>* FSB_R acc0, V4<R>* FSB_R acc1, const V4<R>* FSB_R ext0,
                                           V4<R>* FSB_R ext1, const R* FSB_R rho0, R* FSB_R rho1,
                                           const R* FSB_R p0, R* FSB_R p1, const uint8_t* FSB_R t0,
                                           uint8_t* FSB_R t1, const uint32_t* FSB_R h0, uint32_t* FSB_R h1,
                                           const uint16_t* FSB_R sc0, uint16_t* FSB_R sc1) {
    const uint32_t s = perm[k];
    pos1[k] = pos0[s];
    vel1[k] = vel0[s];
    acc1[k] = acc0[s];
    ext1[k] = ext0[s];
    rho1[k] = rho0[s];
    p1[k] = p0[s];
    t1[k] = t0[s];
    h1[k] = h0[s];
    if (sc0) sc1[k] = sc0[s];
}
template <typename R>
__global__ void k_reorder(int64_t n, const uint32_t* FSB_R perm, const V4<R>* FSB_R pos0, V4<R>* FSB_R pos1,
                          const V4<R>* FSB_R vel0, V4<R>* FSB_R vel1, const V4<R>* FSB_R acc0,
                          V4<R>* FSB_R acc1, const V4<R>* FSB_R ext0, V4<R>* FSB_R ext1,
                          const R* FSB_R rho0, R* FSB_R rho1, const R* FSB_R p0, R* FSB_R p1,
                          const uint8_t* FSB_R t0, uint8_t* FSB_R t1, const uint32_t* FSB_R h0,
                          uint32_t* FSB_R h1, const uint16_t* FSB_R sc0, uint16_t* FSB_R sc1) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    reorder_at<R>(k, perm, pos0, pos1, vel0, vel1, acc0, acc1, ext0, ext1, rho0, rho1, p0, p1, t0, t1, h0, h1, sc0,
                  sc1);
}

// ---------------------------------------------------------------------------
// candidate walks
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// compact hashing: a hashed cell table for sparse domains
// ---------------------------------------------------------------------------
// CompactHashingNeighborhoodSearch (CompactHashingNeighborhoodSearch.cpp:99-107,
// 342-349) finds a cell's particles through an open-addressing hash table of
// the occupied cells, so memory follows the particles, not the domain's
// extent. Here: particles are sorted by their full (region, cell) key -- no
// dense grid, so no cell is ever clamped however far apart the particles
// lie --, every run of equal keys (one occupied cell of one region) is entered
// into a table of at least twice as many slots as particles, and a walk looks
// each of its cells up by key. The slot of a cell is the spatial hash the
// reference uses (Teschner et al., primes 73856093 and 19349663, here with
// 83492791 for the region) over a power-of-two table, probed linearly.
// Entries are only looked up by their full key, so which slot a cell takes
// (which can depend on the order of concurrent insertions) never changes
// a result.
struct HashCell {
    unsigned long long key;   // kHashEmpty: free slot
    uint32_t start, end;      // the cell's run in the sorted order
};
constexpr unsigned long long kHashEmpty = ~0ull;
constexpr int kHashCoordBits = 31;   // per cell coordinate, biased by 2^30

__device__ __forceinline__ int clamp_cell_coord(int c) { return min(max(c, -(1 << 30)), (1 << 30) - 1); }
// 2 region bits, then the biased x and y cell coordinates (31 bits each)
__device__ __forceinline__ unsigned long long compact_cell_key(uint32_t region, int cx, int cy) {
    const unsigned long long bx = (unsigned long long)(clamp_cell_coord(cx) + (1 << 30));
    const unsigned long long by = (unsigned long long)(clamp_cell_coord(cy) + (1 << 30));
    return ((unsigned long long)region << (2 * kHashCoordBits)) | (bx << kHashCoordBits) | by;
}
__device__ __forceinline__ uint32_t compact_hash(uint32_t region, int cx, int cy, uint32_t mask) {
    return ((uint32_t)clamp_cell_coord(cx) * 73856093u ^ (uint32_t)clamp_cell_coord(cy) * 19349663u ^
            region * 83492791u) & mask;
}
// the run of key in the table, or false; at most mask + 1 probes
__device__ __forceinline__ bool hash_lookup(const HashCell* FSB_R table, uint32_t mask, uint32_t slot,
                                            unsigned long long key, uint32_t& start, uint32_t& end) {
    for (uint32_t probe = 0; probe <= mask; probe++, slot = (slot + 1) & mask) {
        const unsigned long long k = table[slot].key;
        if (k == key) {
            start = table[slot].start;
            end = table[slot].end;
            return true;
        }
        if (k == kHashEmpty) return false;
    }
    return false;
}

// Compact hashing's sort keys (2D): (region, cell x, cell y) of every
// particle in the structure; excluded inactive particles sort last.
template <typename R>
__global__ void k_compact_keys(int64_t n, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                               bool include_inactive, bool single_region, float r,
                               unsigned long long* FSB_R keys, uint32_t* FSB_R perm,
                               int* FSB_R status) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint8_t t = type[k];
    unsigned long long key = kHashEmpty;
    if (include_inactive || t != FS_TYPE_INACTIVE) {
        V4<R> p = pos[k];
        if (!(isfinite(p.x) && isfinite(p.y))) {
            raise_status(status, FS_ERR_NAN);
            p.x = p.y = R(0);
        }
        key = compact_cell_key(region_of(t, single_region), cell_coord<R>(p.x, r, false),
                               cell_coord<R>(p.y, r, false));
    }
    keys[k] = key;
    perm[k] = (uint32_t)k;
}

// Enters every run of equal sorted keys (one occupied cell of one region)
// into the cleared table: the run's first particle probes from the cell's
// hash for a free slot (at most mask + 1 probes; the table has at least
// twice as many slots as particles, so one is always free).
static __global__ void k_hash_insert(int64_t n_struct, const unsigned long long* FSB_R keys,
                              HashCell* FSB_R table, uint32_t mask) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_struct) return;
    const unsigned long long key = keys[k];
    if (k > 0 && keys[k - 1] == key) return;
    int64_t e = k + 1;
    while (e < n_struct && keys[e] == key) e++;
    const uint32_t region = (uint32_t)(key >> (2 * kHashCoordBits));
    const int cx = (int)((key >> kHashCoordBits) & ((1ull << kHashCoordBits) - 1)) - (1 << 30);
    const int cy = (int)(key & ((1ull << kHashCoordBits) - 1)) - (1 << 30);
    uint32_t slot = compact_hash(region, cx, cy, mask);
    for (uint32_t probe = 0; probe <= mask; probe++, slot = (slot + 1) & mask) {
        if (atomicCAS(&table[slot].key, kHashEmpty, key) == kHashEmpty) {
            table[slot].start = (uint32_t)k;
            table[slot].end = (uint32_t)e;
            return;
        }
    }
}

struct WalkParams {
    float r;        // search radius
    float r2;       // r * r
    int dim;        // 2 or 3
    int regions;    // number of regions to visit (1 in single-region mode)
    bool candidates_inactive;  // contract lists inactive neighbors
    bool trunc;                // cells by truncation toward zero (hashed 2D order)
    bool length_test;          // sqrt(dot) <= r instead of dot <= r * r
    const SceneGrid* FSB_R grids;  // per scene
    const uint16_t* FSB_R scene;   // per particle (null: one scene)
    int64_t cells;  // cells of all scenes; each region's table has cells + 1 entries
    const HashCell* table = nullptr;      // compact hashing (2D): cells by key instead of the dense grid
    uint32_t table_mask = 0;
    __device__ __forceinline__ SceneGrid grid_of(int64_t k) const { return grids[scene ? scene[k] : 0]; }
};

// predicate of the contract; d = x_i - x_j. The 2D searches and every
// position query but the compressed one test glm::length(d) <= r
// (HashedNeighborhoodSearch.cpp:56, HashedNeighborhoodSearch3D.cpp:335,
// QuadraticNeighborhoodSearch3D.cpp:212); the 3D index lists and the
// compressed position query test dot(d, d) <= r * r
// (HashedNeighborhoodSearch3D.cpp:173, CompressedNeighbors.cpp:576). In 2D,
// z == 0 adds an exact +0 to the sum.
template <typename R> __device__ __forceinline__ bool within(V3<R> d, const WalkParams& w) {
    const float q = ((float)d.x * (float)d.x + (float)d.y * (float)d.y) + (float)d.z * (float)d.z;
    return w.length_test ? __fsqrt_rn(q) <= w.r : q <= w.r2;
}

// Visits the neighbors of position xi in HashedNeighborhoodSearch3D's order
// (cells dx, dy, dz ascending with dx outermost; within a cell, sorted order).
// f(j, type_j) is called for every neighbor j.
template <typename R, typename F>
__device__ __forceinline__ void walk_cells(V3<R> xi, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                                           const uint32_t* FSB_R cell_start, const SceneGrid& gr,
                                           const WalkParams& w, F&& f) {
    const int ci[3] = {cell_coord<R>(xi.x, w.r, w.trunc), cell_coord<R>(xi.y, w.r, w.trunc), cell_coord<R>(xi.z, w.r, w.trunc)};
    if (w.table) {
        // compact hashing (2D): the 3 x 3 cells looked up by key
        for (int dx = -1; dx <= 1; dx++) {
            for (int dy = -1; dy <= 1; dy++) {
                for (int g = 0; g < w.regions; g++) {
                    uint32_t b, e;
                    if (!hash_lookup(w.table, w.table_mask, compact_hash(g, ci[0] + dx, ci[1] + dy, w.table_mask),
                                     compact_cell_key(g, ci[0] + dx, ci[1] + dy), b, e))
                        continue;
                    for (uint32_t j = b; j < e; j++) {
                        const uint8_t tj = type[j];
                        if (!w.candidates_inactive && tj == FS_TYPE_INACTIVE) continue;
                        if (within<R>(xi - xyz<R>(pos[j]), w)) f(j, tj);
                    }
                }
            }
        }
        return;
    }
    const int zr = w.dim == 2 ? 0 : 1;
    const int o0 = gr.o0, o1 = gr.o1, o2 = gr.o2;
    for (int dx = -1; dx <= 1; dx++) {
        for (int dy = -1; dy <= 1; dy++) {
            for (int dz = -zr; dz <= zr; dz++) {
                const int c0 = ci[0] + dx, c1 = ci[1] + dy, c2 = ci[2] + dz;
                bool cl = false;
                const int l0 = local_cell(c0, o0, gr.d0, cl);
                const int l1 = local_cell(c1, o1, gr.d1, cl);
                const int l2 = local_cell(c2, o2, gr.d2, cl);
                const int64_t lc = gr.base + ((int64_t)l2 * gr.d1 + l1) * gr.d0 + l0;
                for (int g = 0; g < w.regions; g++) {
                    const uint32_t* cs = cell_start + g * (w.cells + 1);
                    const uint32_t b = cs[lc], e = cs[lc + 1];
                    for (uint32_t j = b; j < e; j++) {
                        const V4<R> pj = pos[j];
                        if (cl) {
                            if (cell_coord<R>(pj.x, w.r, w.trunc) != c0 || cell_coord<R>(pj.y, w.r, w.trunc) != c1 ||
                                cell_coord<R>(pj.z, w.r, w.trunc) != c2)
                                continue;
                        }
                        const uint8_t tj = type[j];
                        if (!w.candidates_inactive && tj == FS_TYPE_INACTIVE) continue;
                        const V3<R> d = xi - xyz<R>(pj);
                        if (within<R>(d, w)) f(j, tj);
                    }
                }
            }
        }
    }
}

// Fast walk for the solver lists (3D, fluid and boundary regions, no
// inactive candidates): 9 contiguous row ranges per region. Returns false
// (and visits nothing) for particles in or next to the grid border, which
// take walk_cells instead.
template <typename R, typename F>
__device__ __forceinline__ bool walk_rows(V3<R> xi, const V4<R>* FSB_R pos, const uint32_t* FSB_R cell_start,
                                          const SceneGrid& gr, const WalkParams& w, F&& f) {
    const int lx = cell_coord<R>(xi.x, w.r, false) - gr.o0;
    const int ly = cell_coord<R>(xi.y, w.r, false) - gr.o1;
    const int lz = cell_coord<R>(xi.z, w.r, false) - gr.o2;
    if (lx < 2 || ly < 2 || lz < 2 || lx > gr.d0 - 3 || ly > gr.d1 - 3 || lz > gr.d2 - 3) return false;
    const float r2 = w.r2;
    const float x0 = (float)xi.x, x1 = (float)xi.y, x2 = (float)xi.z;
#pragma unroll 1
    for (int g = 0; g < 2; g++) {
        const uint32_t* cs = cell_start + g * (w.cells + 1);
#pragma unroll 1
        for (int row = 0; row < 9; row++) {
            const int64_t base = gr.base + ((int64_t)(lz + row / 3 - 1) * gr.d1 + (ly + row % 3 - 1)) * gr.d0 + lx;
            const uint32_t b = cs[base - 1], e = cs[base + 2];
            for (uint32_t j = b; j < e; j++) {
                const V4<R> pj = pos[j];
                const float d0 = x0 - (float)pj.x, d1 = x1 - (float)pj.y, d2 = x2 - (float)pj.z;
                const float q2 = (d0 * d0 + d1 * d1) + d2 * d2;
                if (q2 <= r2) f(j, g, q2);
            }
        }
    }
    return true;
}

// One owner's solver list: up to K entries slot-major (nbr[s * stride + k]);
// returns the neighbor count. rows: the 9-row walk where the owner is away
// from the grid border (list order then differs from the reference's).
template <typename R>
__device__ __forceinline__ uint32_t build_list_one(int64_t k, const V4<R>* FSB_R pos,
                                                   const uint8_t* FSB_R type,
                                                   const uint32_t* FSB_R cell_start,
                                                   const WalkParams& w, bool rows,
                                                   uint32_t* FSB_R nbr, int64_t stride, int K) {
    uint32_t c = 0;
    const V3<R> xi = xyz<R>(pos[k]);
    const SceneGrid gr = w.grid_of(k);
    bool done = false;
    if (rows) {
        done = walk_rows<R>(xi, pos, cell_start, gr, w, [&](uint32_t j, int g, float) {
            if ((int)c < K) nbr[(int64_t)c * stride + k] = j | (g == 1 ? kBoundaryBit : 0u);
            c++;
        });
    }
    if (!done) {
        walk_cells<R>(xi, pos, type, cell_start, gr, w, [&](uint32_t j, uint8_t tj) {
            // solver lists never carry inactive particles (the solvers skip them)
            if (tj == FS_TYPE_INACTIVE) return;
            if ((int)c < K) nbr[(int64_t)c * stride + k] = j | (tj == FS_TYPE_BOUNDARY ? kBoundaryBit : 0u);
            c++;
        });
    }
    return c;
}

// capacity status and the warp-aggregated maximum of a list length
__device__ __forceinline__ void note_list_length(uint32_t c, int K, int* FSB_R status,
                                                 StepScalars* FSB_R sc) {
    if ((int)c > K) raise_status(status, FS_ERR_CAPACITY);
    // the maximum over the warp's active lanes (a partial warp at the end of
    // the owners, or of a block-stride loop), issued by its first active lane
    const unsigned act = __activemask();
    const unsigned mx = __reduce_max_sync(act, c);
    if ((threadIdx.x & 31) == __ffs(act) - 1) atomicMax(&sc->max_neighbors, (int)mx);
}

// Solver lists: for owner k in [0, n_owners) with an owner type accepted by
// owner_mask (bit per particle type), write up to K entries slot-major. The
// entry is the sorted index, with kBoundaryBit for boundary neighbors.
template <typename R>
__device__ __forceinline__ void list_owner_at(int64_t k, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                                              const uint32_t* FSB_R cell_start, const WalkParams& w,
                                              uint32_t owner_mask, bool rows, uint32_t* FSB_R nbr, int64_t stride,
                                              int K, uint32_t* FSB_R count, int* FSB_R status,
                                              StepScalars* FSB_R sc) {
    uint32_t c = 0;
    if ((owner_mask >> type[k]) & 1u) c = build_list_one<R>(k, pos, type, cell_start, w, rows, nbr, stride, K);
    count[k] = c;
    note_list_length(c, K, status, sc);
}
template <typename R>
__global__ void __launch_bounds__(128) k_build_lists(int64_t n_owners, const V4<R>* FSB_R pos,
                                                     const uint8_t* FSB_R type,
                                                     const uint32_t* FSB_R cell_start,
                                                     WalkParams w, uint32_t owner_mask,
                                                     bool rows, uint32_t* FSB_R nbr, int64_t stride, int K,
                                                     uint32_t* FSB_R count, int* FSB_R status,
                                                     StepScalars* FSB_R sc) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_owners) return;
    // an overflow elsewhere does not stop the counting: the largest list decides how far the lists grow
    const int err = *status;
    if (err && err != FS_ERR_CAPACITY) return;
    list_owner_at<R>(k, pos, type, cell_start, w, owner_mask, rows, nbr, stride, K, count, status, sc);
}

// Quadratic searches list neighbors by ascending index
// (QuadraticNeighborhoodSearch3D.cpp:52-66); with the reference's summation
// order requested, each solver list is sorted by host index.
__device__ __forceinline__ void sort_list_by_host_at(int64_t k, uint32_t* FSB_R nbr, int64_t stride, int K,
                                                     const uint32_t* FSB_R count, const uint32_t* FSB_R hidx) {
    const int c = min((int)count[k], K);
    for (int a = 1; a < c; a++) {
        const uint32_t e = nbr[(int64_t)a * stride + k];
        const uint32_t h = hidx[e & kIndexMask];
        int b = a - 1;
        while (b >= 0) {
            const uint32_t f = nbr[(int64_t)b * stride + k];
            if (hidx[f & kIndexMask] <= h) break;
            nbr[(int64_t)(b + 1) * stride + k] = f;
            b--;
        }
        nbr[(int64_t)(b + 1) * stride + k] = e;
    }
}
static __global__ void k_sort_lists_by_host(int64_t n_owners, uint32_t* FSB_R nbr, int64_t stride, int K,
                                     const uint32_t* FSB_R count, const uint32_t* FSB_R hidx) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_owners) return;
    sort_list_by_host_at(k, nbr, stride, K, count, hidx);
}

// CSR export: counts (pass 1) and fill (pass 2) in sorted index space
template <typename R>
__global__ void k_csr_count(int64_t n, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                            const uint32_t* FSB_R cell_start, WalkParams w,
                            uint32_t owner_mask, uint32_t* FSB_R count) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t c = 0;
    if ((owner_mask >> type[k]) & 1u)
        walk_cells<R>(xyz<R>(pos[k]), pos, type, cell_start, w.grid_of(k), w, [&](uint32_t, uint8_t) { c++; });
    count[k] = c;
}

template <typename R>
__global__ void k_csr_fill(int64_t n, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                           const uint32_t* FSB_R cell_start, WalkParams w,
                           uint32_t owner_mask, const int64_t* FSB_R offsets, uint32_t* FSB_R out) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!((owner_mask >> type[k]) & 1u)) return;
    int64_t o = offsets[k];
    walk_cells<R>(xyz<R>(pos[k]), pos, type, cell_start, w.grid_of(k), w, [&](uint32_t j, uint8_t) { out[o++] = j; });
}

// neighbors of one arbitrary position (get_neighbors(vec)), sorted space.
// skip_cell_min reproduces HashedNeighborhoodSearch3D's position iterator
// (HashedNeighborhoodSearch3D.cpp:279-344): when it moves on to the next
// cell it sets the cell's set iterator to begin() and then advances it once
// more before testing, so in every cell but the first one visited
// (dx = dy = dz = -1) the member with the smallest particle index is never
// tested. Members are the cell's non-inactive particles
// (HashedNeighborhoodSearch3D.cpp:90-101); the index is the host index.
template <typename R>
__global__ void k_query_position(V3<R> x, const V4<R>* FSB_R pos, const uint8_t* FSB_R type,
                                 const uint32_t* FSB_R hidx, const uint32_t* FSB_R cell_start,
                                 WalkParams w, bool skip_cell_min,
                                 uint32_t* FSB_R out, int64_t cap, unsigned long long* FSB_R count) {
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
                // visits the members of true cell (c0, c1, c2)
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
                if (skip_cell_min && ordinal > 0) {
                    members([&](uint32_t j, const V4<R>&) { skip = min(skip, hidx[j]); });
                }
                members([&](uint32_t j, const V4<R>& pj) {
                    if (hidx[j] == skip) return;
                    if (!within<R>(x - xyz<R>(pj), w)) return;
                    if ((int64_t)c < cap) out[c] = j;
                    c++;
                });
            }
        }
    }
    *count = c;
}

// neighbors of one position over every particle, inactive ones included
// (QuadraticNeighborhoodSearch3D.cpp:199-219,
// QuadraticNeighborhoodSearchDynamicAllocated.cpp:190-225); unordered, the
// host sorts. count must be zero before the launch.
template <typename R>
__global__ void k_query_all(V3<R> x, int64_t n, const V4<R>* FSB_R pos, WalkParams w,
                            uint32_t* FSB_R out, int64_t cap, unsigned long long* FSB_R count) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        if (!within<R>(x - xyz<R>(pos[j]), w)) continue;
        const unsigned long long slot = atomicAdd(count, 1ull);
        if ((int64_t)slot < cap) out[slot] = (uint32_t)j;
    }
}

}  // namespace fsb
