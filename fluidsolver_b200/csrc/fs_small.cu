// The small-scene step kernel (fs_small.cuh): search and solver phases of
// whole steps in one thread-block cluster, in the order of the step-by-step
// path (fs_api.cu: search_impl, begin_solver_phases, step_sesph,
// step_iisph3d, step_iisph2d), each phase a loop over the particles that
// calls the same per-particle device function as the separate kernel does.
#define FSB_COHERENT_LOADS 1

#include <algorithm>
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

// The launch is one cluster of CTAs (1 to kSmallMaxCtas, one per SM). The
// per-particle phases are loops over each CTA's share of the particles; the
// per-step scalars and the convergence test are thread 0 of CTA 0's, the
// sort and the cell table are the cluster's (sort_small_cluster, the
// binary-searched table). Phases are separated by the cluster
// barrier, whose arrive releases and whose wait acquires at cluster scope:
// what one CTA wrote to global memory before the barrier is what every CTA
// reads after it (this translation unit loads through coherent paths only).
// Every thread of every CTA reaches every barrier: the branches around them
// test launch parameters or a decision CTA 0 published (publish_decision).
// A loop over m items gives each CTA one contiguous share of ceil(m / size)
// items (about kSmallPerCta particles), walked by its threads:
//   for (int64_t k = T.first(m); k < T.end(m); k += kSmallThreads)
struct Team {
    uint32_t rank, size;   // this CTA's rank in the cluster, the cluster's CTAs
    __device__ __forceinline__ int64_t share(int64_t m) const { return (m + size - 1) / size; }
    __device__ __forceinline__ int64_t first(int64_t m) const {
        return min(m, (int64_t)rank * share(m)) + threadIdx.x;
    }
    __device__ __forceinline__ int64_t end(int64_t m) const { return min(m, (int64_t)(rank + 1) * share(m)); }
};
__device__ __forceinline__ Team team() {
    Team T;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(T.rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(T.size));
    return T;
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the address of a shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_store(uint32_t addr, int v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ int cluster_load(uint32_t addr) {
    int v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}
// A decision every CTA must take alike (leaving the pressure loop): thread 0
// of CTA 0 computes it and stores it in CTA 0's shared memory, a cluster
// barrier follows, and every thread reads it. The next store comes after at
// least one more barrier, which every thread reaches only after its read.
__device__ __forceinline__ bool publish_decision(const Team& T, int* slot, bool v) {
    if (T.rank == 0 && threadIdx.x == 0) *slot = v;
    cluster_sync();
    return cluster_load(cluster_addr(slot, 0)) != 0;
}

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

// The fields a phase gathers from neighbors, copied into every CTA's shared
// memory (SmallStepArgs::stage): the positions once per step, after the
// search (they stay fixed until the integration), and before a phase the
// fields it reads of its neighbors but does not write. The phase then runs
// the same per-particle function on a State whose pointers for those fields
// are the copies (generic addresses; the loads of this translation unit are
// plain loads), so every value is the same and only its latency changes.
template <typename R> struct SmallStage {
    V4<R>* pos;
    V4<R>* f4;
    R *f1, *f2;
    uint32_t *nbr, *cnt;   // this CTA's owners' lists (slot-major, stride: its share) and counts
};
template <typename R> __device__ __forceinline__ SmallStage<R> small_stage(unsigned char* smem, int64_t n,
                                                                          int64_t share) {
    const int64_t np = (n + 3) & ~int64_t(3);
    SmallStage<R> g;
    g.pos = reinterpret_cast<V4<R>*>(smem);
    g.f4 = g.pos + np;
    g.f1 = reinterpret_cast<R*>(g.f4 + np);
    g.f2 = g.f1 + np;
    g.cnt = reinterpret_cast<uint32_t*>(g.f2 + np);
    g.nbr = g.cnt + share;
    return g;
}
// m elements of src into this CTA's copy dst, eight loads in flight per
// thread before their stores (a load and its store per iteration would wait
// out one memory latency per element); every thread of the CTA calls it, and
// a block barrier follows
template <typename T> __device__ __noinline__ void stage_field(T* dst, const T* src, int64_t m) {
    constexpr int U = 8;
    for (int64_t b = threadIdx.x; b < m; b += U * kSmallThreads) {
        T v[U];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (b + u * kSmallThreads < m) v[u] = src[b + u * kSmallThreads];
#pragma unroll
        for (int u = 0; u < U; u++)
            if (b + u * kSmallThreads < m) dst[b + u * kSmallThreads] = v[u];
    }
    __syncthreads();
}

__device__ __forceinline__ unsigned long long cluster_load64(uint32_t addr) {
    unsigned long long v;
    asm volatile("ld.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
    return v;
}

// The stable sort of n <= kSmallMax (key, value) pairs by the low `bits`
// bits of the key, rounded up to whole bytes (what sort_small_block gives;
// at most 40 bits), by the whole cluster, in two
// phases. (1) Each CTA sorts its share of the pairs in shared memory as
// unique 64-bit words (masked key << 12 | index: equal keys keep their index
// order, which is what makes the result that of a stable sort): each word
// goes to the place given by the number of the share's words below it (a
// bitonic network for shares above 2 kSmallThreads words, which only a
// device that schedules no large cluster gives). (2) After a cluster
// barrier each CTA copies every CTA's
// sorted run out of that CTA's shared memory (distributed shared memory);
// a word's place in the output is the sum over the runs of the number of
// words below it, found by binary searches that step through all runs
// together. Every thread of every CTA calls it; a cluster barrier follows.
// smem: 2 kSmallMax words.
template <typename K>
__device__ __noinline__ void sort_small_cluster(const Team& T, int64_t n, int bits, const K* kin,
                                                   const uint32_t* vin, K* kout, uint32_t* vout, unsigned char* smem) {
    static_assert(kSmallMax <= 4096, "the index field of the sort words has 12 bits");
    unsigned long long* run = reinterpret_cast<unsigned long long*>(smem);
    unsigned long long* all = run + kSmallMax;
    const uint32_t t = threadIdx.x, N = (uint32_t)n;   // n <= kSmallMax: 32-bit indices throughout
    const uint32_t share = (uint32_t)T.share(n), lo = min(N, T.rank * share), m = (uint32_t)T.end(n) - lo;
    // the radix passes' whole 8-bit digits: the key bits sort_small_block orders by
    const int rbits = (bits + 7) / 8 * 8;
    const K kmask = rbits >= (int)(8 * sizeof(K)) ? ~K(0) : (K(1) << rbits) - K(1);
    auto word = [&](uint32_t i) { return ((unsigned long long)(kin[lo + i] & kmask) << 12) | (unsigned long long)(lo + i); };
    if (m <= 2 * kSmallThreads) {
        // the share's words, each placed by the number of words below it
        // (every thread reads the same word at a time: a broadcast)
        for (uint32_t i = t; i < m; i += kSmallThreads) all[i] = word(i);
        __syncthreads();
        for (uint32_t i = t; i < m; i += kSmallThreads) {
            const unsigned long long v = all[i];
            uint32_t c = 0;
#pragma unroll 8
            for (uint32_t q = 0; q < m; q++) c += all[q] < v ? 1u : 0u;
            run[c] = v;
        }
    } else {
        // a larger share (a device that schedules only small clusters): bitonic network
        uint32_t P = 1;
        while (P < m) P <<= 1;
        for (uint32_t i = t; i < P; i += kSmallThreads) run[i] = i < m ? word(i) : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = t; i < P; i += kSmallThreads) {
                    const uint32_t x = i ^ j;
                    if (x > i) {
                        const unsigned long long u = run[i], w = run[x];
                        if ((u > w) == ((i & k) == 0)) {
                            run[i] = w;
                            run[x] = u;
                        }
                    }
                }
                __syncthreads();
            }
        }
    }
    cluster_sync();
    // run q: words [base[q], base[q] + len[q]) of `all`, in every CTA
    uint32_t base[kSmallMaxCtas], len[kSmallMaxCtas];
#pragma unroll
    for (int q = 0; q < kSmallMaxCtas; q++) {
        base[q] = min(N, (uint32_t)q * share);
        len[q] = (q < (int)T.size ? min(N, (uint32_t)(q + 1) * share) : base[q]) - base[q];
    }
    // every run's element j at once (their remote loads in flight together)
    for (uint32_t j0 = 0; j0 < share; j0 += kSmallThreads) {
        const uint32_t j = j0 + t;
        unsigned long long v[kSmallMaxCtas];
#pragma unroll
        for (int q = 0; q < kSmallMaxCtas; q++)
            if (j < len[q]) v[q] = cluster_load64(cluster_addr(run + j, q));
#pragma unroll
        for (int q = 0; q < kSmallMaxCtas; q++)
            if (j < len[q]) all[base[q] + j] = v[q];
    }
    __syncthreads();
    uint32_t top = 1;   // the largest power of two <= share
    while (top * 2 <= share) top <<= 1;
    for (uint32_t i = t; i < m; i += kSmallThreads) {
        const unsigned long long v = run[i];
        // The input is the last step's sorted order, so a block's share
        // mostly spans its own range of cells: against most runs a word lies
        // below the first or above the last word, and only the runs it
        // falls inside take a binary search.
        uint32_t rank = 0;
#pragma unroll 1
        for (int q = 0; q < (int)T.size; q++) {
            const uint32_t b = min(N, (uint32_t)q * share), l = min(N, (uint32_t)(q + 1) * share) - b;
            if (l == 0 || v < all[b]) continue;
            if (v > all[b + l - 1]) {
                rank += l;
                continue;
            }
            uint32_t pos = 0;
            for (uint32_t step = top; step > 0; step >>= 1) {
                const uint32_t p = pos + step;
                if (p <= l && all[b + p - 1] < v) pos = p;
            }
            rank += pos;
        }
        const uint32_t k = (uint32_t)(v & 0xfffu);
        kout[rank] = kin[k];
        vout[rank] = vin[k];
    }
    cluster_sync();
}

// a float4 field and two scalar fields at once (the SESPH forces' gather)
template <typename R>
__device__ __noinline__ void stage_fields3(V4<R>* d4, const V4<R>* s4, R* d1, const R* s1, R* d2, const R* s2,
                                           int64_t m) {
    constexpr int U = 4;
    for (int64_t b = threadIdx.x; b < m; b += U * kSmallThreads) {
        V4<R> v[U];
        R x[U], y[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t i = b + u * kSmallThreads;
            if (i < m) {
                v[u] = s4[i];
                x[u] = s1[i];
                y[u] = s2[i];
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t i = b + u * kSmallThreads;
            if (i < m) {
                d4[i] = v[u];
                d1[i] = x[u];
                d2[i] = y[u];
            }
        }
    }
    __syncthreads();
}

// the search of one step (search_impl); returns the buffer set now current
template <typename R>
__device__ __forceinline__ int small_search(const SmallStepArgs<R>& a, const Team& T, int cur, R* const (&rho)[2],
                                            unsigned char* smem) {
    const int t = threadIdx.x;
    const int64_t n = a.n;
    __shared__ SceneGrid s_grid;   // this step's grid (scene 0), as every CTA computes it
    {
        // bounding box of the cells (k_bbox; the bounds start from the
        // table's reset pattern) and the grid origin (k_origin)
        const V4<R>* pos = (const V4<R>*)a.buf[cur].pos;
        const uint8_t* type = a.buf[cur].type;
        int mn[3] = {0x7f7f7f7f, 0x7f7f7f7f, 0x7f7f7f7f};
        int mx[3] = {(int)0x80808080, (int)0x80808080, (int)0x80808080};
        for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads) {
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
        // This CTA's bounds, in its shared memory; after a cluster barrier
        // every CTA combines all CTAs' bounds (distributed shared memory) into
        // its own copy of the grid, which its phases of this step read, and
        // CTA 0 stores the bounds and the grid for the context.
        __shared__ int s_part[6];
        if (t == 0) s_grid = a.grids[0];   // the dims and base (the origin follows)
        if (t < 32) {
#pragma unroll
            for (int d = 0; d < 6; d++) {
                const bool in = t < kSmallThreads / 32;
                const int v = d < 3 ? __reduce_min_sync(0xffffffffu, in ? s_b[d][t] : INT_MAX)
                                    : __reduce_max_sync(0xffffffffu, in ? s_b[d][t] : INT_MIN);
                if (t == 0) s_part[d] = v;
            }
        }
        cluster_sync();
        if (t < 32) {
            __shared__ int s_box[6];
            const bool in = t < (int)T.size;
#pragma unroll
            for (int d = 0; d < 6; d++) {
                const int v = in ? cluster_load(cluster_addr(&s_part[d], t)) : (d < 3 ? INT_MAX : INT_MIN);
                const int b = d < 3 ? __reduce_min_sync(0xffffffffu, v) : __reduce_max_sync(0xffffffffu, v);
                if (t == 0) s_box[d] = b;
            }
            if (t == 0) {
                grid_origin_at(0, s_box, &s_grid, 1);
                if (T.rank == 0) {
                    for (int d = 0; d < 6; d++) a.bbox[d] = s_box[d];
                    a.grids[0] = s_grid;
                }
            }
        }
        __syncthreads();
    }
    // Keys (k_keys). The reference-order keys carry the order inside a cell
    // in their low 32 bits: a host index or a rank below kSmallMax, or an
    // arrival flagged by the top bit. Below kSmallMax particles it fits
    // kOrderBits bits with the flag moved down, which keeps every comparison
    // and keeps the sort words within 64 bits; each thread compresses the
    // keys it has just written.
    const bool k64 = a.keys64[0] != nullptr;
    constexpr int kOrderBits = 14;
    static_assert(kSmallMax <= (1 << (kOrderBits - 1)), "the order field's values must fit below its flag bit");
    for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads) {
        keys_at<R>(k, (const V4<R>*)a.buf[cur].pos, a.buf[cur].type, a.buf[cur].hidx, a.include_inactive,
                   a.single_region, a.radius, a.trunc, &s_grid, nullptr, a.key_bits, a.keys[0], a.keys64[0],
                   a.perm[0], a.h2d_cell, a.h2d_rank, a.status);
        if (k64) {
            const unsigned long long x = a.keys64[0][k];
            const uint32_t order = (uint32_t)x;
            const uint32_t o = (order & 0x80000000u) ? (1u << (kOrderBits - 1)) | (order & 0x7fffffffu) : order;
            a.keys64[0][k] = ((x >> 32) << kOrderBits) | o;
        }
    }
    cluster_sync();
    // stable sort of (key, index) (sort_pairs), by the cluster
    const int res = n > 1 ? 1 : 0;
    if (n > 1) {
        if (k64)
            sort_small_cluster<unsigned long long>(T, n, kOrderBits + a.key_bits + 2, a.keys64[0], a.perm[0],
                                                   a.keys64[1], a.perm[1], smem);
        else
            sort_small_cluster<uint32_t>(T, n, a.key_bits + 2, a.keys[0], a.perm[0], a.keys[1], a.perm[1], smem);
    }
    // gather every persistent field into the other buffer set (k_reorder)
    const int nx = cur ^ 1;
    {
        const SmallBuffers &f = a.buf[cur], &g = a.buf[nx];
        for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads)
            reorder_at<R>(k, a.perm[res], (const V4<R>*)f.pos, (V4<R>*)g.pos, (const V4<R>*)f.vel, (V4<R>*)g.vel,
                          (const V4<R>*)f.acc, (V4<R>*)g.acc, (const V4<R>*)f.ext, (V4<R>*)g.ext, rho[cur], rho[nx],
                          (const R*)f.p, (R*)g.p, f.type, g.type, f.hidx, g.hidx, nullptr, nullptr);
    }
    // (no barrier: the cell table below needs only the sorted keys; the
    // barrier after it publishes both)
    cur = nx;
    // Cell-start table (cell_start_table: zeroed run counts, scanned in
    // place): entry t, for region g and cell c at t = g (cells + 1) + c, is the
    // first sorted index whose key's entry is >= t. Every CTA copies the
    // sorted keys' entries into its shared memory and finds those of its
    // share of the table by binary search: the scan's values in one phase.
    const int64_t table = (int64_t)a.regions * (a.cells + 1);
    {
        const int64_t ns = a.n_struct;
        int64_t* te = reinterpret_cast<int64_t*>(smem);   // kSmallMax entries fit every launch's shared memory
        const uint32_t mask = (1u << a.key_bits) - 1u;
        constexpr int U = 8;   // keys loaded in flight per thread
        for (int64_t b = threadIdx.x; b < ns; b += U * kSmallThreads) {
            uint32_t key[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int64_t k = b + u * kSmallThreads;
                if (k < ns) key[u] = k64 ? (uint32_t)(a.keys64[res][k] >> kOrderBits) : a.keys[res][k];
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int64_t k = b + u * kSmallThreads;
                if (k < ns) te[k] = (int64_t)(key[u] >> a.key_bits) * (a.cells + 1) + (key[u] & mask);
            }
        }
        __syncthreads();
        for (int64_t i = T.first(table); i < T.end(table); i += kSmallThreads) {
            int64_t lo = 0, hi = ns;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (te[mid] < i) lo = mid + 1;
                else hi = mid;
            }
            a.cell_start[i] = (uint32_t)lo;
        }
    }
    cluster_sync();
    if (a.h2d_cell) {
        for (int64_t k = T.first(a.n_struct); k < T.end(a.n_struct); k += kSmallThreads)
            h2d_rank_at(k, a.keys64[res], a.cells, a.key_bits, a.cell_start, a.buf[cur].hidx, a.h2d_rank, kOrderBits);
        cluster_sync();
    }
    // solver lists (k_build_lists; an overflow elsewhere does not stop the counting)
    {
        WalkParams w;
        w.r = a.radius;
        w.r2 = a.radius2;
        w.dim = a.dim;
        w.regions = (int)min(a.regions, 2);   // solver lists never hold inactive particles (search_impl's walk)
        w.candidates_inactive = false;
        w.trunc = a.trunc;
        w.length_test = a.dim == 2;
        w.grids = &s_grid;
        w.scene = nullptr;
        w.cells = a.cells;
        const int64_t no = a.n_owners, share = T.share(no), lo = min(no, (int64_t)T.rank * share);
        const SmallStage<R> g = small_stage<R>(smem, n, share);
        const V4<R>* pos = (const V4<R>*)a.buf[cur].pos;
        const uint8_t* type = a.buf[cur].type;
        const uint32_t* cs = a.cell_start;
        if (a.stage) {
            stage_field(g.pos, pos, n);
            pos = g.pos;
            // the cell table and the types, in the space the later phases' fields take
            const int64_t np = (n + 3) & ~int64_t(3);
            if (table * 4 + n <= np * (int64_t)(sizeof(V4<R>) + 2 * sizeof(R))) {
                uint32_t* st = reinterpret_cast<uint32_t*>(g.f4);
                uint8_t* sy = reinterpret_cast<uint8_t*>(st + table);
                stage_field(st, cs, table);
                stage_field(sy, type, n);
                cs = st;
                type = sy;
            }
        }
        // with staged lists: written into this CTA's copy (which the solver
        // phases read), then stored to the context's lists
        uint32_t* nbr = a.stage_lists ? g.nbr - lo : a.nbr;
        uint32_t* cnt = a.stage_lists ? g.cnt - lo : a.count;
        const int64_t stride = a.stage_lists ? share : a.stride;
        const int err = status_now(a.status);
        if (!err || err == FS_ERR_CAPACITY)
            for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads)
                list_owner_at<R>(k, pos, type, cs, w, a.owner_mask, a.rows, nbr, stride, a.K, cnt, a.status, a.sc);
        if (!a.stage_lists) cluster_sync();
        if (a.sort_by_host) {
            // the host indices the insertion sorts compare, staged over the
            // cell table (which the walk no longer needs)
            const uint32_t* hidx = a.buf[cur].hidx;
            if (a.stage) {
                __syncthreads();
                uint32_t* sh = reinterpret_cast<uint32_t*>(g.f4);
                stage_field(sh, hidx, n);
                hidx = sh;
            } else if (a.stage_lists) {
                __syncthreads();
            }
            for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads)
                sort_list_by_host_at(k, nbr, stride, a.K, cnt, hidx);
            if (!a.stage_lists) cluster_sync();
        }
        if (a.stage_lists) {
            // each thread stores its owners' entries (a row of the slot-major
            // lists at a time across the threads)
            __syncthreads();
            const int64_t m = T.end(no) - lo;
            for (int64_t i = threadIdx.x; i < m; i += kSmallThreads) {
                const uint32_t c = min(g.cnt[i], (uint32_t)a.K);
                a.count[lo + i] = g.cnt[i];
                for (uint32_t q = 0; q < c; q++) a.nbr[(int64_t)q * a.stride + lo + i] = g.nbr[(int64_t)q * share + i];
            }
            cluster_sync();
        }
    }
    return cur;
}

// the per-step scalars (k_step_begin) and, with the dynamic generator, the
// time step from the state (begin_solver_phases)
template <typename R>
__device__ __forceinline__ void small_begin_solver(const SmallStepArgs<R>& a, const Team& T, const State<R>& s,
                                                   bool next_reads_no_scalar) {
    const int t = threadIdx.x;
    if (T.rank == 0 && t == 0) {
        StepScalars z{};
        z.desired_dt = a.desired_dt;
        z.dt = a.desired_dt;
        z.max_neighbors = ((const volatile StepScalars*)a.sc)->max_neighbors;
        *a.sc = z;
    }
    // a next phase that touches no scalar (the SESPH density) leaves the
    // publishing to the barrier after it
    if (!a.dynamic_generator && next_reads_no_scalar) return;
    cluster_sync();
    if (!a.dynamic_generator) return;
    float v2 = 0.f, a2 = 0.f;
    for (int64_t k = T.first(a.n); k < T.end(a.n); k += kSmallThreads) {
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
    cluster_sync();
    if (T.rank == 0 && t == 0) generator_finish_one(a.sc, a.particle_size, a.min_ts, a.max_ts, a.lambda_v, a.lambda_a);
    cluster_sync();
}

__device__ __forceinline__ void stamp(const Team& T, unsigned long long* stamps, int i) {
    if (T.rank == 0 && threadIdx.x == 0) stamps[i] = global_ns();
}

template <typename R, bool KAHAN, int SOLVER>
__global__ void __launch_bounds__(kSmallThreads, 1) k_small_steps(SmallStepArgs<R> a) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    __shared__ int s_dec;   // CTA 0: the decision every CTA reads (publish_decision)
    const Team T = team();
    const int t = threadIdx.x;
    const int64_t n = a.n, no = a.n_owners;
    int cur = a.cur;
    R* rho[2] = {(R*)a.buf[0].rho, (R*)a.buf[1].rho};
    R* rho_prev = a.rho_prev;
    StepScalars* sc = a.sc;
    const Lists L{a.nbr, a.count, a.stride, a.K};
    for (int step = 0; step < a.steps; step++) {
        stamp(T, a.stamps, 0);
        // (the search's first phases touch no scalar: the barriers after
        // them publish this before the lists count into it)
        if (T.rank == 0 && t == 0) {
            StepScalars z{};
            z.desired_dt = a.desired_dt;
            z.dt = a.desired_dt;
            *sc = z;
        }
        cur = small_search<R>(a, T, cur, rho, small_smem);
        if (SOLVER != kSmallSESPH) {
            // density double buffer: the current density becomes rho_prev
            R* x = rho[cur];
            rho[cur] = rho_prev;
            rho_prev = x;
        }
        State<R> s = small_state<R>(a, cur, rho[cur]);
        s.rho_prev = rho_prev;
        small_begin_solver<R>(a, T, s, SOLVER == kSmallSESPH);
        stamp(T, a.stamps, 1);
        // the gathering phases' view of the state: positions from this CTA's
        // copy (made for the lists), per phase more fields (small_stage)
        const int64_t lshare = T.share(no), llo = min(no, (int64_t)T.rank * lshare);
        const SmallStage<R> g = small_stage<R>(small_smem, n, lshare);
        State<R> v = s;
        if (a.stage) v.pos = g.pos;
        // the lists of this CTA's owners: its copy when staged (owners outside
        // its share never read them: every list-reading loop runs over the
        // owners' shares)
        const Lists Lv = a.stage_lists ? Lists{g.nbr - llo, g.cnt - llo, lshare, a.K} : L;
        if constexpr (SOLVER == kSmallSESPH) {
            if (!status_now(a.status))
                for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads)
                    if (s.type[k] == FS_TYPE_NORMAL) sesph_density_one<R, KAHAN>(k, v, Lv, a.c);
            cluster_sync();
            stamp(T, a.stamps, 2);
            State<R> va = v;   // the acceleration gathers velocities, densities and pressures
            if (a.stage) {
                stage_fields3<R>(g.f4, s.vel, g.f1, s.rho, g.f2, s.p, n);
                va.vel = g.f4;
                va.rho = g.f1;
                va.p = g.f2;
            }
            if (!status_now(a.status))
                for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads)
                    if (s.type[k] == FS_TYPE_NORMAL) sesph_accel_one<R, KAHAN>(k, va, Lv, a.c);
            cluster_sync();
            stamp(T, a.stamps, 3);
            if (a.dim == 3) {
                // maxima, CFL clamp (k_sesph_maxima, k_sesph_maxima_final, k_cfl)
                float a2 = 0.f, v2 = 0.f;
                if (!status_now(a.status))
                    for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads) {
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
                cluster_sync();
                if (T.rank == 0 && t == 0) {
                    sesph_maxima_final_one(sc);
                    if (!status_now(a.status)) cfl_one(sc, a.particle_size, a.cfl_timestep, a.lambda_v, a.lambda_a);
                }
                cluster_sync();
            }
            stamp(T, a.stamps, 4);
            if (!status_now(a.status))
                for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads) sesph_integrate_at<R>(k, s, sc);
            cluster_sync();
        } else {
            constexpr bool two_d = SOLVER == kSmallIISPH2D;
            // first loop
            const bool ok1 = !__syncthreads_or(status_now(a.status));   // uniform in the CTA: staging inside
            // the loops over all particles take the owners' shares (whose
            // lists this CTA holds) and then shares of the rest (no lists)
            auto all_particles = [&](auto&& f) {
                for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads) f(k);
                for (int64_t k = no + T.first(n - no); k < no + T.end(n - no); k += kSmallThreads) f(k);
            };
            if (ok1 && a.split) {
                all_particles([&](int64_t k) {
                    if (two_d) iisph2d_density_at<R, KAHAN>(k, v, Lv, a.c);
                    else iisph3d_density_at<R, KAHAN>(k, v, Lv, a.c);
                });
            }
            if (a.split) cluster_sync();
            if (ok1) {
                // the first loop gathers velocities and the previous densities
                // (and, split, the densities just computed, which it does not write)
                State<R> v1 = v;
                if (a.stage) {
                    stage_field(g.f4, s.vel, n);
                    stage_field(g.f1, s.rho_prev, n);
                    v1.vel = g.f4;
                    v1.rho_prev = g.f1;
                    if (a.split) {
                        stage_field(g.f2, s.rho, n);
                        v1.rho = g.f2;
                    }
                }
                const R dt = (R)sc->dt;
                all_particles([&](int64_t k) {
                    if (two_d) {
                        if (a.split) iisph2d_l1_at<R, KAHAN, true>(k, v1, Lv, a.c, dt);
                        else iisph2d_l1_at<R, KAHAN, false>(k, v1, Lv, a.c, dt);
                    } else {
                        if (a.split) iisph3d_l1_one<R, KAHAN, true>(k, v1, Lv, a.c, dt);
                        else iisph3d_l1_one<R, KAHAN, false>(k, v1, Lv, a.c, dt);
                    }
                });
            }
            cluster_sync();
            stamp(T, a.stamps, 2);
            // second loop
            if (!status_now(a.status)) {
                const R dt = (R)sc->dt;
                for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads) {
                    // (v* is gathered and written: only the positions are copies)
                    if (two_d) {
                        iisph2d_l2_at<R, KAHAN>(k, v, Lv, a.c, dt);
                    } else if (s.type[k] == FS_TYPE_NORMAL) {
                        if (a.fp32) iisph3d_l2_one<R, KAHAN, true>(k, v, Lv, a.c, dt);
                        else iisph3d_l2_one<R, KAHAN, false>(k, v, Lv, a.c, dt);
                    }
                }
            }
            cluster_sync();
            stamp(T, a.stamps, 3);
            // pressure iterations, each ended by the convergence test (k_iisph_check)
            const bool fp64_test = !a.fp32;
            for (int it = 0; it < a.max_it; it++) {
                // gates work with block barriers (reduce_err_parts) and warp
                // shuffles but no cluster barrier: uniform in each CTA
                const bool run = !__syncthreads_or(status_now(a.status) || ((const volatile StepScalars*)sc)->done);
                if (run) {
                    State<R> vp = v;   // gathers the pressures
                    if (a.stage) {
                        stage_field(g.f1, s.p, n);
                        vp.p = g.f1;
                    }
                    for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads) {
                        if (two_d) iisph2d_pressure_acc_at<R, KAHAN>(k, vp, Lv, a.c);
                        else if (s.type[k] == FS_TYPE_NORMAL) iisph3d_pressure_acc_one<R, KAHAN>(k, vp, Lv, a.c);
                    }
                }
                cluster_sync();
                if (run) {
                    State<R> vu = v;   // gathers the pressure accelerations
                    if (a.stage) {
                        stage_field(g.f4, s.acc, n);
                        vu.acc = g.f4;
                    }
                    const R dt = (R)sc->dt;
                    if (two_d) {
                        double e_sum = 0.0;
                        unsigned int e_cnt = 0;
                        for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads)
                            iisph2d_pressure_update_at<R, KAHAN>(k, vu, Lv, a.c, dt, e_sum, e_cnt);
                        e_sum = warp_sum(e_sum);
                        e_cnt = warp_sum(e_cnt);
                        if ((t & 31) == 0 && e_cnt) {
                            atomicAdd(&sc->err_sum, e_sum);
                            atomicAdd(&sc->err_count, (unsigned long long)e_cnt);
                        }
                    } else {
                        ErrPart o;
                        for (int64_t k = T.first(no); k < T.end(no); k += kSmallThreads) {
                            if (s.type[k] != FS_TYPE_NORMAL) continue;
                            const ErrPart q = iisph3d_pressure_update_one<R, KAHAN>(k, vu, Lv, a.c, dt);
                            o.e_sum += q.e_sum;
                            o.e_cnt += q.e_cnt;
                            o.e_max = fmaxf(o.e_max, q.e_max);
                            o.a2 = fmaxf(o.a2, q.a2);
                            o.v2 = fmaxf(o.v2, q.v2);
                        }
                        reduce_err_parts(o, sc);
                    }
                }
                cluster_sync();
                if (T.rank == 0 && t == 0)
                    iisph_check_one(sc, a.min_it, a.max_it, a.max_err, fp64_test, two_d, a.status,
                                    cudaGraphConditionalHandle{}, false);
                const volatile StepScalars* v = sc;
                if (publish_decision(T, &s_dec, status_now(a.status) || v->done)) break;
            }
            stamp(T, a.stamps, 4);
            if (!two_d) {
                if (T.rank == 0 && t == 0 && !status_now(a.status))
                    cfl_one(sc, a.particle_size, a.cfl_timestep, a.lambda_v, a.lambda_a);
                cluster_sync();
            }
            if (!status_now(a.status))
                for (int64_t k = T.first(n); k < T.end(n); k += kSmallThreads) {
                    if (two_d) iisph2d_integrate_at<R>(k, s, sc);
                    else iisph3d_integrate_at<R>(k, s, sc);
                }
            cluster_sync();
        }
        stamp(T, a.stamps, 5);
    }
    cluster_sync();   // no CTA leaves while another may still read CTA 0's shared memory
}

}  // namespace

size_t small_steps_smem() {
    // the sort's runs (sort_small_cluster); the cell table's key entries and
    // the staged fields reuse the same space
    return 2 * (size_t)kSmallMax * sizeof(unsigned long long);
}

namespace {
cudaLaunchConfig_t small_config(int ctas, size_t smem, cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(kSmallThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr->id = cudaLaunchAttributeClusterDimension;
    attr->val.clusterDim.x = ctas;
    attr->val.clusterDim.y = 1;
    attr->val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}
}  // namespace

template <typename R, bool KAHAN, int SOLVER>
cudaError_t launch_small_steps(const SmallStepArgs<R>& a, cudaStream_t st, int* blocks) {
    auto* kern = k_small_steps<R, KAHAN, SOLVER>;
    // per process: the largest shared-memory size the kernel may ask for, and
    // the largest cluster (a power of two up to kSmallMaxCtas) the device
    // schedules with it; 16 CTAs need the non-portable cluster size
    static int limit = 0;
    if (limit == 0) {
        const size_t most = std::max(small_steps_smem(), kSmallStageMax);   // within the 227 KB a block may take
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        int ctas = kSmallMaxCtas;
        for (; ctas > 1; ctas /= 2) {
            cudaLaunchAttribute attr;
            const cudaLaunchConfig_t cfg = small_config(ctas, most, st, &attr);
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) == cudaSuccess && clusters > 0) break;
            (void)cudaGetLastError();
        }
        limit = ctas;
    }
    // about kSmallPerCta particles per CTA
    int ctas = 1;
    while (ctas < limit && (int64_t)ctas * kSmallPerCta < a.n) ctas *= 2;
    SmallStepArgs<R> b = a;
    const size_t fields = small_stage_bytes<R>(a.n);
    const size_t lists = small_list_bytes((a.n_owners + ctas - 1) / ctas, a.K);
    b.stage = fields <= kSmallStageMax;
    b.stage_lists = b.stage && fields + lists <= kSmallStageMax;
    size_t smem = small_steps_smem();
    if (b.stage) smem = std::max(smem, b.stage_lists ? fields + lists : fields);
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t cfg = small_config(ctas, smem, st, &attr);
    *blocks = ctas;
    return cudaLaunchKernelEx(&cfg, kern, b);
}

#define FSB_SMALL_INSTANCE(R, KAHAN, SOLVER) \
    template cudaError_t launch_small_steps<R, KAHAN, SOLVER>(const SmallStepArgs<R>&, cudaStream_t, int*);
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
