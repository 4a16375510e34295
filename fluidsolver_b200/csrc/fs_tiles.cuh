// Tile lists: the neighbor lists of the 3D IISPH and SESPH fast paths (FP32 with
// compensated sums, device order) and the kernels that walk them.
//
// A tile is kTileOwners consecutive fluid particles of the sorted order.
// Sorted order is linear cell order (x fastest), so a tile's owners lie in a
// few (y, z) rows of cells -- its "groups". The union of a group's 27-cell
// neighborhoods is 9 contiguous ranges of the sorted fluid block plus 9 of
// the sorted boundary block (rows y-1..y+1, z-1..z+1, cells from the group's
// first x - 1 to its last x + 1). A pass copies those ranges of the arrays it
// reads (position and mass, plus one per-neighbor field) into shared memory
// with bulk copies, then every owner walks its own list, whose entries are
// 16-bit offsets into the staged arrays. Neighbor data thus crosses the
// memory system once per tile instead of once per pair, and an entry costs
// 2 bytes instead of 4. Two threads share an owner in the passes (each takes
// half of every octet of entries), which doubles the warps that the shared
// memory of a tile feeds.
//
// A tile whose owners touch the grid's border cells, form more than
// kTileGroups groups, or need more than the staging cap (TileLists::cap) of candidates is a
// fallback tile: its owners get the ordinary 32-bit slot-major lists, which
// the two threads of an owner split in the passes, with the pair arithmetic
// of the tiled owners and the neighbors' data read from global memory.
//
// The neighbor sets are the contract's (hashed 3D: dot(d, d) <= r * r over
// the 27 cells, fs_search.cuh); only the summation order differs from the
// reference, which the compensated sums absorb.
#pragma once

#include "fs_common.cuh"
#include "fs_search.cuh"
#include "fs_solvers.cuh"

namespace fsb {

constexpr int kTileOwners = 128;
constexpr int kPassThreads = 2 * kTileOwners;  // two threads per owner in the passes
constexpr int kTileGroups = 4;
constexpr int kTileRanges = 2 * 9 * kTileGroups;
constexpr int kTileCap = 1536;                 // staged candidates per tile (default; fs_autotune may change it)
constexpr int kTileCapMax = 3072;              // the largest cap (entries address up to 4,096 staged candidates)
constexpr uint32_t kTileFallback = 0xffffffffu;
// entry: byte offset of the candidate's float4 in a staged array (index << 4),
// bit 0 set for boundary neighbors
constexpr uint32_t kEntOffset = 0xfff0u;
constexpr uint32_t kEntBoundary = 0x1u;

// Staged slots: range r of a tile occupies slots [base_r, base_r + len_r) of
// every staged array. In the padded layout base_r is congruent to the range's
// first sorted index modulo 4 and at least the previous range's end rounded up
// to a multiple of 4: a float array's range then starts and ends, rounded
// outwards to 4 floats, on 16-byte boundaries in global and in shared memory
// alike, so it is staged by one bulk copy, as the float4 arrays are; the
// rounding lands in padding slots that no entry addresses. A tile whose
// padded layout exceeds the staging cap but whose candidates fit keeps the
// packed layout (base_r = the lengths before r), and its float arrays go
// through 4-byte copies. The range's padded extent:
__host__ __device__ __forceinline__ uint32_t padded_slots(uint32_t start, uint32_t len) {
    return len ? ((start + len + 3u) & ~3u) - (start & ~3u) : 0u;
}

// a tile's header as stored (TileDesc::h)
struct TileHeadRaw {
    uint32_t nranges;                  // non-empty candidate ranges, or kTileFallback
    uint32_t staged;                   // candidates staged in total | (of them in fluid ranges << 16)
    uint32_t slots;                    // padded layout: slots in total | (of them in fluid ranges << 16); 0: packed
    uint32_t octets;                   // octets of entries of the tile's longest list
};
// the header as the passes use it
struct TileHead {
    uint32_t nranges, staged, staged_fluid, slots, slots_fluid, octets;
};
struct alignas(16) TileDesc {
    TileHeadRaw h;
    uint32_t start[kTileRanges];       // first sorted index of each range
    uint32_t len_base[kTileRanges];    // length | kRangeBoundary for boundary ranges | (first staged slot << 16)
};

__device__ __forceinline__ TileHead load_head(const TileDesc* d) {
    const uint4 a = *reinterpret_cast<const uint4*>(d);
    return TileHead{a.x, a.y & 0xffffu, a.y >> 16, a.z & 0xffffu, a.z >> 16, a.w};
}

// the range of thread t (t < kTileRanges), loaded before the tile's header
// is known
struct TileRange {
    uint32_t start, len_base;
};
__device__ __forceinline__ TileRange load_range(const TileDesc* d, int t) {
    return t < kTileRanges ? TileRange{d->start[t], d->len_base[t]} : TileRange{0u, 0u};
}
constexpr uint32_t kRangeBoundary = 0x8000u;
constexpr uint32_t kRangeLen = 0x7fffu;

struct TileLists {
    const TileDesc* __restrict__ desc;
    const uint4* __restrict__ ent;     // [K / 8][stride]: 8 entries of 16 bits per owner and octet
    const uint32_t* __restrict__ count;  // per owner: entries | (fluid entries << 16); fluid entries come first
    int64_t stride;
    int K;
    int cap;                           // staged candidates per tile the lists were built for
};

// dynamic shared memory of the list builder and of the passes. A pass
// stages its candidates (bytes per candidate: 36 for the first loop --
// position, velocity, density --, 32 for position and a float4 field, 20 for
// position and a float field), then the tile's entries and list lengths.
inline size_t tile_build_smem(int K, int cap) { return (size_t)cap * 16 + (size_t)kTileOwners * (K + 8) * 2; }
inline size_t tile_pass_smem(int bytes_per_candidate, int K, bool slab, int cap) {
    return (size_t)cap * bytes_per_candidate + (slab ? (size_t)(K / 8) * kTileOwners * 16 + kTileOwners * 4 : 0);
}
// Whether a pass reads its entries straight from the global octet planes
// (one octet ahead of use) instead of staging them in shared memory. Without
// the slab, the first loop and the pressure passes fit 4 and 4-5 blocks per
// SM instead of 3 and were faster on the 1M-particle dam (B200); the second
// loop would need more than the 64 registers that 4 blocks leave it.
constexpr bool kL1GlobalEntries = true;
constexpr bool kL2GlobalEntries = false;
constexpr bool kPressureGlobalEntries = true;

// ---------------------------------------------------------------------------
// asynchronous staging (the builder and the passes)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// the mbarrier that a tile's bulk copies complete on
struct TileStage {
    uint64_t bar;
};

// One try of the wait for phase 0: the thread sleeps until the phase
// completes or kTileWaitHintNs pass (the try's time limit), so that waiting
// warps issue no instructions while the copies land.
constexpr uint32_t kTileWaitHintNs = 20000;
__device__ __forceinline__ uint32_t mbar_try_wait0(TileStage& st) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(&st.bar)), "r"(kTileWaitHintNs)
        : "memory");
    return ok;
}

// Tries of the first wait for a tile's staging (each try sleeps up to
// kTileWaitHintNs: about 1.3 s in all). fs_set_tile_wait_limit lowers it so
// that a test can make the wait run out and check the error path; it is
// kTileWaitTries otherwise.
constexpr int kTileWaitTries = 1 << 16;
constexpr int kTileDrainTries = 1 << 16;
static __device__ int g_tile_wait_tries = kTileWaitTries;

// Waits for the staging to land, with a bounded number of tries. Returns
// false, with FS_ERR_TIMEOUT raised, if the copies did not complete; the
// caller then skips the tile. Before that, a second, longer bounded wait
// (kTileDrainTries, independent of the first's limit) lets copies still in
// flight land, so that none writes into shared memory after the block has
// left it.
__device__ __forceinline__ bool stage_tile_wait(TileStage& st, int* __restrict__ status) {
    asm volatile("cp.async.wait_all;" ::: "memory");   // the packed layout's 4-byte copies
    uint32_t ok = 0;
    const int tries = g_tile_wait_tries;
    for (int it = 0; it < tries && !ok; it++) ok = mbar_try_wait0(st);
    const int late = __syncthreads_or(!ok);
    if (late) {
        if (threadIdx.x == 0) raise_status(status, FS_ERR_TIMEOUT);
        for (int it = 0; it < kTileDrainTries && !ok; it++) ok = mbar_try_wait0(st);
        __syncthreads();
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// list builder: one block of kTileOwners threads per tile
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTileOwners, 4) k_build_tiles(
    int64_t n_owners, const float4* __restrict__ pos, const uint8_t* __restrict__ type,
    const uint32_t* __restrict__ cell_start, WalkParams w, TileDesc* __restrict__ desc,
    uint4* __restrict__ ent, int64_t ent_stride, uint32_t* __restrict__ nbr, int64_t stride, int K, int cap,
    uint32_t* __restrict__ count, int* __restrict__ status, StepScalars* __restrict__ sc) {
    extern __shared__ float4 tile_smem[];
    float4* sp = tile_smem;                                          // staged positions
    uint16_t* sent = reinterpret_cast<uint16_t*>(tile_smem + cap);   // [owner][K + 8] entries
    const int KP = K + 8;
    __shared__ long long s_key[kTileOwners];
    __shared__ uint32_t s_cnt[kTileOwners];
    __shared__ int s_lead[kTileOwners / 32];
    // per group: the first cell of its own row, the row and plane strides of
    // its scene's grid, and its first and last x
    __shared__ long long s_grow[kTileGroups];
    __shared__ int s_gd0[kTileGroups], s_gd01[kTileGroups], s_gx0[kTileGroups], s_gx1[kTileGroups];
    // s_base: first staged slot | (position among the non-empty ranges << 16)
    __shared__ uint32_t s_start[kTileRanges], s_len[kTileRanges], s_base[kTileRanges];
    // per-warp partial results, in arrays whose contents are dead by then
    // (static shared memory decides whether 5 blocks fit on an SM)
    uint32_t* s_wlen = s_cnt;                                     // warp sums of the range scans
    uint32_t* s_wne = s_cnt + kTileOwners / 32;
    uint32_t* s_wl = s_cnt + 2 * (kTileOwners / 32);              // warp sums of the header's totals
    uint32_t* s_wlf = s_cnt + 3 * (kTileOwners / 32);
    uint32_t* s_wpf = s_cnt + 4 * (kTileOwners / 32);
    uint32_t* s_wmax = reinterpret_cast<uint32_t*>(s_lead);       // warp maxima of the list lengths
    {
        // an earlier error (e.g. non-finite positions) ends the step; an overflow
        // elsewhere does not stop the counting (the largest list decides the growth)
        const int err = *status;
        if (err && err != FS_ERR_CAPACITY) return;
    }

    const int t = threadIdx.x, lane = t & 31;
    const int64_t tile = blockIdx.x;
    const int64_t k = tile * kTileOwners + t;
    const bool valid = k < n_owners;
    float4 pk = make_float4(0.f, 0.f, 0.f, 0.f);
    int lx = 0;
    long long key = -1;   // first cell of the owner's own row (unique across scenes)
    int d0 = 0, d01 = 0;
    bool border = false;
    if (valid) {
        pk = pos[k];
        const SceneGrid gr = w.grid_of(k);
        lx = cell_coord<float>(pk.x, w.r, false) - gr.o0;
        const int ly = cell_coord<float>(pk.y, w.r, false) - gr.o1;
        const int lz = cell_coord<float>(pk.z, w.r, false) - gr.o2;
        border = lx < 2 || ly < 2 || lz < 2 || lx > gr.d0 - 3 || ly > gr.d1 - 3 || lz > gr.d2 - 3;
        d0 = gr.d0;
        d01 = gr.d0 * gr.d1;
        key = border ? -2 : gr.base + ((long long)lz * gr.d1 + ly) * gr.d0;
    }
    s_key[t] = key;
    const int any_border = __syncthreads_or(valid && border);
    // groups: runs of equal row keys (non-decreasing in k: sorted order)
    const bool lead = valid && (t == 0 || s_key[t - 1] != key);
    const unsigned bal = __ballot_sync(0xffffffffu, lead);
    if (lane == 0) s_lead[t >> 5] = __popc(bal);
    __syncthreads();
    int G = 0, before = 0;
#pragma unroll
    for (int i = 0; i < kTileOwners / 32; i++) {
        G += s_lead[i];
        if (i < (t >> 5)) before += s_lead[i];
    }
    const int g = before + __popc(bal & ((1u << lane) - 1u)) + (lead ? 1 : 0) - 1;
    bool fallback = any_border || G > kTileGroups;
    int NR = 0;
    // the header's totals: candidates and padded slots, all and in fluid ranges
    uint32_t tot_len = 0, tot_len_fluid = 0, tot_slots = 0, tot_slots_fluid = 0;
    bool padded = false;
    if (!fallback) {
        if (lead) {
            s_grow[g] = key;
            s_gd0[g] = d0;
            s_gd01[g] = d01;
            s_gx0[g] = lx;
        }
        if (valid && (t == kTileOwners - 1 || s_key[t + 1] != key)) s_gx1[g] = lx;
        __syncthreads();
        NR = 18 * G;
        uint32_t len = 0, a = 0;
        if (t < NR) {
            const int region = t / (9 * G), gg = (t % (9 * G)) / 9, r = t % 9;
            const int64_t rb = s_grow[gg] + (int64_t)(r / 3 - 1) * s_gd01[gg] + (int64_t)(r % 3 - 1) * s_gd0[gg];
            const uint32_t* cs = cell_start + region * (w.cells + 1);
            a = cs[rb + s_gx0[gg] - 1];
            len = cs[rb + s_gx1[gg] + 2] - a;
            s_start[t] = a;
            s_len[t] = len;
        }
        // exclusive prefix sums over the ranges (thread t: range t) of their
        // padded extents -- first staged slots -- and of their non-emptiness
        // -- positions in the descriptor --, by warp scans; and the header's
        // totals (fluid ranges, t < 9 G, come first)
        const uint32_t ps = padded_slots(a, len);
        const bool fluid_range = t < 9 * G;
        uint32_t incl = ps, incl_len = len, ne = len ? 1u : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o), y = __shfl_up_sync(0xffffffffu, ne, o);
            const uint32_t z = __shfl_up_sync(0xffffffffu, incl_len, o);
            if (lane >= o) {
                incl += x;
                ne += y;
                incl_len += z;
            }
        }
        const uint32_t wl = __reduce_add_sync(0xffffffffu, len);
        const uint32_t wlf = __reduce_add_sync(0xffffffffu, fluid_range ? len : 0u);
        const uint32_t wpf = __reduce_add_sync(0xffffffffu, fluid_range ? ps : 0u);
        if (lane == 31) {
            s_wlen[t >> 5] = incl;
            s_wne[t >> 5] = ne;
        }
        if (lane == 0) {
            s_wl[t >> 5] = wl;
            s_wlf[t >> 5] = wlf;
            s_wpf[t >> 5] = wpf;
        }
        __syncthreads();
        uint32_t before = 0, before_ne = 0, before_len = 0;
#pragma unroll
        for (int i = 0; i < kTileOwners / 32; i++) {
            if (i < (t >> 5)) {
                before += s_wlen[i];
                before_ne += s_wne[i];
                before_len += s_wl[i];
            }
            tot_slots += s_wlen[i];
            tot_len += s_wl[i];
            tot_len_fluid += s_wlf[i];
            tot_slots_fluid += s_wpf[i];
        }
        // the padded layout where it fits the cap, else the packed one
        // (every thread has read the warp sums before s_cnt is reused)
        padded = tot_slots <= (uint32_t)cap;
        const uint32_t slot = padded ? before + incl - ps + (a & 3u) : before_len + incl_len - len;
        if (t < NR) s_base[t] = slot | ((before_ne + ne - (len ? 1u : 0u)) << 16);
        fallback = !padded && tot_len > (uint32_t)cap;
        __syncthreads();
    }

    if (fallback) {
        // ordinary 32-bit lists for this tile's owners
        if (t == 0) desc[tile].h.nranges = kTileFallback;
        uint32_t c = 0;
        if (valid) {
            c = build_list_one<float>(k, pos, type, cell_start, w, true, nbr, stride, K);
            count[k] = c;
        }
        note_list_length(c, K, status, sc);
        return;
    }

    // the owner's 18 row bounds (its 27 cells), loaded while the staging lands
    uint32_t lo[18], hi[18];
    if (valid) {
#pragma unroll
        for (int q = 0; q < 18; q++) {
            const uint32_t* cs = cell_start + (q / 9) * (w.cells + 1);
            const int64_t rb = key + (int64_t)((q % 9) / 3 - 1) * d01 + (int64_t)(q % 3 - 1) * d0;
            lo[q] = cs[rb + lx - 1];
            hi[q] = cs[rb + lx + 2];
        }
    }

    // stage the candidates' positions: a bulk copy per range (the TMA engine)
    __shared__ TileStage stg;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&stg.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (t == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&stg.bar)),
                     "r"(tot_len * 16u)
                     : "memory");
    if (t < NR && s_len[t])
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(sp + (s_base[t] & 0xffffu))),
            "l"(pos + s_start[t]), "r"(s_len[t] * 16u), "r"(smem_u32(&stg.bar))
            : "memory");
    if (!stage_tile_wait(stg, status)) return;

    // each owner tests the candidates of its own 27 cells, two at a time
    uint32_t c = 0;
    if (valid) {
        uint16_t* my = sent + t * KP;
        auto test = [&](float4 pj, uint32_t entry) {
            const float d0 = pk.x - pj.x, d1 = pk.y - pj.y, d2 = pk.z - pj.z;
            if ((d0 * d0 + d1 * d1) + d2 * d2 <= w.r2) {
                if ((int)c < K) my[c] = (uint16_t)entry;
                c++;
            }
        };
        uint32_t cf = 0;
#pragma unroll
        for (int q = 0; q < 18; q++) {
            if (q == 9) cf = c;
            const int qq = ((q / 9) * G + g) * 9 + q % 9;
            const uint32_t off = (s_base[qq] & 0xffffu) - s_start[qq];
            const uint32_t flag = q >= 9 ? kEntBoundary : 0u;
            uint32_t i = lo[q] + off;
            const uint32_t e = hi[q] + off;
            for (; i + 2 <= e; i += 2) {
                const float4 p0 = sp[i], p1 = sp[i + 1];
                test(p0, (i << 4) | flag);
                test(p1, ((i + 1) << 4) | flag);
            }
            if (i < e) test(sp[i], (i << 4) | flag);
        }
        count[k] = min(c, 0xffffu) | (min(cf, 0xffffu) << 16);
    }
    s_cnt[t] = c;
    note_list_length(c, K, status, sc);
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, c);
    if (lane == 0) s_wmax[t >> 5] = wmax;
    // the descriptor: the non-empty ranges in order (thread t: range t), then
    // the header
    if (t < NR && s_len[t]) {
        const uint32_t slot = s_base[t] >> 16;
        desc[tile].start[slot] = s_start[t];
        desc[tile].len_base[slot] = s_len[t] | (t >= 9 * G ? kRangeBoundary : 0u) | (s_base[t] << 16);
    }
    __syncthreads();
    if (t == 0) {
        uint32_t mx = 0;
#pragma unroll
        for (int i = 0; i < kTileOwners / 32; i++) mx = max(mx, s_wmax[i]);
        const uint32_t last = NR - 1;
        const uint32_t nonempty = (s_base[last] >> 16) + (s_len[last] ? 1u : 0u);
        // fluid ranges come first: the first boundary range's slot is their total
        *reinterpret_cast<uint4*>(desc + tile) =
            make_uint4(nonempty, tot_len | (tot_len_fluid << 16), padded ? tot_slots | (tot_slots_fluid << 16) : 0u,
                       (min(mx, (uint32_t)K) + 7) / 8);
    }
    // octets of entries, coalesced across the tile's owners
    const int O = K / 8;
    for (int idx = t; idx < kTileOwners * O; idx += kTileOwners) {
        const int ow = idx % kTileOwners, o = idx / kTileOwners;
        if ((uint32_t)o * 8 < min(s_cnt[ow], (uint32_t)K))
            ent[(int64_t)o * ent_stride + tile * kTileOwners + ow] =
                *reinterpret_cast<const uint4*>(sent + ow * KP + o * 8);
    }
}

// Shared-memory view of a tile's lists: entries [octet][owner] and lengths.
struct TileSlab {
    uint4* ent;
    uint32_t* count;
};

// Starts the copies of the tile's candidate ranges into shared memory: a
// bulk copy (the TMA engine) per range and float4 array, issued by the
// range's thread, and one per octet plane of the tile's entries and for its
// list lengths, issued by threads from the top of the block; completion is
// counted in bytes on the mbarrier. In the padded layout a float array's
// range is copied rounded outwards to 16-byte boundaries into its padded
// slots (padded_slots); in the packed layout it goes through 4-byte cp.async
// copies, a warp per range. h and rg are the tile's header and the calling
// thread's range, loaded up front. FLUID_ONLY skips the boundary ranges;
// SLAB false leaves the entries and list lengths in global memory. A float
// array (src1) must be readable up to its length rounded up to a multiple of 4.
template <int NV4, bool FLUID_ONLY = false, bool SLAB = true>
__device__ __forceinline__ void stage_tile_async(TileStage& st, const TileDesc* __restrict__ d, const TileHead& h,
                                                 const TileRange& rg,
                                                 const float4* const (&src4)[NV4], float4* const (&dst4)[NV4],
                                                 const float* __restrict__ src1, float* dst1, const TileLists& T,
                                                 const TileSlab& slab) {
    const int t = threadIdx.x;
    const int64_t first = (int64_t)blockIdx.x * kTileOwners;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&st.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (t == 0) {
        const uint32_t bytes = (FLUID_ONLY ? h.staged_fluid : h.staged) * 16u * (uint32_t)NV4 +
                               (src1 != nullptr ? (FLUID_ONLY ? h.slots_fluid : h.slots) * 4u : 0u) +   // 0: packed
                               (SLAB ? h.octets * (uint32_t)kTileOwners * 16u + (uint32_t)kTileOwners * 4u : 0u);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&st.bar)), "r"(bytes)
                     : "memory");
    }
    // the tile's list lengths and its entry octets (one contiguous run of
    // kTileOwners octets per slot group)
    const int tb = SLAB ? (int)blockDim.x - 1 - t : -1;   // threads from the top of the block, clear of the range copies
    if (tb == 0)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(slab.count)),
            "l"(T.count + first), "r"((uint32_t)kTileOwners * 4u), "r"(smem_u32(&st.bar))
            : "memory");
    else if (tb > 0 && tb <= (int)h.octets)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(slab.ent + (tb - 1) * kTileOwners)),
            "l"(T.ent + (int64_t)(tb - 1) * T.stride + first), "r"((uint32_t)kTileOwners * 16u),
            "r"(smem_u32(&st.bar))
            : "memory");
    if ((uint32_t)t < h.nranges && !(FLUID_ONLY && (rg.len_base & kRangeBoundary))) {
        const uint32_t a = rg.start, len = rg.len_base & kRangeLen, base = rg.len_base >> 16;
        // the candidates' arrays are re-read by the neighboring tiles and by the
        // next pass: kept in L2 ahead of the streamed lists (evict_last)
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
#pragma unroll
        for (int v = 0; v < NV4; v++) {
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
                "%4;" ::"r"(smem_u32(dst4[v] + base)),
                "l"(src4[v] + a), "r"(len * 16u), "r"(smem_u32(&st.bar)), "l"(pol)
                : "memory");
        }
        if (src1 != nullptr && h.slots) {
            // base is congruent to a modulo 4: both ends round to 16-byte boundaries
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
                "%4;" ::"r"(smem_u32(dst1 + (base - (a & 3u)))),
                "l"(src1 + (a & ~3u)), "r"(padded_slots(a, len) * 4u), "r"(smem_u32(&st.bar)), "l"(pol)
                : "memory");
        }
    }
    if (src1 != nullptr && !h.slots) {
        const int lane = t & 31;
        for (uint32_t q = t >> 5; q < h.nranges; q += blockDim.x / 32) {
            const uint32_t a = d->start[q], lb = d->len_base[q];
            if (FLUID_ONLY && (lb & kRangeBoundary)) continue;
            const uint32_t len = lb & kRangeLen, base = lb >> 16;
            for (uint32_t i = lane; i < len; i += 32)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst1 + base + i)),
                             "l"(src1 + a + i)
                             : "memory");
        }
    }
}

// Where a pass reads a tile's entries from: the staged slab in shared memory
// or the octet planes in global memory. src(o, half): half `half` of the
// owner's octet o -- entries 4 half .. 4 half + 3, two 32-bit words, so the
// two threads of an owner load disjoint 8 bytes.
struct SlabEntries {
    const uint4* e;   // slab.ent + local owner
    __device__ __forceinline__ uint2 operator()(uint32_t o, int half) const {
        return reinterpret_cast<const uint2*>(e + o * kTileOwners)[half];
    }
};
struct GlobalEntries {
    const uint4* __restrict__ e;   // T.ent + owner
    int64_t stride;
    __device__ __forceinline__ uint2 operator()(uint32_t o, int half) const {
        return __ldg(reinterpret_cast<const uint2*>(e + o * stride) + half);
    }
};

// The first AHEAD octets (this thread's halves) of an owner's list, loaded
// before they are walked; octets are read up to `octets`, which may exceed
// the owner's own list (the planes hold that many octets for every owner of
// the tile) but never its plane count.
template <int AHEAD, typename Src>
__device__ __forceinline__ void load_entry_head(const Src& src, uint32_t octets, int half, uint2 (&ahead)[AHEAD]) {
#pragma unroll
    for (int d = 0; d < AHEAD; d++) ahead[d] = (uint32_t)d < octets ? src(d, half) : make_uint2(0u, 0u);
}

// Visits one half of an owner's list (entries 4 half .. 4 half + 3 of every
// octet; cnt: the owner's packed list length): f(byte offset into a staged
// float4 array, boundary) for each, and flush() after every second octet and
// at the end (where the passes fold their partial sums into the compensated
// accumulators). ahead holds the list's first AHEAD octets (load_entry_head);
// the next AHEAD octets are loaded while one is visited. FLUID_ONLY visits the
// fluid entries, which come first in a list and have the boundary bit clear.
template <bool FLUID_ONLY, int AHEAD, typename Src, typename F, typename Flush>
__device__ __forceinline__ void for_tile_entries(const Src& src, uint32_t cnt, int K, int half, uint2 (&ahead)[AHEAD],
                                                 F&& f, Flush&& flush) {
    constexpr int kEntryPrefetch = AHEAD;
    const uint32_t all = min(cnt & 0xffffu, (uint32_t)K);
    const uint32_t n = FLUID_ONLY ? min(cnt >> 16, all) : all;
    auto visit = [&](uint32_t v) {
        if (FLUID_ONLY) f(v, false);
        else f(v & kEntOffset, (v & kEntBoundary) != 0u);
    };
    const uint32_t full = n / 8, octets = (n + 7) / 8;
    uint32_t o = 0;
    for (; o < full; o++) {
        const uint2 cur = ahead[0];
#pragma unroll
        for (int d = 0; d + 1 < kEntryPrefetch; d++) ahead[d] = ahead[d + 1];
        if (o + kEntryPrefetch < octets) ahead[kEntryPrefetch - 1] = src(o + kEntryPrefetch, half);
        visit(cur.x & 0xffffu);
        visit(cur.x >> 16);
        visit(cur.y & 0xffffu);
        visit(cur.y >> 16);
        if (o & 1u) flush();
    }
    const int m = (int)(n - full * 8) - 4 * half;   // this half's entries of the last, partial octet
    if (m > 0) {
        const uint2 cur = ahead[0];
        visit(cur.x & 0xffffu);
        if (m > 1) visit(cur.x >> 16);
        if (m > 2) visit(cur.y & 0xffffu);
        if (m > 3) visit(cur.y >> 16);
    }
    flush();
}

// The first AHEAD octets of owner k's list in the global octet planes, for
// a pass that walks them from there (GLOBAL), issued before the tile's
// staging has landed: the entries do not depend on it. h: the tile's header.
template <bool GLOBAL, int AHEAD>
__device__ __forceinline__ void prefetch_tile_list(const TileLists& T, const TileHead& h, int64_t k, int half,
                                                   uint2 (&ahead)[AHEAD]) {
    if constexpr (GLOBAL) load_entry_head(GlobalEntries{T.ent + k, T.stride}, h.octets, half, ahead);
}

// Walks one half of owner k's list (threadIdx.x / 2 within its tile) from
// the global octet planes (GLOBAL; cnt: the owner's packed list length,
// loaded by the caller; ahead: from prefetch_tile_list) or from the staged
// slab.
template <bool GLOBAL, bool FLUID_ONLY, int AHEAD, typename F, typename Flush>
__device__ __forceinline__ void walk_tile_list(const TileLists& T, const TileSlab& slab, int64_t k, uint32_t cnt,
                                               int half, uint2 (&ahead)[AHEAD], F&& f, Flush&& flush) {
    if constexpr (GLOBAL) {
        for_tile_entries<FLUID_ONLY, AHEAD>(GlobalEntries{T.ent + k, T.stride}, cnt, T.K, half, ahead, f, flush);
    } else {
        const int ol = (int)(threadIdx.x >> 1);
        const SlabEntries src{slab.ent + ol};
        const uint32_t c = slab.count[ol];
        const uint32_t all = min(c & 0xffffu, (uint32_t)T.K);
        load_entry_head(src, ((FLUID_ONLY ? min(c >> 16, all) : all) + 7) / 8, half, ahead);
        for_tile_entries<FLUID_ONLY, AHEAD>(src, c, T.K, half, ahead, f, flush);
    }
}

// Walks owner k's 32-bit list in a fallback tile, the entries of this
// thread of the owner's TPO (half, half + TPO, ...): f(sorted index, boundary)
// for each (the fluid entries only with FLUID_ONLY), flush() after every 8
// visits and at the end, as for_tile_entries does.
template <bool FLUID_ONLY, int TPO = 2, typename F, typename Flush>
__device__ __forceinline__ void walk_fallback_list(const Lists& L, int64_t k, int half, F&& f, Flush&& flush) {
    const uint32_t nn = L.size(k);
    uint32_t visited = 0;
    for (uint32_t q = (uint32_t)half; q < nn; q += TPO) {
        const uint32_t e = L.at(k, q);
        const bool bnd = (e & kBoundaryBit) != 0u;
        if (FLUID_ONLY && bnd) continue;
        f(e & kIndexMask, bnd);
        if ((++visited & 7u) == 0u) flush();
    }
    flush();
}

// The pressure passes with TPO threads per owner (1, 2 or 4; fs_autotune
// chooses): each thread takes a contiguous 8 / TPO of every octet of the
// owner's fluid entries, 4 / TPO 32-bit words, read straight from the global
// octet planes AHEAD octets ahead of use.
template <int TPO> struct OctetShare {
    uint32_t w[4 / TPO];
};
template <int TPO>
__device__ __forceinline__ OctetShare<TPO> load_share(const uint4* __restrict__ e, int64_t stride, uint32_t o, int part) {
    OctetShare<TPO> r;
    const uint4* q = e + o * stride;
    if constexpr (TPO == 1) {
        const uint4 v = __ldg(q);
        r.w[0] = v.x;
        r.w[1] = v.y;
        r.w[2] = v.z;
        r.w[3] = v.w;
    } else if constexpr (TPO == 2) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(q) + part);
        r.w[0] = v.x;
        r.w[1] = v.y;
    } else {
        r.w[0] = __ldg(reinterpret_cast<const uint32_t*>(q) + part);
    }
    return r;
}
// the first AHEAD octets' shares of owner k, issued before the tile's
// staging has landed (h.octets: the tile's longest list in octets)
template <int TPO, int AHEAD>
__device__ __forceinline__ void prefetch_shares(const TileLists& T, const TileHead& h, int64_t k, int part,
                                                OctetShare<TPO> (&ahead)[AHEAD]) {
#pragma unroll
    for (int d = 0; d < AHEAD; d++) {
        if ((uint32_t)d < h.octets) {
            ahead[d] = load_share<TPO>(T.ent + k, T.stride, d, part);
        } else {
#pragma unroll
            for (int i = 0; i < 4 / TPO; i++) ahead[d].w[i] = 0u;
        }
    }
}
// Visits this thread's share of owner k's fluid entries: f(byte offset into
// a staged float4 array) for each, flush() after every 8 visits and at the
// end. With TPO 2 the visits and flushes are those of for_tile_entries.
template <int TPO, int AHEAD, typename F, typename Flush>
__device__ __forceinline__ void walk_fluid_shares(const TileLists& T, int64_t k, uint32_t cnt, int part,
                                                  OctetShare<TPO> (&ahead)[AHEAD], F&& f, Flush&& flush) {
    constexpr int W = 4 / TPO;
    const uint32_t all = min(cnt & 0xffffu, (uint32_t)T.K);
    const uint32_t n = min(cnt >> 16, all);
    const uint32_t full = n / 8, octets = (n + 7) / 8;
    for (uint32_t o = 0; o < full; o++) {
        const OctetShare<TPO> cur = ahead[0];
#pragma unroll
        for (int d = 0; d + 1 < AHEAD; d++) ahead[d] = ahead[d + 1];
        if (o + AHEAD < octets) ahead[AHEAD - 1] = load_share<TPO>(T.ent + k, T.stride, o + AHEAD, part);
#pragma unroll
        for (int i = 0; i < W; i++) {
            f(cur.w[i] & 0xffffu);
            f(cur.w[i] >> 16);
        }
        if ((o & (TPO - 1)) == TPO - 1) flush();
    }
    const int m = (int)(n - full * 8) - part * (8 / TPO);   // this thread's entries of the last, partial octet
    if (m > 0) {
        const OctetShare<TPO> cur = ahead[0];
#pragma unroll
        for (int i = 0; i < W; i++) {
            if (2 * i < m) f(cur.w[i] & 0xffffu);
            if (2 * i + 1 < m) f(cur.w[i] >> 16);
        }
    }
    flush();
}

// Octets a pass loads ahead of the one it visits. The first loop's and the
// pressure passes' depths are chosen per context by fs_autotune among
// 1..kMaxAhead (defaults: what the 1M dam preferred on a B200, 1 and 3); the
// second loop walks its staged slab with 1.
constexpr int kMaxAhead = 4;
constexpr int kL2Ahead = 1;
struct TileTuning {
    int l1_ahead = 1;
    int pressure_ahead = 3;
    int cap = kTileCap;   // staged candidates per tile
    int block = 128;      // threads per block of the step's per-particle kernels (keys, reorder, integration)
    int pressure_tpo = 2; // threads per owner in the pressure passes (1, 2, 4)
};

// the slab after a pass's staged candidates (bytes_per_candidate each)
__device__ __forceinline__ TileSlab slab_at(float4* smem, int bytes_per_candidate, int K, int cap) {
    char* b = reinterpret_cast<char*>(smem) + cap * bytes_per_candidate;
    return TileSlab{reinterpret_cast<uint4*>(b), reinterpret_cast<uint32_t*>(b + (K / 8) * kTileOwners * 16)};
}

template <typename T> __device__ __forceinline__ const T& at_offset(const T* base, uint32_t off) {
    return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + off);
}

// value of a compensated accumulator, summed over the TPO threads of an owner
template <int TPO = 2> __device__ __forceinline__ float pair_total(const Acc<float, true>& a) {
    float v = a.s - a.c;
#pragma unroll
    for (int o = 1; o < TPO; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <int TPO = 2> __device__ __forceinline__ V3<float> pair_total(const Acc3<float, true>& a) {
    return v3<float>(pair_total<TPO>(a.x), pair_total<TPO>(a.y), pair_total<TPO>(a.z));
}

__device__ __forceinline__ V3<float> sub3(float4 a, float4 b) { return v3<float>(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(V3<float> a, V3<float> b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ float r2_of(V3<float> d) { return __fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, d.x * d.x)); }
__device__ __forceinline__ V3<float> fma3(float s, V3<float> d, V3<float> acc) {
    return v3<float>(__fmaf_rn(s, d.x, acc.x), __fmaf_rn(s, d.y, acc.y), __fmaf_rn(s, d.z, acc.z));
}

// 1/sqrt(x) for normal x (the MUFU approximation; with x >= FastSpline::kTiny no input
// is denormal, so the flush-to-zero form gives rsqrtf's result without its
// denormal-input handling)
__device__ __forceinline__ float rsqrt_normal(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The cubic spline of the fast mode, evaluated from a listed pair's squared
// distance r2 (r2 <= (2h)^2). The reference's piecewise cubic
// (CubicSplineKernel3D.cpp:7-66) with its polynomials expanded, q = |d| / h:
//   W        = alpha (4 - 6 q^2 + 3 q^3)              q < 1
//            = alpha (2 - q)^3                        1 <= q <= 2
//   gradW(d) = f d,  f = alpha (9 q - 12)             q < 1
//                    f = -3 alpha h (2 - q)^2 / |d|   1 <= q <= 2
// (for q < 1 that is alpha h (-3 (2 - q)^2 + 12 (1 - q)^2) / |d| with
// |d| = q h). One rsqrt per pair, no divisions, no branches. The self pair
// (d = 0; the rsqrt takes max(r2, 1e-30), so q = 0) gets the finite
// f = -12 alpha and so a zero gradient, as the reference's |d| <= FLT_EPSILON
// test gives.
struct FastSpline {
    static constexpr float kTiny = 1e-30f;   // r2 floor of the rsqrt: the self pair gets q = 0
    float a, inv_h, a9, a12, a3h;
    __device__ explicit FastSpline(const SplineKernel<float>& k)
        : a(k.alpha), inv_h(1.f / k.h), a9(9.f * k.alpha), a12(12.f * k.alpha), a3h(3.f * k.alpha * k.h) {}
    __device__ __forceinline__ float grad(float r2) const {
        const float inv = rsqrt_normal(fmaxf(r2, kTiny));
        const float q = (r2 * inv) * inv_h;
        const float t = fmaxf(2.f - q, 0.f);
        return q < 1.f ? __fmaf_rn(a9, q, -a12) : -a3h * (t * t) * inv;
    }
    __device__ __forceinline__ void value_grad(float r2, float& w, float& f) const {
        const float inv = rsqrt_normal(fmaxf(r2, kTiny));
        const float q = (r2 * inv) * inv_h;
        const float t = fmaxf(2.f - q, 0.f);
        const bool inner = q < 1.f;
        f = inner ? __fmaf_rn(a9, q, -a12) : -a3h * (t * t) * inv;
        w = a * (inner ? __fmaf_rn(q * q, __fmaf_rn(3.f, q, -6.f), 4.f) : (t * t) * t);
    }
};

// ---------------------------------------------------------------------------
// IISPH 3D passes on tile lists (the fast-mode formulas of the gather
// kernels: IISPHFluidSolver3D.hpp:141-212, :216-339, :348-397, :402-461).
// Blocks of kPassThreads threads: owner = threadIdx.x / 2, half =
// threadIdx.x % 2; the even thread of a pair writes the owner's results.
// ---------------------------------------------------------------------------

// first loop. Blocks [0, n_tiles) are tiles of fluid owners; the blocks after
// them take the boundary and inactive particles [n_fluid, n), which need no
// neighbor sums.
template <int AHEAD>
__global__ void __launch_bounds__(kPassThreads, kL1GlobalEntries ? 4 : 3) k_tile_iisph3d_l1(int64_t n_fluid, int64_t n, int64_t n_tiles,
                                                                  State<float> s, TileLists T, Lists L,
                                                                  SolverConsts<float> c,
                                                                  const StepScalars* __restrict__ sc,
                                                                  int* __restrict__ status) {
    extern __shared__ float4 tile_smem[];
    if (blockIdx.x >= n_tiles) {
        if (*status) return;
        const int64_t k = n_fluid + (blockIdx.x - n_tiles) * (int64_t)kPassThreads + threadIdx.x;
        if (k < n) iisph3d_l1_one<float, true, false>(k, s, L, c, sc[s.scene_of(k)].dt);
        return;
    }
    const int half = threadIdx.x & 1;
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + (threadIdx.x >> 1);
    // the status word and the tile's header and ranges, loaded together
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    if (__syncthreads_or(err)) return;   // one decision for the whole block
    // owners past n_fluid (last tile) walk no entries but take part in the shuffles
    const bool valid = k < n_fluid;
    const int64_t kk = valid ? k : 0;
    const float4 pk = s.pos[kk], vk = s.vel[kk], ek = s.ext[kk];
    const float dt = sc[s.scene_of(kk)].dt;
    const FastSpline S(c.kern);
    Acc3<float, true> visc;
    Acc<float, true> rho;
    V3<float> vpart = v3<float>(0.f, 0.f, 0.f);
    float rpart = 0.f;
    const float gb = c.single_layer ? c.gamma1 : 1.f;
    auto pair = [&](const float4& pj, const float4& vj, float rj, bool bnd) {
        const V3<float> xij = sub3(pk, pj);
        const float r2 = r2_of(xij);
        float w, f;
        S.value_grad(r2, w, f);
        rpart = __fmaf_rn(bnd ? pj.w * gb : pj.w, w, rpart);
        if (rj != 0.f) {
            const float cf = __fdividef(pj.w * dot3(sub3(vk, vj), xij), rj * (r2 + c.visc_eps)) * f;
            vpart = fma3(cf, xij, vpart);
        }
    };
    auto flush = [&] {
        visc.add(vpart);
        rho.add(rpart);
        vpart = v3<float>(0.f, 0.f, 0.f);
        rpart = 0.f;
    };
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its two threads
        if (valid)
            walk_fallback_list<false>(L, k, half, [&](uint32_t j, bool bnd) {
                pair(s.pos[j], s.vel[j], s.rho_prev[j], bnd);
            }, flush);
    } else {
        float4* sp = tile_smem;
        float4* sv = tile_smem + T.cap;
        float* sr = reinterpret_cast<float*>(tile_smem + 2 * T.cap);
        __shared__ TileStage stg;
        const float4* src4[2] = {s.pos, s.vel};
        float4* dst4[2] = {sp, sv};
        const TileSlab slab = slab_at(tile_smem, 36, T.K, T.cap);
        stage_tile_async<2, false, !kL1GlobalEntries>(stg, d, h, rg, src4, dst4, s.rho_prev, sr, T, slab);
        const uint32_t cnt = kL1GlobalEntries ? T.count[kk] : 0u;
        uint2 ahead[AHEAD];
        prefetch_tile_list<kL1GlobalEntries>(T, h, k, half, ahead);
        if (!stage_tile_wait(stg, status)) return;
        if (valid)
            walk_tile_list<kL1GlobalEntries, false, AHEAD>(T, slab, k, cnt, half, ahead, [&](uint32_t off, bool bnd) {
                pair(at_offset(sp, off), at_offset(sv, off), at_offset(sr, off >> 2), bnd);
            }, flush);
    }
    const V3<float> vs = pair_total(visc);
    const float rk = pair_total(rho);
    if (half || !valid) return;
    s.p[k] = 0.f;
    const V3<float> npa = v3<float>(ek.x, ek.y - c.gravity, ek.z) + c.two_nu * vs;
    const V3<float> vstar = v3<float>(vk.x, vk.y, vk.z) + dt * npa;
    s.vstar[k] = v4<float>(vstar, 0.f);
    s.anp[k] = v4<float>(npa, 0.f);
    s.ext[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.rho[k] = rk;
}

// second loop: source term and diagonal element (single-pass a_ii), then
// the first pressure iteration, which needs no neighbor sums
// (iisph3d_first_iteration), with its part of the convergence scan
__global__ void __launch_bounds__(kPassThreads, kL2GlobalEntries ? 4 : 3) k_tile_iisph3d_l2(int64_t n_fluid, State<float> s, TileLists T,
                                                                  Lists L, SolverConsts<float> c,
                                                                  StepScalars* __restrict__ sc,
                                                                  int* __restrict__ status) {
    extern __shared__ float4 tile_smem[];
    const int half = threadIdx.x & 1;
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + (threadIdx.x >> 1);
    const bool valid = k < n_fluid;
    const int64_t kk = valid ? k : 0;
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    const int scene = s.scene_of(kk);
    if (__syncthreads_or(err)) return;   // one decision for the whole block
    const float dt = sc[scene].dt;
    ErrPart o;
    const float4 pk = s.pos[kk], vsk = s.vstar[kk];
    const float rk = s.rho[kk];
    const FastSpline S(c.kern);
    Acc<float, true> contrib, mg2;
    Acc3<float, true> mg, gb;
    float cpart = 0.f, g2part = 0.f;
    V3<float> mpart = v3<float>(0.f, 0.f, 0.f), bpart = v3<float>(0.f, 0.f, 0.f);
    const float wb = c.single_layer ? c.two_gamma : 2.f;
    auto pair = [&](const float4& pj, const float4& vsj, bool bnd) {
        const V3<float> xij = sub3(pk, pj);
        const float r2 = r2_of(xij);
        const float f = S.grad(r2);
        const float mf = pj.w * f;            // m_j gradW = mf d
        const V3<float> dv = bnd ? v3<float>(vsk.x, vsk.y, vsk.z) : sub3(vsk, vsj);
        cpart = __fmaf_rn(mf, dot3(dv, xij), cpart);
        if (!bnd) g2part = __fmaf_rn(mf * f, r2, g2part);
        else bpart = fma3(mf, xij, bpart);
        mpart = fma3(mf, xij, mpart);
    };
    auto flush = [&] {
        contrib.add(cpart);
        mg2.add(g2part);
        mg.add(mpart);
        gb.add(bpart);
        cpart = g2part = 0.f;
        mpart = bpart = v3<float>(0.f, 0.f, 0.f);
    };
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its two threads; the same sums
        // as a tiled owner's, so that gbnd is there for the pressure passes
        if (valid)
            walk_fallback_list<false>(L, k, half, [&](uint32_t j, bool bnd) { pair(s.pos[j], s.vstar[j], bnd); },
                                      flush);
    } else {
        float4* sp = tile_smem;
        float4* sa = tile_smem + T.cap;
        __shared__ TileStage stg;
        const float4* src4[2] = {s.pos, s.vstar};
        float4* dst4[2] = {sp, sa};
        const TileSlab slab = slab_at(tile_smem, 32, T.K, T.cap);
        stage_tile_async<2, false, !kL2GlobalEntries>(stg, d, h, rg, src4, dst4, nullptr, nullptr, T, slab);
        const uint32_t cnt = kL2GlobalEntries ? T.count[kk] : 0u;
        if (!stage_tile_wait(stg, status)) return;
        uint2 ahead[kL2Ahead];
        if (valid)
            walk_tile_list<kL2GlobalEntries, false, kL2Ahead>(T, slab, k, cnt, half, ahead, [&](uint32_t off, bool bnd) {
                pair(at_offset(sp, off), at_offset(sa, off), bnd);
            }, flush);
    }
    const float ct = pair_total(contrib), g2 = pair_total(mg2);
    const V3<float> m = pair_total(mg), gbt = pair_total(gb);
    // the inner sum of d_ii, -sum_fluid m_j gradW - lambda sum_bnd m_j gradW, from the two sums above
    const V3<float> in = v3<float>(__fmaf_rn(1.f - wb, gbt.x, -m.x), __fmaf_rn(1.f - wb, gbt.y, -m.y),
                                   __fmaf_rn(1.f - wb, gbt.z, -m.z));
    if (!half && valid) {
        const float source = (c.rest_density - rk) - dt * ct;
        const float diag = (c.inv_rho0_sq * dot(in, m) - (pk.w / c.rho0_sq) * g2) * (dt * dt);
        // sum_bnd m_j gradW for the pressure iterations, with the diagonal beside it
        // (one float4 read per owner instead of two in the update pass)
        s.gbnd[k] = v4<float>(gbt, diag);
        const float4 vs = make_float4(vsk.x, vsk.y, vsk.z, source);
        s.vstar[k] = vs;
        s.anp[k].w = diag;
        o = iisph3d_first_iteration<float>(k, s, c, dt, vs, diag);
    }
    reduce_err_parts(o, sc, scene);
}

// Blocks of the pressure passes with TPO threads per owner, and how many of
// them an SM holds (the register budget each is compiled for)
template <int TPO> constexpr int pressure_threads() { return kTileOwners * TPO; }
template <int TPO> constexpr int acc_blocks_per_sm() { return TPO == 1 ? 6 : (TPO == 2 ? 5 : 2); }
template <int TPO> constexpr int update_blocks_per_sm() { return TPO == 1 ? 4 : (TPO == 2 ? 4 : 2); }

// iteration (a): pressure acceleration
template <int AHEAD, int TPO>
__global__ void __launch_bounds__(pressure_threads<TPO>(), acc_blocks_per_sm<TPO>()) k_tile_iisph3d_pressure_acc(
    int64_t n_fluid, State<float> s, TileLists T, Lists L, SolverConsts<float> c, const StepScalars* __restrict__ sc,
    int* __restrict__ status) {
    static_assert(kPressureGlobalEntries, "the pressure passes read their entries from the global octet planes");
    extern __shared__ float4 tile_smem[];
    launch_dependents();   // the update pass may be scheduled while this grid runs
    const int half = threadIdx.x % TPO;   // this thread's share of the owner's entries
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + threadIdx.x / TPO;
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    // owners of scenes whose loop has ended take no part; a tile without
    // iterating owners ends at once
    const bool live = k < n_fluid && !sc[s.scene_of(k)].done;
    if (__syncthreads_or(err) || !__syncthreads_or(live)) return;
    const bool valid = live;
    const int64_t kk = valid ? k : 0;
    const float4 pk = s.pos[kk], gbk = s.gbnd[kk];
    const float prk = s.p[kk];
    const FastSpline S(c.kern);
    Acc3<float, true> pa;
    V3<float> part = v3<float>(0.f, 0.f, 0.f);
    auto pair = [&](const float4& pj, float prj) {
        const V3<float> xij = sub3(pk, pj);
        const float coef = pj.w * (prk + prj) * S.grad(r2_of(xij));
        part = fma3(-coef, xij, part);
    };
    auto flush = [&] {
        pa.add(part);
        part = v3<float>(0.f, 0.f, 0.f);
    };
    // boundary neighbors enter through sum_bnd m_j gradW (second loop), so
    // only the fluid candidates and entries are visited
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its threads
        if (valid)
            walk_fallback_list<true, TPO>(L, k, half, [&](uint32_t j, bool) { pair(s.pos[j], s.p[j]); }, flush);
    } else {
        float4* sp = tile_smem;
        float* sa = reinterpret_cast<float*>(tile_smem + T.cap);
        __shared__ TileStage stg;
        const float4* src4[1] = {s.pos};
        float4* dst4[1] = {sp};
        const TileSlab slab = slab_at(tile_smem, 20, T.K, T.cap);
        stage_tile_async<1, true, false>(stg, d, h, rg, src4, dst4, s.p, sa, T, slab);
        const uint32_t cnt = T.count[kk];
        OctetShare<TPO> ahead[AHEAD];
        prefetch_shares<TPO, AHEAD>(T, h, k, half, ahead);
        if (!stage_tile_wait(stg, status)) return;
        if (valid)
            walk_fluid_shares<TPO, AHEAD>(T, k, cnt, half, ahead, [&](uint32_t off) {
                pair(at_offset(sp, off), at_offset(sa, off >> 2));
            }, flush);
    }
    const V3<float> a = pair_total<TPO>(pa);
    if (half || !valid) return;
    // boundary: - sum_bnd (lambda m_j p_i / rho0^2) gradW, lambda = 2 gamma (single layer) or 2
    const float wb = (c.single_layer ? c.two_gamma : 2.f) * prk;
    s.acc[k] = v4<float>(c.inv_rho0_sq * (a - wb * v3<float>(gbk.x, gbk.y, gbk.z)), 0.f);
}

// iteration (b): A p, relaxed Jacobi update, density error, fused scan.
// Launched as a programmatic dependent of the acceleration pass: it reads
// what that pass does not write before waiting for it.
template <int AHEAD, int TPO>
__global__ void __launch_bounds__(pressure_threads<TPO>(), update_blocks_per_sm<TPO>()) k_tile_iisph3d_pressure_update(
    int64_t n_fluid, State<float> s, TileLists T, Lists L, SolverConsts<float> c, StepScalars* __restrict__ sc,
    int* __restrict__ status) {
    extern __shared__ float4 tile_smem[];
    launch_dependents();   // the convergence test may be scheduled while this grid runs
    const int half = threadIdx.x % TPO;   // this thread's share of the owner's entries
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + threadIdx.x / TPO;
    const int64_t kk = k < n_fluid ? k : 0;
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    const int scene = s.scene_of(kk);
    const StepScalars* q = sc + scene;
    const bool live = k < n_fluid && !q->done;
    if (__syncthreads_or(err) || !__syncthreads_or(live)) return;
    const float dt = q->dt;
    ErrPart o;
    // the owner's own data, loaded while the staging lands
    const bool valid = live;
    const float4 pk = s.pos[kk], vsk = s.vstar[kk], gbk = s.gbnd[kk];
    const float aii = gbk.w, prk = s.p[kk];   // gbnd.w: the diagonal (second loop)
    const uint32_t cnt = T.count[kk];
    grid_dependency_wait();   // the accelerations of this iteration
    const float4 ak = s.acc[kk];
    const FastSpline S(c.kern);
    Acc<float, true> ap;
    float part = 0.f;
    auto pair = [&](const float4& pj, const float4& aj) {
        const V3<float> xij = sub3(pk, pj);
        part = __fmaf_rn(pj.w * S.grad(r2_of(xij)), dot3(sub3(ak, aj), xij), part);
    };
    auto flush = [&] {
        ap.add(part);
        part = 0.f;
    };
    // boundary neighbors enter through sum_bnd m_j gradW (second loop)
    bool done = true;
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its threads
        if (valid)
            walk_fallback_list<true, TPO>(L, k, half, [&](uint32_t j, bool) { pair(s.pos[j], s.acc[j]); }, flush);
    } else {
        float4* sp = tile_smem;
        float4* sa = tile_smem + T.cap;
        __shared__ TileStage stg;
        const float4* src4[2] = {s.pos, s.acc};
        float4* dst4[2] = {sp, sa};
        const TileSlab slab = slab_at(tile_smem, 32, T.K, T.cap);
        stage_tile_async<2, true, false>(stg, d, h, rg, src4, dst4, nullptr, nullptr, T, slab);
        OctetShare<TPO> ahead[AHEAD];
        prefetch_shares<TPO, AHEAD>(T, h, k, half, ahead);
        done = stage_tile_wait(stg, status);
        if (done && valid)
            walk_fluid_shares<TPO, AHEAD>(T, k, cnt, half, ahead, [&](uint32_t off) {
                pair(at_offset(sp, off), at_offset(sa, off));
            }, flush);
    }
    if (done) {
        // boundary: sum_bnd m_j dot(a_i, gradW) = dot(a_i, sum_bnd m_j gradW)
        const float sum = pair_total<TPO>(ap) + dot3(v3<float>(ak.x, ak.y, ak.z), v3<float>(gbk.x, gbk.y, gbk.z));
        if (!half && valid)
            o = iisph3d_pressure_update_tail<float>(k, s, c, dt, v3<float>(ak.x, ak.y, ak.z), sum, vsk, aii, prk);
    }
    reduce_err_parts(o, sc, scene);
}

// ---------------------------------------------------------------------------
// SESPH 3D passes on tile lists (the fast-mode formulas of k_sesph_density
// and k_sesph_accel: SESPHFluidSolver3D.hpp:49-130). Same block layout as the
// IISPH passes; in a fallback tile the two threads of an owner split its
// 32-bit list, with the same pair arithmetic.
// ---------------------------------------------------------------------------

// density and pressure of the fluid owners: rho = sum_j m_j W, boundary
// neighbors weighted by gamma_1 in the single-layer model;
// p = max(k (rho / rho0 - 1), 0). p / rho^2 goes to the velocity's unused w
// component, where the acceleration pass finds it staged with the velocity.
template <int AHEAD>
__global__ void __launch_bounds__(kPassThreads, 5) k_tile_sesph3d_density(int64_t n_fluid, State<float> s,
                                                                          TileLists T, Lists L, SolverConsts<float> c,
                                                                          int* __restrict__ status) {
    extern __shared__ float4 tile_smem[];
    const int half = threadIdx.x & 1;
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + (threadIdx.x >> 1);
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    if (__syncthreads_or(err)) return;   // one decision for the whole block
    const bool valid = k < n_fluid;
    auto pressure_terms = [&](float r) {
        const float pr = c.stiffness * (r / c.rest_density - 1.f);
        const float p = (pr < 0.f) ? 0.f : pr;
        s.p[k] = p;
        s.vel[k].w = r == 0.f ? 0.f : fdiv<true>(p, r * r);
    };
    const int64_t kk = valid ? k : 0;
    const float4 pk = s.pos[kk];
    const FastSpline S(c.kern);
    const float gb = c.single_layer ? c.gamma1 : 1.f;
    Acc<float, true> rho;
    float part = 0.f;
    auto pair = [&](const float4& pj, bool bnd) {
        float w, f;
        S.value_grad(r2_of(sub3(pk, pj)), w, f);
        part = __fmaf_rn(bnd ? pj.w * gb : pj.w, w, part);
    };
    auto flush = [&] {
        rho.add(part);
        part = 0.f;
    };
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its two threads
        const uint32_t nn = valid ? L.size(k) : 0u;
        for (uint32_t q = half; q < nn; q += 2) {
            const uint32_t e = L.at(k, q);
            pair(s.pos[e & kIndexMask], (e & kBoundaryBit) != 0u);
            if ((q & 15u) >= 14u) flush();
        }
        flush();
    } else {
        float4* sp = tile_smem;
        __shared__ TileStage stg;
        const float4* src4[1] = {s.pos};
        float4* dst4[1] = {sp};
        const TileSlab none{nullptr, nullptr};
        stage_tile_async<1, false, false>(stg, d, h, rg, src4, dst4, nullptr, nullptr, T, none);
        const uint32_t cnt = T.count[kk];
        uint2 ahead[AHEAD];
        prefetch_tile_list<true>(T, h, k, half, ahead);
        if (!stage_tile_wait(stg, status)) return;
        if (valid)
            walk_tile_list<true, false, AHEAD>(T, none, k, cnt, half, ahead,
                                               [&](uint32_t off, bool bnd) { pair(at_offset(sp, off), bnd); }, flush);
    }
    const float r = pair_total(rho);
    if (half || !valid) return;
    s.rho[k] = r;
    pressure_terms(r);
}

// accelerations of the fluid owners: gravity + viscosity + pressure
// acceleration. Fluid j: -m_j (p_i / rho_i^2 + p_j / rho_j^2) gradW;
// boundary j: -m_i (2 p_i / rho_i^2) gradW, times gamma_2 in the single-layer
// model; viscosity over every j of non-zero density, as k_sesph_accel.
template <int AHEAD>
__global__ void __launch_bounds__(kPassThreads, 4) k_tile_sesph3d_accel(int64_t n_fluid, State<float> s,
                                                                        TileLists T, Lists L, SolverConsts<float> c,
                                                                        int* __restrict__ status) {
    extern __shared__ float4 tile_smem[];
    const int half = threadIdx.x & 1;
    const int64_t k = blockIdx.x * (int64_t)kTileOwners + (threadIdx.x >> 1);
    const TileDesc* d = T.desc + blockIdx.x;
    const int err = *status;
    const TileHead h = load_head(d);
    const TileRange rg = load_range(d, threadIdx.x);
    if (__syncthreads_or(err)) return;   // one decision for the whole block
    const bool valid = k < n_fluid;
    const int64_t kk = valid ? k : 0;
    const float4 pk = s.pos[kk], vk = s.vel[kk];
    const float rk = s.rho[kk], prk = s.p[kk];
    const FastSpline S(c.kern);
    const float pdd = rk == 0.f ? 0.f : prk / (rk * rk);
    // the boundary coefficient of gradW, the same for every boundary neighbor
    const float cb = -pk.w * (pdd + pdd) * (c.single_layer ? c.gamma2 : 1.f);
    Acc3<float, true> visc, pres;
    V3<float> vpart = v3<float>(0.f, 0.f, 0.f), ppart = v3<float>(0.f, 0.f, 0.f);
    auto pair = [&](const float4& pj, const float4& vj, float rj, bool bnd) {
        const V3<float> xij = sub3(pk, pj);
        const float r2 = r2_of(xij);
        const float f = S.grad(r2);
        if (rj != 0.f) {
            const float cf = __fdividef(pj.w * dot3(sub3(vk, vj), xij), rj * (r2 + c.visc_eps)) * f;
            vpart = fma3(cf, xij, vpart);
        }
        // vj.w: p_j / rho_j^2 (k_tile_sesph3d_density)
        const float cp = (bnd ? cb : -pj.w * (pdd + vj.w)) * f;
        ppart = fma3(cp, xij, ppart);
    };
    auto flush = [&] {
        visc.add(vpart);
        pres.add(ppart);
        vpart = v3<float>(0.f, 0.f, 0.f);
        ppart = v3<float>(0.f, 0.f, 0.f);
    };
    if (h.nranges == kTileFallback) {
        // the owner's 32-bit list, split between its two threads
        const uint32_t nn = valid ? L.size(k) : 0u;
        for (uint32_t q = half; q < nn; q += 2) {
            const uint32_t e = L.at(k, q);
            const uint32_t j = e & kIndexMask;
            pair(s.pos[j], s.vel[j], s.rho[j], (e & kBoundaryBit) != 0u);
            if ((q & 15u) >= 14u) flush();
        }
        flush();
    } else {
        float4* sp = tile_smem;
        float4* sv = tile_smem + T.cap;
        float* sr = reinterpret_cast<float*>(tile_smem + 2 * T.cap);
        __shared__ TileStage stg;
        const float4* src4[2] = {s.pos, s.vel};
        float4* dst4[2] = {sp, sv};
        const TileSlab none{nullptr, nullptr};
        stage_tile_async<2, false, false>(stg, d, h, rg, src4, dst4, s.rho, sr, T, none);
        const uint32_t cnt = T.count[kk];
        uint2 ahead[AHEAD];
        prefetch_tile_list<true>(T, h, k, half, ahead);
        if (!stage_tile_wait(stg, status)) return;
        if (valid)
            walk_tile_list<true, false, AHEAD>(T, none, k, cnt, half, ahead, [&](uint32_t off, bool bnd) {
                pair(at_offset(sp, off), at_offset(sv, off), at_offset(sr, off >> 2), bnd);
            }, flush);
    }
    const V3<float> vs = pair_total(visc);
    const V3<float> pa = pair_total(pres);
    if (half || !valid) return;
    const V3<float> npa = v3<float>(0.f, -c.gravity, 0.f) + c.two_nu * vs;
    s.acc[k] = v4<float>(pa + npa, 0.f);
}

// Export of the lists that the solver passes walk, as sorted indices: owner
// k's list length (out == nullptr) or its entries from out[offsets[k]]. A
// tile list entry is a staged slot, which the tile's ranges map back to a
// sorted index; fallback tiles and untiled contexts hold slot-major 32-bit
// lists (sorted index | kBoundaryBit).
__global__ void k_export_solver_lists(int64_t n_owners, bool tiled, TileLists T, Lists L,
                                      const int64_t* __restrict__ offsets, uint32_t* __restrict__ counts,
                                      uint32_t* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_owners) return;
    const TileDesc* d = T.desc + k / kTileOwners;
    const bool tile_list = tiled && d->h.nranges != kTileFallback;
    const uint32_t n = tile_list ? min(T.count[k] & 0xffffu, (uint32_t)T.K) : min(L.count[k], (uint32_t)L.K);
    if (out == nullptr) {
        counts[k] = n;
        return;
    }
    uint32_t* o = out + offsets[k];
    for (uint32_t q = 0; q < n; q++) {
        if (!tile_list) {
            o[q] = L.nbr[(int64_t)q * L.stride + k] & kIndexMask;   // without the boundary bit
            continue;
        }
        const uint4 oc = T.ent[(int64_t)(q / 8) * T.stride + k];
        const uint32_t wd = (q & 7) < 2 ? oc.x : (q & 7) < 4 ? oc.y : (q & 7) < 6 ? oc.z : oc.w;
        const uint32_t slot = ((wd >> ((q & 1) * 16)) & kEntOffset) >> 4;
        uint32_t idx = 0xf0000000u | slot;   // no range holds the slot: a broken list (the slot, for the report)
        for (uint32_t r = 0; r < d->h.nranges; r++) {
            const uint32_t lb = d->len_base[r], base = lb >> 16;
            if (slot - base < (lb & kRangeLen)) idx = d->start[r] + (slot - base);
        }
        o[q] = idx;
    }
}

// the instantiation of a tuned kernel for a prefetch depth in 1..kMaxAhead
#define FSB_AHEAD_SWITCH(ahead, KERNEL, ...)       \
    switch (ahead) {                                  \
        case 1: KERNEL<1> __VA_ARGS__; break;         \
        case 2: KERNEL<2> __VA_ARGS__; break;         \
        case 3: KERNEL<3> __VA_ARGS__; break;         \
        default: KERNEL<kMaxAhead> __VA_ARGS__; break; \
    }

// the pressure passes' instantiation for a prefetch depth and a number of
// threads per owner (1, 2, 4)
#define FSB_PRESSURE_SWITCH(ahead, tpo, KERNEL, CALL) \
    switch ((ahead) * 8 + (tpo)) {                   \
        case 1 * 8 + 1: CALL(KERNEL<1, 1>); break;    \
        case 2 * 8 + 1: CALL(KERNEL<2, 1>); break;    \
        case 3 * 8 + 1: CALL(KERNEL<3, 1>); break;    \
        case 4 * 8 + 1: CALL(KERNEL<4, 1>); break;    \
        case 1 * 8 + 4: CALL(KERNEL<1, 4>); break;    \
        case 2 * 8 + 4: CALL(KERNEL<2, 4>); break;    \
        case 3 * 8 + 4: CALL(KERNEL<3, 4>); break;    \
        case 4 * 8 + 4: CALL(KERNEL<4, 4>); break;    \
        case 1 * 8 + 2: CALL(KERNEL<1, 2>); break;    \
        case 2 * 8 + 2: CALL(KERNEL<2, 2>); break;    \
        case 3 * 8 + 2: CALL(KERNEL<3, 2>); break;    \
        default: CALL(KERNEL<4, 2>); break;           \
    }
static_assert(kMaxAhead == 4, "FSB_PRESSURE_SWITCH lists depths 1..4");

template <int AHEAD, int TPO> inline cudaError_t set_pressure_smem(int K) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_iisph3d_pressure_acc<AHEAD, TPO>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tile_pass_smem(20, K, false, kTileCapMax));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_iisph3d_pressure_update<AHEAD, TPO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_pass_smem(32, K, false, kTileCapMax));
    return e;
}

template <int AHEAD> inline cudaError_t set_tuned_pass_smem(int K) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_iisph3d_l1<AHEAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tile_pass_smem(36, K, !kL1GlobalEntries, kTileCapMax));
    if (e == cudaSuccess) e = set_pressure_smem<AHEAD, 1>(K);
    if (e == cudaSuccess) e = set_pressure_smem<AHEAD, 2>(K);
    if (e == cudaSuccess) e = set_pressure_smem<AHEAD, 4>(K);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_sesph3d_density<AHEAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_pass_smem(16, K, false, kTileCapMax));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_sesph3d_accel<AHEAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_pass_smem(36, K, false, kTileCapMax));
    return e;
}

inline cudaError_t set_tile_pass_smem(int K) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_iisph3d_l2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tile_pass_smem(32, K, !kL2GlobalEntries, kTileCapMax));
    if (e == cudaSuccess) e = set_tuned_pass_smem<1>(K);
    if (e == cudaSuccess) e = set_tuned_pass_smem<2>(K);
    if (e == cudaSuccess) e = set_tuned_pass_smem<3>(K);
    if (e == cudaSuccess) e = set_tuned_pass_smem<kMaxAhead>(K);
    return e;
}

}  // namespace fsb
