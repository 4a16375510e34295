// The search's sort, written for its keys: a stable least-significant-digit
// radix sort of (key, value) pairs, and the cell-start table read straight
// off the sorted keys.
//
// The reference sorts its particle collection with a quick sort over 64-bit
// Morton keys that permutes every component through ParticleCollection::swap
// (ParticleCollectionAlgorithm.hpp:28-133). Here the keys are the bounded
// (region, linear cell) indices of fs_search.cuh (key_bits + 2 bits; in the
// reference-order mode 32 more bits of order within a cell), the values the
// particles' current positions in the array, and the permutation is applied
// afterwards by one gather of every field (k_reorder).
//
// One pass per 8-bit digit, three kernels each:
//   k_sort_hist     per-tile digit counts, stored digit-major (hist[d][tile]);
//   k_sort_rowscan  one block per digit turns its row into exclusive offsets
//                   over the tiles and stores the digit's total;
//   k_sort_scatter  every tile takes the digits' first slots (a scan of the
//                   256 totals) plus its row offsets, ranks its keys per digit
//                   in input order (warps own consecutive 128-key runs and
//                   count with match_any) and writes each pair to its slot.
// Tiles are 1,024 consecutive keys (8 warps x 32 lanes x 4). Because ranks
// follow input order within a tile and the slots follow tile order, every
// pass is stable, which makes the whole sort stable: keys that compare equal
// keep their input order. The searches feed it the previous step's sorted
// order, so a particle that stays in its cell keeps its place among the
// cell's particles from step to step.
#pragma once

#include <algorithm>

#include "fs_common.cuh"

namespace fsb {

constexpr int kSortWarps = 8;
constexpr int kSortThreads = 32 * kSortWarps;
constexpr int kSortPerLane = 4;   // 1,024-key tiles: enough blocks to fill the SMs at a million keys
constexpr int kSortWarpKeys = 32 * kSortPerLane;            // consecutive keys per warp
constexpr int kSortTile = kSortWarps * kSortWarpKeys;       // consecutive keys per block
constexpr int kSortDigits = 256;

inline int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }
// entries of the per-tile histogram matrix, followed by the 256 digit totals
inline int64_t sort_hist_entries(int64_t n) {
    return (int64_t)kSortDigits * std::max<int64_t>(sort_tiles(n), 1) + kSortDigits;
}

template <typename K> __device__ __forceinline__ uint32_t digit_of(K key, int shift) {
    return (uint32_t)(key >> shift) & (kSortDigits - 1u);
}

// hist[d * tiles + t] = keys of tile t whose digit at `shift` is d
template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(int64_t n, const K* FSB_R keys, int shift,
                                                            int64_t tiles, uint32_t* FSB_R hist) {
    __shared__ uint32_t h[kSortDigits];
    h[threadIdx.x] = 0u;
    __syncthreads();
    const int64_t base = blockIdx.x * (int64_t)kSortTile;
    const int lane = threadIdx.x & 31;
#pragma unroll 4
    for (int r = 0; r < kSortTile / kSortThreads; r++) {
        const int64_t i = base + r * kSortThreads + threadIdx.x;
        const bool v = i < n;
        const uint32_t d = v ? digit_of<K>(keys[i], shift) : 0u;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (v) {
            // one shared-memory atomic per run of equal digits in the warp
            const unsigned peers = __match_any_sync(act, d);
            if (lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Row d of the histogram matrix (block d) into exclusive offsets over the
// tiles, in place; totals[d] = the digit's keys in all tiles.
static __global__ void __launch_bounds__(kSortThreads) k_sort_rowscan(uint32_t* FSB_R hist, int64_t tiles,
                                                               uint32_t* FSB_R totals) {
    __shared__ uint32_t s_warp[kSortWarps];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t* row = hist + (int64_t)blockIdx.x * tiles;
    uint32_t carry = 0u;
    for (int64_t a = 0; a < tiles; a += kSortThreads) {
        const int64_t i = a + t;
        const uint32_t v = i < tiles ? row[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[w] = incl;
        __syncthreads();
        uint32_t before = 0u, chunk = 0u;
#pragma unroll
        for (int q = 0; q < kSortWarps; q++) {
            const uint32_t x = s_warp[q];
            if (q < w) before += x;
            chunk += x;
        }
        if (i < tiles) row[i] = carry + before + incl - v;
        carry += chunk;
        __syncthreads();
    }
    if (t == 0) totals[blockIdx.x] = carry;
}

// Exclusive scan of m counts by one block of 1024 threads (each scans a
// contiguous run, the runs' sums are scanned across the block); used for
// list exports and small cell tables. out may alias in when both have one
// type. Every thread of the block calls scan_exclusive_block.
template <typename In, typename Out>
__device__ __forceinline__ void scan_exclusive_block(const In* in, Out* out, int64_t m) {
    __shared__ Out s_warp[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t per = (m + 1023) / 1024;
    const int64_t lo = min(m, (int64_t)t * per), hi = min(m, lo + per);
    Out sum = 0;
    for (int64_t i = lo; i < hi; i++) sum += (Out)in[i];
    // inclusive warp scan, then the warps' totals
    Out incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Out y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        Out x = s_warp[lane];
        Out xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Out y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        s_warp[lane] = xi - x;   // exclusive over warps
    }
    __syncthreads();
    Out run = s_warp[w] + incl - sum;
    for (int64_t i = lo; i < hi; i++) {
        const Out v = (Out)in[i];
        out[i] = run;
        run += v;
    }
}
template <typename In, typename Out>
__global__ void __launch_bounds__(1024) k_scan_exclusive(const In* in, Out* out, int64_t m) {
    scan_exclusive_block<In, Out>(in, out, m);
}

// Scatters tile blockIdx.x of (kin, vin) to its slots: slot of a key =
// (keys of smaller digits, from totals) + offs[d * tiles + tile] (the row
// scan of k_sort_hist) + keys of digit d before it in the tile. Warp w ranks
// its own 128 consecutive keys, 32 at a time in lane order, with a per-warp
// counter per digit; then the counters turn into each warp's first slot per
// digit.
template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(int64_t n, const K* FSB_R kin,
                                                               const uint32_t* FSB_R vin, K* FSB_R kout,
                                                               uint32_t* FSB_R vout, int shift, int64_t tiles,
                                                               const uint32_t* FSB_R offs,
                                                               const uint32_t* FSB_R totals) {
    __shared__ uint32_t wh[kSortWarps][kSortDigits];
    __shared__ uint32_t s_base[kSortWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // first slot of every digit: exclusive scan of the totals (thread d: digit d)
    uint32_t digit_base;
    {
        const uint32_t v = totals[threadIdx.x];
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_base[w] = incl;
        __syncthreads();
        uint32_t before = 0u;
#pragma unroll
        for (int q = 0; q < kSortWarps; q++)
            if (q < w) before += s_base[q];
        digit_base = before + incl - v;
    }
    for (int d = lane; d < kSortDigits; d += 32) wh[w][d] = 0u;
    __syncwarp();
    const int64_t base = blockIdx.x * (int64_t)kSortTile + (int64_t)w * kSortWarpKeys;
    const unsigned below = (1u << lane) - 1u;
    K key[kSortPerLane];
    uint32_t val[kSortPerLane], rank[kSortPerLane];
#pragma unroll
    for (int j = 0; j < kSortPerLane; j++) {
        const int64_t i = base + j * 32 + lane;
        const bool v = i < n;
        key[j] = v ? kin[i] : K(0);
        val[j] = v ? vin[i] : 0u;
        rank[j] = 0u;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (v) {
            const uint32_t d = digit_of<K>(key[j], shift);
            const unsigned peers = __match_any_sync(act, d);
            const uint32_t before = wh[w][d];
            __syncwarp(act);   // every peer has read the counter before the leader moves it
            rank[j] = before + (uint32_t)__popc(peers & below);
            if (lane == __ffs(peers) - 1) wh[w][d] = before + (uint32_t)__popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: the tile's first slot, then each warp's, in warp order
    {
        const int d = threadIdx.x;
        uint32_t run = digit_base + offs[(int64_t)d * tiles + blockIdx.x];
#pragma unroll
        for (int q = 0; q < kSortWarps; q++) {
            const uint32_t c = wh[q][d];
            wh[q][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortPerLane; j++) {
        const int64_t i = base + j * 32 + lane;
        if (i < n) {
            const uint32_t pos = wh[w][digit_of<K>(key[j], shift)] + rank[j];
            kout[pos] = key[j];
            vout[pos] = val[j];
        }
    }
}

// Cell-start table from the sorted keys of the particles in the structure
// ([0, n_struct)). Entry t of the concatenated per-region tables (region g,
// cell c at t = g (cells + 1) + c; entry g (cells + 1) + cells ends region
// g) is the first sorted index whose key's entry is >= t: the exclusive scan
// of the per-entry counts. k_cell_counts writes, for the first particle of
// every run of equal keys, the run's length (the table is zeroed before);
// the scan runs in place.
template <typename K>
__device__ __forceinline__ void cell_count_at(int64_t k, int64_t n_struct, const K* FSB_R keys, int key_shift,
                                              int key_bits, int64_t cells, uint32_t* FSB_R counts) {
    const uint32_t key = (uint32_t)(keys[k] >> key_shift);
    if (k > 0 && (uint32_t)(keys[k - 1] >> key_shift) == key) return;
    int64_t e = k + 1;
    while (e < n_struct && (uint32_t)(keys[e] >> key_shift) == key) e++;
    counts[(int64_t)(key >> key_bits) * (cells + 1) + (key & ((1u << key_bits) - 1u))] = (uint32_t)(e - k);
}
template <typename K>
__global__ void k_cell_counts(int64_t n_struct, const K* FSB_R keys, int key_shift, int key_bits,
                              int64_t cells, uint32_t* FSB_R counts) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n_struct) return;
    cell_count_at<K>(k, n_struct, keys, key_shift, key_bits, cells, counts);
}

// Device-wide exclusive scan of m counts, in place, in three launches:
// k_scan_tiles scans every tile of kScanTile entries and stores the tile's
// total, one block scans the totals (k_scan_exclusive), k_scan_add adds each
// tile's offset.
constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 8;
constexpr int kScanTile = kScanThreads * kScanPerThread;
inline int64_t scan_tiles(int64_t m) { return (m + kScanTile - 1) / kScanTile; }
constexpr int64_t kSmallScanMax = 65536;   // tables scanned by one block in one launch

static __global__ void __launch_bounds__(kScanThreads) k_scan_tiles(uint32_t* FSB_R a, int64_t m,
                                                             uint32_t* FSB_R partials) {
    __shared__ uint32_t tile[kScanTile];
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t base = blockIdx.x * (int64_t)kScanTile;
    for (int i = t; i < kScanTile; i += kScanThreads) tile[i] = base + i < m ? a[base + i] : 0u;
    __syncthreads();
    uint32_t v[kScanPerThread], sum = 0u;
#pragma unroll
    for (int j = 0; j < kScanPerThread; j++) {
        v[j] = tile[t * kScanPerThread + j];
        sum += v[j];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        const uint32_t x = s_warp[lane];
        uint32_t xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        s_warp[lane] = xi - x;
        if (lane == 31) partials[blockIdx.x] = xi;
    }
    __syncthreads();
    uint32_t run = s_warp[w] + incl - sum;
#pragma unroll
    for (int j = 0; j < kScanPerThread; j++) {
        tile[t * kScanPerThread + j] = run;
        run += v[j];
    }
    __syncthreads();
    for (int i = t; i < kScanTile; i += kScanThreads)
        if (base + i < m) a[base + i] = tile[i];
}

static __global__ void k_scan_add(uint32_t* FSB_R a, int64_t m, const uint32_t* FSB_R partials) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        a[i] += partials[i / kScanTile];
}

// the cell-start table of n_struct sorted keys: zero, count, scan in place;
// partials holds scan_tiles(table) entries
template <typename K>
inline void cell_start_table(int64_t n_struct, const K* keys, int key_shift, int key_bits, int64_t cells,
                             int64_t table, uint32_t* cell_start, uint32_t* partials, int block, cudaStream_t st,
                             int64_t& launches) {
    cudaMemsetAsync(cell_start, 0, sizeof(uint32_t) * (size_t)table, st);
    if (n_struct > 0)
        k_cell_counts<K><<<(unsigned)((n_struct + block - 1) / block), block, 0, st>>>(n_struct, keys, key_shift,
                                                                                       key_bits, cells, cell_start);
    if (table <= kSmallScanMax) {   // small tables: one block, one launch
        k_scan_exclusive<uint32_t, uint32_t><<<1, 1024, 0, st>>>(cell_start, cell_start, table);
        launches += 2;
        return;
    }
    const int64_t tiles = scan_tiles(table);
    k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(cell_start, table, partials);
    k_scan_exclusive<uint32_t, uint32_t><<<1, 1024, 0, st>>>(partials, partials, tiles);
    k_scan_add<<<(unsigned)std::min<int64_t>((table + 255) / 256, 148 * 8), 256, 0, st>>>(cell_start, table, partials);
    launches += 4;
}

// Small sorts (n <= kSmallSortMax, e.g. a 2D dam of a few thousand
// particles) in one block and one launch: the same stable passes, with the
// keys in shared memory between them, so that a scene whose whole step lasts
// a few microseconds does not pay three launches per digit. 32 warps own 128
// consecutive keys each; the result lands in buffer 1.
constexpr int kSmallSortThreads = 1024;
constexpr int kSmallSortWarps = kSmallSortThreads / 32;
constexpr int kSmallSortPerLane = 4;
constexpr int kSmallSortMax = kSmallSortThreads * kSmallSortPerLane;
template <typename K> constexpr size_t small_sort_smem() {
    return (size_t)2 * kSmallSortMax * (sizeof(K) + sizeof(uint32_t)) + (size_t)kSmallSortWarps * kSortDigits * 4;
}

// the whole small sort by one block of kSmallSortThreads threads;
// sort_smem: small_sort_smem<K>() bytes of shared memory
template <typename K>
__device__ __forceinline__ void sort_small_block(int64_t n, int bits, const K* FSB_R kin, const uint32_t* FSB_R vin,
                                                 K* FSB_R kout, uint32_t* FSB_R vout, unsigned char* sort_smem) {
    K* sk[2] = {reinterpret_cast<K*>(sort_smem), reinterpret_cast<K*>(sort_smem) + kSmallSortMax};
    uint32_t* sv[2] = {reinterpret_cast<uint32_t*>(sk[1] + kSmallSortMax),
                       reinterpret_cast<uint32_t*>(sk[1] + kSmallSortMax) + kSmallSortMax};
    uint32_t(*wh)[kSortDigits] = reinterpret_cast<uint32_t(*)[kSortDigits]>(sv[1] + kSmallSortMax);
    __shared__ uint32_t s_tot[kSortDigits / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int i = t; i < n; i += kSmallSortThreads) {
        sk[0][i] = kin[i];
        sv[0][i] = vin[i];
    }
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        for (int d = lane; d < kSortDigits; d += 32) wh[w][d] = 0u;
        __syncthreads();
        uint32_t rank[kSmallSortPerLane];
#pragma unroll
        for (int j = 0; j < kSmallSortPerLane; j++) {
            const int i = w * (32 * kSmallSortPerLane) + j * 32 + lane;
            const bool v = i < n;
            rank[j] = 0u;
            const unsigned act = __ballot_sync(0xffffffffu, v);
            if (v) {
                const uint32_t d = digit_of<K>(sk[cur][i], shift);
                const unsigned peers = __match_any_sync(act, d);
                const uint32_t before = wh[w][d];
                __syncwarp(act);
                rank[j] = before + (uint32_t)__popc(peers & below);
                if (lane == __ffs(peers) - 1) wh[w][d] = before + (uint32_t)__popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        // per digit (threads 0..255): its total over the warps, the digits'
        // exclusive scan, then each warp's first slot
        uint32_t total = 0u, incl = 0u;
        if (t < kSortDigits) {
            for (int q = 0; q < kSmallSortWarps; q++) total += wh[q][t];
            incl = total;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) s_tot[w] = incl;
        }
        __syncthreads();
        if (t < kSortDigits) {
            uint32_t run = incl - total;
            for (int q = 0; q < w; q++) run += s_tot[q];
            for (int q = 0; q < kSmallSortWarps; q++) {
                const uint32_t c = wh[q][t];
                wh[q][t] = run;
                run += c;
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSmallSortPerLane; j++) {
            const int i = w * (32 * kSmallSortPerLane) + j * 32 + lane;
            if (i < n) {
                const K key = sk[cur][i];
                const uint32_t pos = wh[w][digit_of<K>(key, shift)] + rank[j];
                sk[cur ^ 1][pos] = key;
                sv[cur ^ 1][pos] = sv[cur][i];
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    for (int i = t; i < n; i += kSmallSortThreads) {
        kout[i] = sk[cur][i];
        vout[i] = sv[cur][i];
    }
}
template <typename K>
__global__ void __launch_bounds__(kSmallSortThreads) k_sort_small(int64_t n, int bits, const K* FSB_R kin,
                                                                  const uint32_t* FSB_R vin,
                                                                  K* FSB_R kout, uint32_t* FSB_R vout) {
    extern __shared__ __align__(16) unsigned char sort_smem[];
    sort_small_block<K>(n, bits, kin, vin, kout, vout, sort_smem);
}

// the small sort's shared memory, set once per process and device
inline cudaError_t prepare_small_sort() {
    cudaError_t e = cudaFuncSetAttribute(k_sort_small<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)small_sort_smem<uint32_t>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sort_small<unsigned long long>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)small_sort_smem<unsigned long long>());
    return e;
}

// Sorts n (key, value) pairs over bits [0, bits) with the passes above,
// ping-ponging between buffers 0 and 1 of keys and vals (or, for n <=
// kSmallSortMax, in one block). Returns the buffer that holds the result.
// hist holds sort_hist_entries(n) counters (capacity for at least n keys).
template <typename K>
inline int sort_pairs(int64_t n, int bits, K* const (&keys)[2], uint32_t* const (&vals)[2], uint32_t* hist,
                      cudaStream_t st, int64_t& launches) {
    const int64_t tiles = sort_tiles(n);
    uint32_t* totals = hist + (int64_t)kSortDigits * tiles;
    int cur = 0;
    if (n <= 1) return cur;
    if (n <= kSmallSortMax) {
        k_sort_small<K><<<1, kSmallSortThreads, small_sort_smem<K>(), st>>>(n, bits, keys[0], vals[0], keys[1], vals[1]);
        launches += 1;
        return 1;
    }
    for (int shift = 0; shift < bits; shift += 8) {
        k_sort_hist<K><<<(unsigned)tiles, kSortThreads, 0, st>>>(n, keys[cur], shift, tiles, hist);
        k_sort_rowscan<<<kSortDigits, kSortThreads, 0, st>>>(hist, tiles, totals);
        k_sort_scatter<K><<<(unsigned)tiles, kSortThreads, 0, st>>>(n, keys[cur], vals[cur], keys[cur ^ 1],
                                                                    vals[cur ^ 1], shift, tiles, hist, totals);
        launches += 3;
        cur ^= 1;
    }
    return cur;
}

}  // namespace fsb
