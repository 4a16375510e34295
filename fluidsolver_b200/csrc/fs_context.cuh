// Host-side context of one simulation (or one batch of scenes) on one GPU:
// device buffers, the stream, and the layout bookkeeping shared by the search
// and the solver phases.
//
// HBM layout (structure of arrays, all in the device's sorted order):
//   pos   V4: x, y, z, mass          vel  V4: x, y, z, -
//   acc   V4: MovementData acceleration (IISPH: pressure acceleration)
//   ext   V4: ExternalForces accumulator
//   rho, rho_prev, p   scalars (rho_prev: the density read by the viscosity term)
//   vstar V4: predicted velocity, w = source term
//   anp   V4: original non-pressure acceleration, w = diagonal element
//   err   scalar: predicted density error
//   type  uint8, hidx uint32 (host index of the particle at this position)
// Sorted order puts fluid particles first, then boundary particles, then the
// inactive particles a contract still lists, then excluded inactive ones,
// each block in linear cell order, x fastest (a single block in the
// reference-order mode). Fluid-only phases run over [0, n_fluid).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fs_common.cuh"
#include "fs_entities.cuh"
#include "fs_sort.cuh"
#include "fs_tiles.cuh"

struct fs_ctx {
    fs_params prm{};
    int dim = 3;
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t cap = 0;          // particle capacity
    int64_t n = 0;            // particles uploaded
    int64_t n_fluid = 0, n_boundary = 0, n_inactive = 0;
    int64_t n_struct = 0;     // particles that take part in the cell structure
    bool have_state = false;
    bool have_lists = false;
    bool have_cells = false;        // cell tables describe the current sorted order
    float searched_dt = 0.f;
    bool reference_order = false;
    bool include_inactive = false;  // contract lists inactive particles (2D quadratic / hashed)
    bool truncate_cells = false;    // hashed-2D cells (reference-order mode)
    bool sort_lists_by_host = false;  // quadratic list order (reference-order mode)
    int ns_owner_mode = 0;          // 0 all in structure, 1 fluid only, 2 active only
    int precision = FS_PRECISION_FP32_KAHAN;
    fsb::TileTuning tuning;         // prefetch depths of the tile passes (fs_autotune)
    size_t real_size = 4;

    // derived constants (float, computed exactly as the reference does)
    float search_radius = 0.f;   // particle_size * 2
    float radius2 = 0.f;         // search_radius * search_radius
    float kernel_h = 0.f;        // kernel_support / 2
    float kernel_alpha = 0.f;

    // state, double-buffered for the reorder gather
    void* pos[2] = {};
    void* vel[2] = {};
    void* acc[2] = {};
    void* ext[2] = {};
    void* rho[2] = {};
    void* p[2] = {};
    uint8_t* type[2] = {};
    uint32_t* hidx[2] = {};
    uint16_t* scene_of[2] = {};      // per-particle scene (batched contexts only)
    int cur = 0;
    void* rho_prev = nullptr;
    void* vstar = nullptr;
    void* anp = nullptr;
    void* err = nullptr;
    void* gbnd = nullptr;     // V4: sum over boundary neighbors of m_j gradW, w: diagonal (tile passes)

    // search
    uint32_t* keys[2] = {};
    unsigned long long* keys64[2] = {};
    uint32_t* perm[2] = {};
    // the 2D hashed grid's history in the reference-order mode, per HOST index
    // (HashedNeighborhoodSearch.cpp:117-151 keeps each cell's particles in
    // order of arrival): the particle's last cell and its rank in the sorted
    // order of that cell (0xffffffff: no cell yet, it arrives at the next search)
    int2* h2d_cell = nullptr;
    uint32_t* h2d_rank = nullptr;
    int64_t h2d_n = -1;               // particle count the history belongs to
    uint32_t* sort_hist = nullptr;    // per-tile digit counts of the radix sort (fs_sort.cuh)
    // compact hashing (2D): the hashed table of occupied cells instead of the dense grid
    fsb::HashCell* hash_table = nullptr;
    uint32_t hash_mask = 0;           // slots - 1 (a power of two, >= 2 x capacity)
    uint32_t* cell_start = nullptr;   // [regions][cells + 1] first sorted index of cell >= c
    uint32_t* cell_partials = nullptr;  // tile totals of the cell table's scan
    int64_t cells = 0;                // dims[0] * dims[1] * dims[2]
    int key_bits = 30;                // bits of the linear cell index in the sort keys
    int64_t cell_alloc = 0;           // entries allocated per table
    int regions = 2;                  // regions in the sorted layout
    int dims[3] = {1, 1, 1};       // scene 0's grid dims
    int* bbox = nullptr;           // device: per scene min xyz [3 scenes], then max xyz [3 scenes]
    fsb::SceneGrid* grids = nullptr;            // device: per-scene grids (origins set every step)
    std::vector<fsb::SceneGrid> grids_host;     // dims and bases
    uint32_t* nbr = nullptr;       // solver lists, slot-major: nbr[s * nbr_stride + k]
    fsb::TileDesc* tile_desc = nullptr;  // tile lists (3D IISPH fast path): per tile of owners
    uint4* tile_ent = nullptr;           // [K / 8][tile_stride] octets of 16-bit entries
    int64_t tile_stride = 0;             // owners per octet plane (tiles * kTileOwners)
    uint32_t* nbr_count = nullptr;
    int nbr_capacity = 0;          // K
    int64_t nbr_stride = 0;
    int64_t n_owners = 0;          // owners of the solver lists: [0, n_owners)
    int64_t launches = 0;          // this library's kernel launches

    // CSR export of the last search (sorted space)
    int64_t* csr_offsets = nullptr;
    uint32_t* csr_indices = nullptr;
    int64_t csr_capacity = 0;
    uint32_t* csr_counts = nullptr;

    // staging for host transfers
    void* staging = nullptr;
    size_t staging_bytes = 0;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;

    int* status = nullptr;                  // device status word
    unsigned long long* small_stamps = nullptr;  // phase boundaries of the small-scene kernel's last step (ns)
    bool small_last = false;                // the last steps ran in the small-scene kernel
    int small_blocks = 0;                   // the blocks of its last launch
    fsb::StatsPart* stats_parts = nullptr;  // global statistics: per-block partials and the result
    fsb::StatsOut* stats_out = nullptr;
    fsb::StepScalars* scalars = nullptr;    // device
    fsb::StepScalars* scalars_host = nullptr;  // pinned mirror

    // CUDA graphs of the solver phases (the IISPH loop is a conditional WHILE
    // node inside), one per buffer assignment they were captured with
    struct SolveGraph {
        int cur = 0;
        void *rho0 = nullptr, *rho1 = nullptr, *rho_prev = nullptr;
        int K = 0;
        int64_t n = 0, n_owners = 0;
        float dt = 0.f;
        bool with_search = false;
        int64_t cells = 0;
        int dims0 = 0, dims1 = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
        int post_cur = 0;
        void *post_rho0 = nullptr, *post_rho1 = nullptr, *post_rho_prev = nullptr;
        bool same_key(const SolveGraph& o) const {
            return cur == o.cur && rho0 == o.rho0 && rho1 == o.rho1 && rho_prev == o.rho_prev && K == o.K &&
                   n == o.n && n_owners == o.n_owners && dt == o.dt && with_search == o.with_search &&
                   cells == o.cells && dims0 == o.dims0 && dims1 == o.dims1;
        }
    };
    std::vector<SolveGraph> solve_graphs;
    cudaStream_t body_stream = nullptr;  // captures conditional-node bodies

    cudaEvent_t ev[6] = {};
    float phase_ms[5] = {};

    // batched scenes (0: a single-scene context)
    int32_t scenes = 0;
    std::vector<int64_t> scene_offsets;   // host particles of scene s: [offsets[s], offsets[s+1])
    int64_t* d_scene_offsets = nullptr;
    int nsc() const { return scenes > 0 ? scenes : 1; }
};
