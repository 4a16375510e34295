// The small-scene step: whole steps (search and solver) of a scene of at most
// kSmallMax particles in one kernel launch of one thread-block cluster, for
// as many steps as the caller asks.
//
// A scene of a few thousand particles (the 2D dams of libFluid's scenarios)
// does a few microseconds of work per phase, so the step-by-step path of
// separate kernels is bound by launch and dependency latency (about twenty
// kernels per step). Here a cluster of up to kSmallMaxCtas blocks of
// kSmallThreads threads (one block per SM, about kSmallPerCta particles per
// block) runs the same phases in the same order -- the same per-particle
// device functions as the separate kernels, so the results are the same bit
// for bit -- with a cluster barrier between phases, and loops over the steps
// inside the kernel. The phases read what earlier phases of the same launch
// wrote, so this translation unit is compiled with coherent loads only
// (FSB_COHERENT_LOADS).
//
// Not covered (the separate kernels serve them): batched contexts, the tile
// lists of the 3D fast mode, compact hashing, host-driven pressure loops.
#pragma once

#include "fs_common.cuh"
#include "fs_search.cuh"
#include "fs_solvers.cuh"

namespace fsb {

constexpr int kSmallThreads = 512;
constexpr int kSmallMaxCtas = 16;   // CTAs of the launch's cluster at most (one per SM)
constexpr int kSmallPerCta = 256;   // particles per CTA the launch aims at
constexpr int64_t kSmallMax = 4096;             // particles at most (the sort words' 12-bit index field)
constexpr int64_t kSmallMaxTable = 1 << 18;     // cell-table entries of a scene the kernel takes (sort keys of at most 40 bits)

// one set of the double-buffered particle fields (the search's reordering
// gathers from one into the other)
struct SmallBuffers {
    void *pos, *vel, *acc, *ext, *rho, *p;
    uint8_t* type;
    uint32_t* hidx;
};

enum SmallSolver { kSmallSESPH = 0, kSmallIISPH3D = 1, kSmallIISPH2D = 2 };

template <typename R> struct SmallStepArgs {
    int steps;
    int dim;
    bool split;         // the reference-order first loop (separate density pass)
    bool fp32;          // FP32 without compensation: two-pass diagonal, float convergence test
    int64_t n, n_struct, n_owners;
    int cur;            // buffer set holding the state at the start
    SmallBuffers buf[2];
    R* rho_prev;        // the third density buffer (IISPH swaps it with the current one every step)
    void *vstar, *anp, *err, *gbnd;
    // search
    bool include_inactive, single_region, trunc, rows, sort_by_host;
    float radius, radius2;
    int key_bits, regions;
    int64_t cells;
    SceneGrid* grids;
    int* bbox;
    uint32_t* keys[2];
    unsigned long long* keys64[2];   // the reference-order mode's 64-bit keys, else null
    uint32_t* perm[2];
    int2* h2d_cell;                  // the 2D hashed grid's history, else null
    uint32_t* h2d_rank;
    uint32_t* cell_start;
    uint32_t owner_mask;
    uint32_t* nbr;
    uint32_t* count;
    int64_t stride;
    int K;
    // solver
    SolverConsts<R> c;
    StepScalars* sc;
    int* status;
    float desired_dt;
    bool dynamic_generator;
    float particle_size, min_ts, max_ts, lambda_v, lambda_a, cfl_timestep;
    int min_it, max_it;
    float max_err;
    unsigned long long* stamps;      // 6 phase boundaries of the last step (ns, %globaltimer)
    bool stage;                      // set by launch_small_steps: the gathered fields fit in shared memory
    bool stage_lists;                // and so do the lists of each CTA's owners (with the fields)
};

// Shared memory of the gathered fields' copies (positions from the lists to
// the integration; per phase one more float4 field and two scalar fields),
// of the lists and counts of a CTA's share of the owners (share owners, K
// entries each) after them, and the most a block takes.
template <typename R> constexpr size_t small_stage_bytes(int64_t n) {
    return (size_t)((n + 3) & ~int64_t(3)) * (2 * sizeof(V4<R>) + 2 * sizeof(R));
}
constexpr size_t small_list_bytes(int64_t share, int K) { return (size_t)share * ((size_t)K + 1) * 4; }
constexpr size_t kSmallStageMax = 220 * 1024;

// shared memory the kernel needs without the staged fields
size_t small_steps_smem();

// enqueues a.steps steps on st; SOLVER is a SmallSolver
// (blocks: the cluster's blocks it chose)
template <typename R, bool KAHAN, int SOLVER>
cudaError_t launch_small_steps(const SmallStepArgs<R>& a, cudaStream_t st, int* blocks);

}  // namespace fsb
