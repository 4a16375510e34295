/*
 * fluidsolver_b200 -- C-ABI of the B200 implementation of libFluid's
 * per-timestep hot path: the neighborhood search and the SESPH / IISPH steps
 * in 2D and 3D.
 *
 * The boundary replaces these reference interfaces (paths relative to the
 * FluidSolver repository):
 *   - IFluidSolverBase::execute_neighborhood_search / execute_simulation_step
 *     (src/libFluid/fluidSolver/IFluidSolver.hpp:16-34), as implemented by
 *     SESPHFluidSolver (solver/SESPHFluidSolver.hpp:49-111),
 *     SESPHFluidSolver3D (solver/SESPHFluidSolver3D.hpp:49-130),
 *     IISPHFluidSolver (solver/IISPHFluidSolver.hpp:139-188) and
 *     IISPHFluidSolver3D (solver/IISPHFluidSolver3D.hpp:120-562);
 *   - the neighborhood-search concept (IFluidSolver.hpp:36-73): find_neighbors,
 *     get_neighbors(index), get_neighbors(position) of
 *     QuadraticNeighborhoodSearchDynamicAllocated, HashedNeighborhoodSearch,
 *     QuadraticNeighborhoodSearch3D, HashedNeighborhoodSearch3D,
 *     CompressedNeighborhoodSearch and CompactHashingNeighborhoodSearch;
 *   - the particle-collection components the path reads and writes
 *     (fluidSolver/Particle.hpp:15-50, ParticleCollection.hpp:11-177).
 *
 * Conventions
 *   - Every function returns an fs_status; FS_OK is 0. fs_last_error() gives a
 *     one-line message for the last failure on the calling thread.
 *   - A context owns one CUDA stream on one device; all work is ordered on it
 *     and every call that returns data to the host synchronises that stream.
 *   - Particle arrays passed in or out are dense, in the caller's index order
 *     ("host order"): vectors hold `dim` floats per particle. The device keeps
 *     its own spatially sorted order internally; indices that cross the
 *     boundary are always host indices.
 *   - No call waits on the device without a bound: device-side failures
 *     (neighbor overflow, non-finite state, an exhausted iteration cap) are
 *     reported through the status word read back by the call.
 */
#ifndef FLUIDSOLVER_B200_H
#define FLUIDSOLVER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FS_ABI_VERSION 4

typedef enum fs_status {
    FS_OK = 0,
    FS_ERR_INVALID = 1,   /* bad argument or configuration (CompatibilityReport issue in the reference) */
    FS_ERR_CAPACITY = 2,  /* a neighbor list exceeded its capacity (the reference throws, CompressedNeighbors.cpp:276-321) */
    FS_ERR_NAN = 3,       /* non-finite particle state detected */
    FS_ERR_TIMEOUT = 4,   /* a bounded device-side wait gave up */
    FS_ERR_CUDA = 5,      /* a CUDA runtime call failed */
    FS_ERR_NO_DEVICE = 6, /* no usable sm_100 device */
    FS_ERR_STATE = 7      /* call out of order (e.g. lists requested before a search) */
} fs_status;

/* Solver selected by SolverSerializer's "type" string (SolverSerializer.cpp:137-219). */
typedef enum fs_solver_kind {
    FS_SOLVER_NONE = 0,     /* neighborhood search only */
    FS_SOLVER_SESPH_2D = 1, /* "sesph"    */
    FS_SOLVER_SESPH_3D = 2, /* "sesph-3d" */
    FS_SOLVER_IISPH_2D = 3, /* "iisph"    */
    FS_SOLVER_IISPH_3D = 4  /* "iisph-3d" */
} fs_solver_kind;

/*
 * Neighbor-set contract of the reference search being replaced. One device
 * search (cell-key radix sort + cell-order reordering + cell table) serves all of
 * them; the contract fixes the predicate, which particles own a list, which
 * particles may appear in one, and the capacity limit.
 */
typedef enum fs_search_kind {
    FS_SEARCH_QUADRATIC_2D = 0,  /* QuadraticNeighborhoodSearchDynamicAllocated.cpp:11-38: every particle, every j, length(d) <= r */
    FS_SEARCH_HASHED_2D = 1,     /* HashedNeighborhoodSearch.cpp:9-73: fluid owners only, every j, length(d) <= r */
    FS_SEARCH_COMPACT_2D = 2,    /* CompactHashingNeighborhoodSearch.cpp:14-84,210-247: active owners, active j, length(d) <= r, <= 40 */
    FS_SEARCH_QUADRATIC_3D = 3,  /* QuadraticNeighborhoodSearch3D.cpp:32-69: active owners, active j, dot(d,d) <= r*r */
    FS_SEARCH_HASHED_3D = 4,     /* HashedNeighborhoodSearch3D.cpp:134-185: as quadratic-3d */
    FS_SEARCH_COMPRESSED_3D = 5  /* CompressedNeighbors.cpp:536-595: as quadratic-3d, <= 97 neighbors */
} fs_search_kind;

typedef enum fs_precision {
    FS_PRECISION_FP32 = 0,       /* plain float sums in the reference's operation order */
    FS_PRECISION_FP32_KAHAN = 1, /* float state, Kahan-compensated neighbor sums, FP64 residual (default) */
    FS_PRECISION_FP64 = 2        /* double state and arithmetic (error reference) */
} fs_precision;

/* fs_params.flags */
#define FS_FLAG_REFERENCE_ORDER 0x1u  /* sum neighbors in HashedNeighborhoodSearch3D's list order and
                                         reproduce the serial L1 density read order of the reference
                                         (IISPHFluidSolver3D.hpp:60-64 vs :210); for bit-level parity runs */
#define FS_FLAG_SYNC_EACH_ITERATION 0x2u /* host-driven IISPH loop (one readback per iteration) instead of the
                                            device-side early exit inside a CUDA graph */
#define FS_FLAG_ONE_KERNEL_STEPS 0x4u  /* fs_step / fs_run of a single scene of at most 4,096 particles (not
                                          the 3D fast mode, not compact hashing) run whole steps in one launch
                                          of one block instead of a CUDA graph of per-phase kernels; the same
                                          results bit for bit */

/* Particle types (Particle.hpp:7-12). */
#define FS_TYPE_NORMAL 0
#define FS_TYPE_BOUNDARY 1
#define FS_TYPE_INACTIVE 2

/* Time step generator of the Simulator (time/TimestepGenerator.hpp:13-33). */
typedef enum fs_timestep_kind {
    FS_TIMESTEP_CONSTANT = 0,    /* ConstantTimestepGenerator.cpp:4-41: desired dt = timestep */
    FS_TIMESTEP_DYNAMIC_CFL = 1  /* DynamicCflTimestepGenerator.cpp:6-97: desired dt from the
                                    largest |v| and |a| of the active particles, computed on the
                                    device at the start of every step; the desired_dt argument of
                                    the step calls is then ignored */
} fs_timestep_kind;

typedef struct fs_params {
    int32_t dim;        /* 2 or 3 */
    int32_t solver;     /* fs_solver_kind */
    int32_t search;     /* fs_search_kind */
    int32_t precision;  /* fs_precision */
    uint32_t flags;     /* FS_FLAG_* */
    int32_t device;     /* CUDA device ordinal */

    /* IFluidSolverBase::SimulationParameters (IFluidSolver.hpp:18-23) */
    float rest_density;
    float gravity;
    float particle_size; /* h; the kernel support and search radius are 2*h (LibFluidMath.hpp:11) */

    /* SESPHSettings / SESPHSettings3D (settings/SESPHSettings*.hpp) */
    float stiffness;
    /* viscosity of whichever solver is selected */
    float viscosity;
    int32_t single_layer_boundary;
    float single_layer_gamma_1;
    float single_layer_gamma_2; /* SESPH-3D only */

    /* IISPHSettings / IISPHSettings3D (settings/IISPHSettings*.hpp) */
    float max_density_error;
    int32_t min_iterations;
    int32_t max_iterations;
    float omega;
    float gamma;

    /* ConstantTimestepGenerator settings (ConstantTimestepGenerator.hpp:8-13); with the
     * dynamic generator, timestep is its max_timestep (the CFL clamp's default) */
    float timestep;
    float lambda_v;
    float lambda_a;

    /* capacities */
    int64_t max_particles;      /* device arrays are sized for this many particles */
    int32_t neighbor_capacity;  /* per-particle list slots for the solver (0: chosen from the scene) */

    /* time step generator (fs_timestep_kind) and DynamicCflTimestepGenerator's
     * bounds (DynamicCflTimestepGenerator.hpp:11-18); lambda_v / lambda_a above */
    int32_t timestep_generator;
    float min_timestep;
    float max_timestep;
} fs_params;

/* Fills *p with libFluid's defaults for the given solver and dimension
 * (IISPHSettings3D.hpp:6-20 etc.; rest density 1000, gravity 9.81, size 0.1). */
void fs_params_default(fs_params* p, int32_t dim, int32_t solver, int32_t search);

/* Dense host arrays in host order. Pointers not needed by a call may be NULL
 * (on upload: NULL means "zero" for velocity/acceleration/external, "rest
 * density" for density, 0 for pressure, tag = index). */
typedef struct fs_particles {
    int64_t n;
    float* position;     /* dim per particle  (MovementData{,3D}.position)      */
    float* velocity;     /* dim per particle  (MovementData{,3D}.velocity)      */
    float* acceleration; /* dim per particle  (MovementData{,3D}.acceleration)  */
    float* external;     /* dim per particle  (ExternalForces{,3D})             */
    float* mass;         /* ParticleData.mass     */
    float* density;      /* ParticleData.density  */
    float* pressure;     /* ParticleData.pressure */
    uint8_t* type;       /* ParticleInfo.type     */
    uint32_t* tag;       /* ParticleInfo.tag      */
    /* IISPH per-particle data (IISPHParticleData3D, IISPHFluidSolver3D.hpp:13-19); download only */
    float* predicted_velocity;       /* dim per particle */
    float* non_pressure_acceleration;/* dim per particle (3D only) */
    float* source_term;
    float* diagonal_element;
} fs_particles;

/* IISPHFluidSolver3D's statistics (IISPHFluidSolver3D.hpp:32-33) plus the step's time step. */
typedef struct fs_step_stats {
    float desired_dt;
    float actual_dt;             /* Timepoint::actual_time_step after the CFL clamp */
    int32_t iterations;          /* stat_last_iteration_count */
    float avg_density_error;     /* stat_last_average_predicted_density_error (absolute, density units) */
    double avg_density_error_fp64;
    float max_density_error;
    float max_velocity;
    float max_acceleration;
    int32_t status;              /* fs_status of the device status word */
    int32_t max_neighbors;       /* largest list seen by the last search */
} fs_step_stats;

typedef struct fs_ctx fs_ctx;

int32_t fs_abi_version(void);
const char* fs_last_error(void);

/* Creates a context (device buffers for p->max_particles particles, a stream). */
fs_status fs_create(const fs_params* p, fs_ctx** out);
fs_status fs_destroy(fs_ctx* ctx);
/* Replaces the settings (data-change propagation of IFluidSolverBase::initialize). */
fs_status fs_set_params(fs_ctx* ctx, const fs_params* p);

/* Copies a whole particle collection to the device (host order). */
fs_status fs_upload(fs_ctx* ctx, const fs_particles* in);
/* Copies the device state back in host order into the non-NULL arrays of *out. */
fs_status fs_download(fs_ctx* ctx, fs_particles* out);

/* Neighborhood search on the current positions (find_neighbors). */
fs_status fs_find_neighbors(fs_ctx* ctx);
/* Neighbor lists of the last search in host-index space, each list ascending:
 * offsets has n+1 entries; indices may be NULL to query *total first. */
fs_status fs_get_neighbors_csr(fs_ctx* ctx, int64_t* offsets, int64_t* indices, int64_t* total);
/* The lists that the solver's passes walk (3D IISPH fast mode: the tile lists),
 * exported like fs_get_neighbors_csr: host-index space, each list ascending,
 * indices NULL to query *total first. No reference counterpart (the
 * reference's solvers walk the search's own lists); it lets a caller check
 * that the solver sees the contract's neighbor sets. Needs a search since the
 * last upload. */
fs_status fs_get_solver_lists_csr(fs_ctx* ctx, int64_t* offsets, int64_t* indices, int64_t* total);
/* Neighbors of an arbitrary position (NeighborhoodInterface::get_neighbors(vec),
 * NeighborhoodInterface.cpp:71-80); ascending host indices, per contract:
 * hashed-3d walks the cells of the last search, skips inactive particles and,
 * like HashedNeighborhoodSearch3D.cpp:279-344, the smallest-index member of
 * every cell after the first; compressed-3d walks the cells, skips inactive
 * particles and tests dot <= r*r; hashed-2d walks the cells; the quadratic
 * contracts test every particle. compact-hashing-2d has none (FS_ERR_INVALID,
 * as the reference throws). Writes min(count, cap) indices (which ones is
 * unspecified when count > cap) and the full count to *count. The cell walks
 * need a search after the last upload (FS_ERR_STATE otherwise). */
fs_status fs_query_position(fs_ctx* ctx, const float* position, int64_t* out, int64_t cap, int64_t* count);

/* fs_query_position without any allocation. It has no counterpart in the
 * reference: libFluid's get_neighbors(vec) hands out a lazy iterator.
 * Results and errors are those of fs_query_position. The difference is the
 * working memory: one fixed device array per device (compiled into the
 * library), and the caller's own buffer. Nothing goes through cudaMalloc,
 * cudaFree or a host-side allocator. Limits:
 *   - cap may be at most FS_QUERY_NOALLOC_MAX; a larger cap is rejected with
 *     FS_ERR_INVALID before anything runs;
 *   - the fixed array is shared by every context on a device, so calls that
 *     overlap in time on one device (two host threads) race on it;
 *   - the first call on each device resolves the array's address, so make
 *     that first call before any stream capture begins;
 *   - that address is kept for the rest of the process: after a
 *     cudaDeviceReset of the device (which also ends every context on it)
 *     this entry point must not be called on that device again. */
#define FS_QUERY_NOALLOC_MAX 65536
fs_status fs_query_position_noalloc(fs_ctx* ctx, const float* position, int64_t* out, int64_t cap,
                                    int64_t* count);

/* The solver's timestep on the lists of the preceding fs_find_neighbors
 * (IFluidSolverBase::execute_simulation_step, IFluidSolver.hpp:30); the
 * CFL-clamped time step is returned in stats->actual_dt. desired_dt <= 0 uses
 * p->timestep. With FS_TIMESTEP_DYNAMIC_CFL the device generates the desired
 * time step (stats->desired_dt) and desired_dt is ignored, here and in
 * fs_step / fs_run. */
fs_status fs_solve_step(fs_ctx* ctx, float desired_dt, fs_step_stats* stats);
/* One solver step: neighborhood search + the solver's timestep, like
 * Simulator::execute_simulation_step (Simulator.cpp:7-57) without entities
 * and sensors. desired_dt <= 0 uses p->timestep. */
fs_status fs_step(fs_ctx* ctx, float desired_dt, fs_step_stats* stats);
/* `steps` steps back to back without host synchronisation in between
 * (captured once in a CUDA graph); stats of the last step. */
fs_status fs_run(fs_ctx* ctx, int32_t steps, float desired_dt, fs_step_stats* stats);

/* Device time of the phases of the last fs_step (ms): [0] search, [1] L1,
 * [2] L2, [3] pressure iterations, [4] integration. */
fs_status fs_last_phase_times(fs_ctx* ctx, float* ms5);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the library's. */
void* fs_stream(fs_ctx* ctx);
/* Number of this library's own kernel launches since the context was created
 * (library kernels such as the radix sort's are not counted). */
int64_t fs_launch_count(fs_ctx* ctx);
/* Blocks (one thread-block cluster) of the last small-scene launch
 * (FS_FLAG_ONE_KERNEL_STEPS), 0 when the last steps took the step-by-step
 * path. */
int32_t fs_small_blocks(fs_ctx* ctx);

/* ---- tuning ------------------------------------------------------------------
 * The 3D fast mode's launch shapes (no reference counterpart: the reference's
 * loops have nothing to tune). fs_autotune times whole steps on a copy of
 * the context (same parameters and particles; the context's own state is
 * left as it was) along each axis in turn, keeping the fastest value of one
 * axis before trying the next, keeps the best for the context and reports
 * every time it measured:
 *   - how far ahead the tile passes load their neighbor lists (octets of 8
 *     entries, 1..4; the first loop's and the pressure passes' depths);
 *   - the staged candidates per tile (1024, 1536, 2048, 3072): tiles whose
 *     neighborhood holds more fall back to 32-bit lists read from global
 *     memory; a larger cap leaves fewer fallback tiles but takes more shared
 *     memory per block, so fewer blocks fit on an SM;
 *   - the block size of the step's per-particle kernels (sort keys, reorder,
 *     cell table, integration): 128, 256, 512 threads.
 * The tile passes' own shape (128 owners per tile, two threads per owner)
 * and the cell edge (the search radius, which the tiles' 27-cell ranges
 * assume) are fixed by the tile design. fs_autotune allocates a second set
 * of device buffers while it runs. Contexts whose passes are not tiled report
 * tuned = 0. A batched context takes the result of a representative single
 * scene through fs_set_tuning. */
typedef struct fs_tuning {
    int32_t tuned;                   /* 1 if fs_autotune measured */
    int32_t first_loop_prefetch;     /* the values in use */
    int32_t pressure_prefetch;
    int32_t tile_cap;                /* fs_set_tuning: 0 keeps the current one */
    int32_t block_size;              /* fs_set_tuning: 0 keeps the current one */
    int32_t pressure_threads_per_owner; /* 1, 2 or 4 threads walk an owner's list in the pressure
                                           passes (fs_set_tuning: 0 keeps the current one) */
    float first_loop_ms[4];          /* measured per depth 1..4 (0: not tried) */
    float pressure_iteration_ms[4];  /* per pressure iteration, per depth 1..4 */
    float step_ms_by_tile_cap[4];    /* whole step, caps 1024, 1536, 2048, 3072 */
    float step_ms_by_block_size[3];  /* whole step, block sizes 128, 256, 512 */
    float fallback_tiles_by_tile_cap[4]; /* fraction of tiles on 32-bit lists, per cap */
    float pressure_iteration_ms_by_threads[3]; /* per pressure iteration, 1, 2, 4 threads per owner */
} fs_tuning;
fs_status fs_autotune(fs_ctx* ctx, fs_tuning* out);
fs_status fs_set_tuning(fs_ctx* ctx, const fs_tuning* in);

/* Test hook for the bounded waits: how many times the tile passes try the
 * wait for a tile's staged copies before they give up with FS_ERR_TIMEOUT
 * (the step then returns it and leaves the state as the last finished phase
 * left it). No reference counterpart: it exists so that the error path of a
 * wait that runs out can be exercised on a GPU without faulting it. tries < 0
 * restores the default (65,536); 0 makes every wait give up at once. The
 * limit is one per device, shared by every context on the context's device. */
fs_status fs_set_tile_wait_limit(fs_ctx* ctx, int32_t tries);

/* The searches' own sort on caller keys, for tests of the sort alone: the
 * stable least-significant-digit radix sort that orders the particles by
 * (region, cell) key every search (and, in the reference-order mode, by the
 * 64-bit key with the order inside a cell), run on `device` over n host keys
 * of key_bytes 4 or 8 bytes. Every key must be below 2^bits (1 <= bits <=
 * 8 * key_bytes). sorted (n keys, may be null) receives the keys in
 * ascending order; order (n, may be null) the input position of each, equal
 * keys in input order. No reference counterpart: the reference sorts its
 * collection with a quick sort over Morton keys
 * (ParticleCollectionAlgorithm.hpp:28-133), whose order of equal keys is not
 * defined. */
fs_status fs_sort_keys(int32_t device, const void* keys, int32_t key_bytes, int64_t n, int32_t bits, void* sorted,
                       uint32_t* order);

/* ---- entities and sensors on the device -----------------------------------
 * Host-side entities and sensors of the Simulator read the whole collection;
 * these run their arithmetic where the state lives, so that a step loop that
 * keeps the state on the device (fs_run, or a caller that does not download
 * every step) still gets them. */

/* BoundaryPreprocessor::execute_simulation_step (BoundaryPreprocessor.cpp:7-48,
 * the entity that runs before the solver): every boundary particle's mass
 * becomes min(rho0 particle_size^3, rho0 gamma_1 / sum_b W(x_i - x_b)), the sum
 * over its boundary neighbors in the neighbor-set contract (itself included),
 * gamma_1 from a perfectly sampled plane (:104-119). rho0 and particle_size are
 * the context's. Needs a search on the current positions (fs_find_neighbors);
 * in the FP32 reference-order mode the sums run in the reference's list order. */
fs_status fs_boundary_preprocess(fs_ctx* ctx);

/* Global sensors of ParticleStatistics.cpp:17-201 over the device state.
 * Maxima start at FLT_MIN and minima at FLT_MAX, as the reference's
 * MaxMinAvgSensorData does. Averages and energies are summed in FP64 (the
 * reference sums serially in float, whose own rounding they differ by).
 * velocity: |v| of the normal particles (the reference's velocity and energy
 * sensors read 2D MovementData; in 3D the same formulas use the 3D velocity). */
typedef struct fs_global_stats {
    float density_max, density_min, density_avg;     /* GlobalDensitySensor (:17-43) */
    float pressure_max, pressure_min, pressure_avg;  /* GlobalPressureSensor (:59-85) */
    float velocity_max, velocity_min, velocity_avg;  /* GlobalVelocitySensor (:101-128) */
    float kinetic_energy, potential_energy;          /* GlobalEnergySensor (:143-167): relative to zero_height */
    int32_t reserved;
    int64_t normal_particles, boundary_particles, inactive_particles; /* GlobalParticleCountSensor (:181-201) */
} fs_global_stats;
fs_status fs_global_statistics(fs_ctx* ctx, float zero_height, fs_global_stats* out);

/* ---- the fluid path tracer ---------------------------------------------------
 * libFluid's FluidRaytracer3D (visualizer/raytracer/) on the device state of a
 * 3D single-scene context, rendering into host memory (no window or graphics
 * API). Both calls first search the current positions; the density at a point
 * sums the particles within the search radius (ParticleIntersectionAccelerator.cpp:76-126).
 *
 * fs_trace_rays: ParticleIntersectionAccelerator::is_intersecting_with_particles
 * (:20-74) for n rays, without a random offset along them. hit: -1 none, 0 the
 * fluid surface reached from outside, 1 from inside, 2 a boundary surface;
 * point, normal (3 floats each) and length (the march distance to the hit). */
fs_status fs_trace_rays(fs_ctx* ctx, float surface_density_fraction, int64_t n, const float* origins,
                        const float* directions, int32_t* hit, float* point, float* normal, float* length);

/* Camera::CameraSettings (Camera.hpp:13-21); field_of_view_x in radians. */
typedef struct fs_camera {
    float position[3];
    float view_direction[3];
    float view_up[3];
    float field_of_view_x;
    int32_t width, height;
    int32_t flip_y;
} fs_camera;
typedef struct fs_render_settings {
    int32_t samples_per_pixel;            /* Camera::SampleSettings::amount_of_samples */
    int32_t maximum_recursion_depth;      /* FluidRaytracer3D::Settings */
    int32_t output_normals_of_first_hit;
    float surface_density_fraction;       /* of the rest density: the surface's iso density */
    float exposure, gamma;                /* ToneMapper::ToneMapperSettings (ToneMapper.hpp:9-20) */
    uint64_t seed;                        /* of the per-pixel random streams */
    int32_t tone_mapper;                  /* 0 exponential (the default), 1 filmic (the ACES curve) */
    int32_t gamma_correction;             /* 1: the gamma correction is applied (the default) */
} fs_render_settings;
void fs_render_settings_default(fs_render_settings* r);
/* ToneMapper::map_render_target_to_image (ToneMapper.cpp:71-102) on host
 * radiance, without a context: exposure, the settings' tone mapping curve,
 * the gamma correction when enabled, bytes; rgba receives 4 bytes per pixel
 * (alpha 255). fs_render applies the same mapping. Host code only. */
fs_status fs_tone_map(const float* radiance, int64_t pixels, const fs_render_settings* settings, uint8_t* rgba);
/* FluidRaytracer3D::render: radiance (width * height * 3 floats, row-major from
 * the top-left pixel), the path tracer's estimate with a white sky
 * (FluidRaytracer3D.cpp:70-165; Skybox without an image); rgba (width * height
 * * 4 bytes, may be NULL): the tone-mapped image (ToneMapper.cpp:79-102). The
 * random numbers come from per-pixel streams, so images match the reference's
 * in distribution, not value by value. */
fs_status fs_render(fs_ctx* ctx, const fs_camera* cam, const fs_render_settings* settings, float* radiance,
                    uint8_t* rgba);

/* ---- particle files ---------------------------------------------------------
 * ParticleSerializer's version-1 files (ParticleSerializer.cpp:41-141): the
 * scenario particle files (scenarios/** / *.data) and FluidConsole's particle
 * dumps. The layout (little-endian): u32 version 1, u32 component count, u32
 * component ids, u64 particle count, then per particle the components present
 * in id order (1/2 MovementData 2D/3D: position, velocity, acceleration;
 * 3 ParticleInfo: u8 type, u32 tag; 4 ParticleData: density, mass, pressure;
 * 5/6 ExternalForces 2D/3D), all inside one LZ4 frame (the lz4 library's
 * LZ4F format, Lz4CompressedStream.cpp:24-180), coded by this library itself.
 * components: bit (1 << id) per component the file holds. */
#define FS_COMPONENT_MOVEMENT_2D (1u << 1)
#define FS_COMPONENT_MOVEMENT_3D (1u << 2)
#define FS_COMPONENT_INFO (1u << 3)
#define FS_COMPONENT_DATA (1u << 4)
#define FS_COMPONENT_EXTERNAL_2D (1u << 5)
#define FS_COMPONENT_EXTERNAL_3D (1u << 6)
fs_status fs_particles_file_info(const char* path, int32_t* dim, int64_t* n, uint32_t* components);
/* Reads a file into the non-NULL arrays of *out (out->n must be the file's
 * count); arrays of components the file lacks are zeroed (tag: the index). */
fs_status fs_particles_file_read(const char* path, fs_particles* out);
/* Writes n particles (in->n) of dimension dim with the components whose
 * arrays are non-NULL: movement if position is (velocity and acceleration
 * NULL: zero), info if type or tag is, data if mass, density or pressure is,
 * external forces if external is. */
fs_status fs_particles_file_write(const char* path, int32_t dim, const fs_particles* in);
/* The context's state in host order, every component, written as a particle
 * file: FluidConsole's particle dump (fluidConsole/main.cpp:24-32, 150-184). */
fs_status fs_dump(fs_ctx* ctx, const char* path);

/* ---- batched scenes -------------------------------------------------------
 * Many independent scenes of uneven size advance together. This has no
 * counterpart in the reference, which runs one solver object per scene (one
 * IISPHFluidSolver3D per scenario). One launch per sub-phase covers every
 * scene. Each scene keeps its own cell grid (particles of different scenes
 * never interact), its own IISPH convergence test and its own CFL-clamped
 * time step. Scene s owns host particles [offsets[s], offsets[s+1]) of the
 * collection passed to fs_upload, which must hold exactly offsets[scenes]
 * particles. Batched contexts run the 3D IISPH solver with the hashed-3d
 * contract in FP32 + Kahan device order (FS_ERR_INVALID otherwise), up to
 * 65,535 scenes; fs_query_position is not available on them (a position names
 * no scene). fs_download, fs_get_neighbors_csr, fs_step and fs_run work as for
 * one scene (fs_step/fs_run report scene 0's statistics). */
fs_status fs_batch_create(const fs_params* p, int32_t scenes, const int64_t* offsets, fs_ctx** out);
/* `steps` steps of every scene (CUDA graphs, no host sync in between); stats
 * has one entry per scene and receives each scene's last-step statistics. */
fs_status fs_batch_run(fs_ctx* ctx, int32_t steps, float desired_dt, fs_step_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* FLUIDSOLVER_B200_H */
