/*
 * slosh_cuda.h -- C ABI of the B200-native Slosh FLIP/APIC substep.
 *
 * The types mirror the plain-data simulation types of the Slosh Unreal plugin
 * (PLUG = SloshDemo/Plugins/Slosh):
 *   slosh_settings_t        <- FSloshSolverSettings   PLUG/Source/SloshCore/Public/SloshTypes.h:113-160
 *   slosh_particle_t        <- FSloshParticleGPU      SloshTypes.h:84-91 (48 bytes, C as 9 halves)
 *   slosh_collider_t        <- FSloshColliderGPU      SloshTypes.h:32-44 (80 bytes)
 *   slosh_manipulator_t     <- FSloshManipulatorGPU   SloshTypes.h:66-80 (80 bytes)
 *   slosh_emit_request_t    <- FSloshEmitRequest      SloshTypes.h:169-181
 *   slosh_frame_input_t     <- FSloshFrameInput       SloshTypes.h:184-194
 *   slosh_results_t         <- FSloshResults          SloshTypes.h:208-231
 *
 * The functions replace the public surface of FSloshProxy
 * (PLUG/Source/SloshCore/Public/SloshProxy.h:23-147); each declaration names the
 * member it stands in for. All calls are synchronous with respect to the host
 * unless stated; device work is issued on the context's CUDA stream.
 *
 * Ownership: the library owns all device memory. Host arrays passed in are
 * copied during the call. Device pointers handed out stay valid until the next
 * step call or slosh_destroy.
 *
 * Threading: one context per host thread at a time; no internal threads.
 */
#ifndef SLOSH_CUDA_H
#define SLOSH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define SLOSH_API __declspec(dllexport)
#else
#define SLOSH_API __attribute__((visibility("default")))
#endif

#define SLOSH_ABI_VERSION 3u

/* Limits, SloshTypes.h:93-110. The particle cap is raised above the reference's 16,777,216. */
#define SLOSH_MAX_COLLIDERS 64u
#define SLOSH_MAX_MANIPULATORS 32u
#define SLOSH_COUPLING_STRIDE 16u
#define SLOSH_NUM_STATS 16u
#define SLOSH_MAX_MG_LEVELS 8u

/* Status codes. The reference has none (values are clamped silently,
 * SloshProxy.cpp:345-347); every entry point here returns one. */
typedef enum slosh_status {
    SLOSH_OK = 0,
    SLOSH_ERR_INVALID_ARG = 1,
    SLOSH_ERR_OUT_OF_MEMORY = 2,
    SLOSH_WARN_POOL_OVERFLOW = 3, /* warning: bricks found the pool full (ballistic fallback ran) */
    SLOSH_ERR_NOT_CONVERGED = 4,  /* warning: a solve hit max_iterations above its tolerance */
    SLOSH_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait gave up */
    SLOSH_ERR_CUDA = 6,
    SLOSH_ERR_NO_DEVICE = 7,
    SLOSH_ERR_CAPACITY = 8        /* particle capacity exceeded */
} slosh_status;

/* ESloshTransferMode, SloshTypes.h:10-14 */
enum { SLOSH_TRANSFER_FLIP = 0, SLOSH_TRANSFER_APIC = 1 };
/* ESloshPressureSolver, SloshTypes.h:16-22 */
enum { SLOSH_SOLVER_RBGS = 0, SLOSH_SOLVER_MGPCG = 1 };
/* ESloshColliderShape, SloshTypes.h:24-29 */
enum { SLOSH_COLLIDER_SPHERE = 0, SLOSH_COLLIDER_BOX = 1, SLOSH_COLLIDER_CAPSULE = 2 };
/* ESloshEmitShape, SloshTypes.h:162-167 */
enum { SLOSH_EMIT_FILL_CELLS = 0, SLOSH_EMIT_SPHERE = 1, SLOSH_EMIT_BOX = 2 };
/* Storage precision of the multigrid preconditioner (extension, no reference counterpart). */
enum { SLOSH_PRECISION_FP32 = 0, SLOSH_PRECISION_FP16_STORAGE = 1, SLOSH_PRECISION_BF16_STORAGE = 2 };
/* Pressure warm start (extension). PREVIOUS is the reference behaviour (MarkCellsCS rescale). */
enum { SLOSH_WARM_START_ZERO = 0, SLOSH_WARM_START_PREVIOUS = 1, SLOSH_WARM_START_LEARNED = 2 };

/* FSloshSolverSettings, field for field (SloshTypes.h:113-160), then extensions. */
typedef struct slosh_settings_t {
    int32_t grid_dim[3];                 /* GridDim                     */
    float cell_size;                     /* CellSize (m)                */
    uint32_t particle_capacity;          /* ParticleCapacity            */
    uint32_t transfer_mode;              /* TransferMode                */
    float flip_ratio;                    /* FlipRatio                   */
    float density;                       /* Density (kg/m^3)            */
    float kinematic_viscosity;           /* KinematicViscosity          */
    float boundary_friction;             /* BoundaryFriction            */
    float adhesion;                      /* Adhesion                    */
    float adhesion_distance;             /* AdhesionDistance            */
    float density_correction;            /* DensityCorrection           */
    float density_deadband;              /* DensityDeadband             */
    uint32_t two_sided_density_projection; /* bTwoSidedDensityProjection */
    float density_relaxation;            /* DensityRelaxation           */
    int32_t density_projection_iterations; /* DensityProjectionIterations */
    int32_t density_projection_interval; /* DensityProjectionInterval   */
    uint32_t sparse_bricks;              /* bSparseBricks               */
    float sparse_max_active_fraction;    /* SparseMaxActiveFraction     */
    float sparse_storage_budget;         /* SparseStorageBudget         */
    float particle_radius_cells;         /* ParticleRadiusCells         */
    float gravity[3];                    /* Gravity                     */
    uint32_t pressure_solver;            /* PressureSolver              */
    int32_t pressure_iterations;         /* PressureIterations (RBGS)   */
    float sor_weight;                    /* SORWeight                   */
    int32_t pcg_iterations;              /* PCGIterations               */
    int32_t mg_coarse_iterations;        /* MGCoarseIterations          */
    int32_t sort_interval;               /* SortInterval                */
    uint32_t smooth_coupling_force;      /* bSmoothCouplingForce        */
    uint32_t ghost_fluid;                /* bGhostFluid                 */
    int32_t viscosity_iterations;        /* ViscosityIterations         */
    int32_t extrapolation_layers;        /* ExtrapolationLayers         */
    int32_t min_substeps;                /* MinSubsteps                 */
    int32_t max_substeps;                /* MaxSubsteps                 */
    float max_frame_dt;                  /* MaxFrameDt                  */
    float cfl;                           /* CFL                         */
    float max_speed;                     /* MaxSpeed                    */
    /* ---- extensions (no reference counterpart) ---- */
    float tolerance;        /* > 0: MGPCG iterates until ||r||/||b|| <= tolerance (or max_iterations);
                               <= 0: the reference's fixed pcg_iterations */
    int32_t max_iterations; /* iteration cap when tolerance > 0 */
    uint32_t precision_mode;/* SLOSH_PRECISION_* of the V-cycle storage */
    uint32_t warm_start;    /* SLOSH_WARM_START_* */
    /* Multigrid preconditioner (extensions; the defaults are the reference's V-cycle). */
    float mg_correction_scale;   /* every restriction multiplies the reference's 1/4 by this factor, which
                                    scales each level's coarse-grid correction; 1 = the reference. Values
                                    of 1.5-1.9 make up for the piecewise-constant prolongation and roughly
                                    halve the PCG iterations on 256^3 grids. Clamped to [0.5, 1.95]. */
    int32_t mg_smoothing_sweeps; /* red-black sweep pairs in each pre- and post-smoothing of every level
                                    above the coarsest; 1 = the reference. Clamped to [1, 4]. */
    uint32_t pcg_flexible;       /* 1: flexible PCG, beta = r_k.(z_k - z_{k-1}) / rho_{k-1} (Polak-Ribiere),
                                    robust to a preconditioner that is not exactly linear (FP16/BF16
                                    storage); 0: beta = rho_k / rho_{k-1} (the reference) */
    float mg_smoother_weight;    /* over-relaxation of the finest level's red-black sweeps: each sweep sets
                                    x + w (x_GS - x) instead of the Gauss-Seidel value x_GS, and the red
                                    initialisation of the preconditioned residual is w r / diag; coarser
                                    levels are unchanged. 1 = the reference; 1.15 saves about one PCG
                                    iteration in ten on 256^3 grids. Clamped to [0.5, 1.9]. */
} slosh_settings_t;

/* FSloshParticleGPU (SloshTypes.h:84-91): Pos, Age (negative or NaN = dead), Vel,
 * C = APIC affine rows Cx, Cy, Cz as 9 halves in 5 words (SloshCommon.ush:63-105). */
typedef struct slosh_particle_t {
    float pos[3];
    float age;
    float vel[3];
    uint32_t c[5];
} slosh_particle_t;

/* FSloshColliderGPU (SloshTypes.h:32-44). */
typedef struct slosh_collider_t {
    float center[3];
    uint32_t type;
    float rotation[4]; /* quaternion x, y, z, w; local -> sim */
    float extent[3];
    uint32_t flags;
    float linear_velocity[3];
    float pad0;
    float angular_velocity[3];
    float pad1;
} slosh_collider_t;

/* ESloshManipulatorKind / ESloshManipulatorShape (SloshTypes.h:47-63). Shapes 0-2 are the collider
 * shapes (sphere, box, capsule); EVERYWHERE applies in the whole domain. */
enum { SLOSH_MANIP_DRAIN = 0, SLOSH_MANIP_DIRECTIONAL = 1, SLOSH_MANIP_RADIAL = 2, SLOSH_MANIP_SWIRL = 3, SLOSH_MANIP_DRAG = 4 };
enum { SLOSH_SHAPE_SPHERE = 0, SLOSH_SHAPE_BOX = 1, SLOSH_SHAPE_CAPSULE = 2, SLOSH_SHAPE_EVERYWHERE = 3 };

/* FSloshManipulatorGPU (SloshTypes.h:66-80). */
typedef struct slosh_manipulator_t {
    float center[3];
    uint32_t kind;
    float rotation[4];
    float extent[3];
    uint32_t shape;
    float axis[3];
    float strength;
    float falloff;
    float param0;
    float param1;
    uint32_t pad;
} slosh_manipulator_t;

/* FSloshEmitRequest (SloshTypes.h:169-181) plus fill_jitter. */
typedef struct slosh_emit_request_t {
    uint32_t shape;           /* SLOSH_EMIT_* */
    float center[3];
    float extent[3];
    float velocity[3];
    float rotation[4];
    float velocity_spread;
    float speed_jitter;
    int32_t cell_min[3];      /* FillCells only */
    int32_t cell_dims[3];
    uint32_t count;           /* Sphere / Box */
    float fill_jitter;        /* extension: FillCells jitter amplitude in half-cells; the reference
                                 hard-codes 0.8 (Slosh.usf:310); 1.0 gives +-0.25 cell */
} slosh_emit_request_t;

/* FSloshFrameInput (SloshTypes.h:184-194) with POD arrays; SimToWorld is a rendering
 * concern and is not carried. */
typedef struct slosh_frame_input_t {
    slosh_settings_t settings;
    const slosh_collider_t* colliders;
    uint32_t num_colliders;
    const slosh_emit_request_t* emits;
    uint32_t num_emits;
    const slosh_manipulator_t* manipulators;
    uint32_t num_manipulators;
    float delta_time;
    uint32_t reset;
    uint32_t paused;
} slosh_frame_input_t;

/* FSloshColliderFeedback (SloshTypes.h:197-206). */
typedef struct slosh_collider_feedback_t {
    float pressure_force[3];
    float pressure_torque[3];
    float mean_fluid_velocity[3];
    float submerged_centroid_offset[3];
    int32_t wetted_faces;
    int32_t submerged_cells;
    int32_t solid_cells;
} slosh_collider_feedback_t;

/* FSloshResults (SloshTypes.h:208-231) decoded synchronously (the reference reads back
 * 2-4 frames late, SloshProxy.cpp:739-805), plus solver statistics. */
typedef struct slosh_results_t {
    float max_particle_speed;
    int32_t fluid_cells;
    float max_divergence;
    float mean_divergence;
    float mean_interior_density;
    int32_t interior_cells;
    float active_brick_fraction;
    float pool_usage;
    int32_t pool_overflow_bricks;
    int32_t clamped_particles;
    int32_t clamped_in_solid;
    float clamped_centroid[3];
    float grid_memory_mb;
    float particle_memory_mb;
    int32_t allocated_particle_capacity;
    int32_t live_particles;
    int64_t drained_particles;
    int32_t substeps;
    uint64_t sim_frame;
    uint32_t num_colliders;
    slosh_collider_feedback_t colliders[SLOSH_MAX_COLLIDERS];
    /* extensions */
    int32_t last_solve_iterations;     /* PCG iterations of the last pressure solve */
    float last_solve_rel_residual;     /* recursive ||r||/||b|| at its end */
    float last_solve_true_rel_residual;/* ||b - A p||/||b|| recomputed at its end */
    uint32_t raw_stats[SLOSH_NUM_STATS];
} slosh_results_t;

/* Grid and pool layout (SloshProxy.cpp:185-306), for parity tools. */
typedef struct slosh_layout_t {
    int32_t grid_dim[3];
    int32_t brick_dim[3];
    uint32_t num_bricks;
    uint32_t num_pool_bricks;   /* pool slots including the null slot 0 */
    uint32_t pool_cells;        /* num_pool_bricks * 512 */
    uint32_t total_faces;       /* 3 * pool_cells */
    int32_t sort_brick_dim[3];
    uint32_t num_sort_keys;
    uint32_t num_mg_levels;
    int32_t mg_dim[SLOSH_MAX_MG_LEVELS][3];
    uint32_t num_particles;     /* particle slots in use (dispatch bound) */
    uint32_t particle_capacity;
    uint32_t current_vel;       /* which face-velocity buffer holds the post-step field */
} slosh_layout_t;

/* Buffer identifiers for slosh_read_buffer / slosh_write_buffer (state export/import
 * for parity tests and checkpoints). Element types: u32 unless noted. */
typedef enum slosh_buffer_id {
    SLOSH_BUF_PARTICLES = 0,    /* slosh_particle_t[num_particles] */
    SLOSH_BUF_VEL = 1,          /* f32[total_faces], the current face-velocity field */
    SLOSH_BUF_VEL_OLD = 2,      /* f32[total_faces] */
    SLOSH_BUF_FACE_FLAGS = 3,   /* u32[total_faces] */
    SLOSH_BUF_FACE_WEIGHT = 4,  /* f32[total_faces] */
    SLOSH_BUF_CELL_TYPE = 5,    /* u32[pool_cells] */
    SLOSH_BUF_CELL_COUNT = 6,   /* i32[pool_cells] */
    SLOSH_BUF_PRESSURE = 7,     /* f32[pool_cells] */
    SLOSH_BUF_DIVERGENCE = 8,   /* f32[pool_cells] */
    SLOSH_BUF_CELL_DIAG = 9,    /* f32[pool_cells] */
    SLOSH_BUF_DENSITY_Q = 10,   /* f32[pool_cells] */
    SLOSH_BUF_DENSITY_RHS = 11, /* f32[pool_cells] */
    SLOSH_BUF_BRICK_TABLE = 12, /* u32[num_bricks] */
    SLOSH_BUF_SLOT_BRICK = 13,  /* u32[num_pool_bricks] */
    SLOSH_BUF_FREE_SLOTS = 14,  /* u32[num_pool_bricks] */
    SLOSH_BUF_ACTIVE_BRICKS = 15, /* u32[num_bricks + 1] */
    SLOSH_BUF_NEW_SLOTS = 16,   /* u32[num_pool_bricks + 1] */
    SLOSH_BUF_BRICK_TOUCH = 17, /* u32[num_bricks] */
    SLOSH_BUF_STATS = 18,       /* u32[16] */
    SLOSH_BUF_SORT_COUNTS = 19, /* u32[num_sort_keys] */
    SLOSH_BUF_SORT_OFFSETS = 20,/* u32[num_sort_keys], global exclusive offsets */
    SLOSH_BUF_SORT_PERM = 21,   /* u32[num_particles]: source slot of each sorted particle (last sort) */
    SLOSH_BUF_PARTICLE_COUNT = 22, /* u32[4] */
    SLOSH_BUF_ACCUM = 23,       /* i32[2 * total_faces] */
    SLOSH_BUF_VEL_EXTRAP = 24,  /* f32[total_faces]: displacement / scratch velocity buffer of the last G2P */
    SLOSH_BUF_COUPLING = 25,    /* i32[SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE]: this frame's collider accumulators */
    /* outputs of the last slosh_build_surface */
    SLOSH_BUF_SURFACE_FIELD = 26,     /* u16 (f16 bits)[field voxels], x fastest */
    SLOSH_BUF_SURFACE_BRICKS = 27,    /* u32[field bricks]: occupancy of 8^3-voxel bricks */
    SLOSH_BUF_SURFACE_POSITIONS = 28, /* f32[3 * num_vertices], sim metres */
    SLOSH_BUF_SURFACE_NORMALS = 29,   /* f32[3 * num_vertices] */
    SLOSH_BUF_SURFACE_TANGENTS = 30,  /* f32[3 * num_vertices] */
    SLOSH_BUF_SURFACE_INDICES = 31,   /* u32[num_indices], triangles */
    SLOSH_BUF_COUNT_
} slosh_buffer_id;

/* ---- library ---- */
SLOSH_API uint32_t slosh_abi_version(void);
/* Reference defaults of FSloshSolverSettings (SloshTypes.h:113-160) and extension defaults. */
SLOSH_API void slosh_settings_default(slosh_settings_t* out);
/* Thread-local text of the last error of any call on this thread. */
SLOSH_API const char* slosh_last_error_string(void);

/* ---- lifecycle: replaces FSloshProxy construction / ReleaseOnRenderThread (SloshProxy.h:26-33)
 * and Allocate (SloshProxy.cpp:185-306). device < 0 uses the current device. */
SLOSH_API slosh_status slosh_create(const slosh_settings_t* settings, int32_t device, void** out_ctx);
SLOSH_API void slosh_destroy(void* ctx);
/* Issue device work on an external stream (cudaStream_t); NULL restores the context's own stream. */
SLOSH_API slosh_status slosh_set_stream(void* ctx, void* cuda_stream);
SLOSH_API slosh_status slosh_synchronize(void* ctx);

/* ---- frame: replaces SubmitFrame_GameThread + Step_RenderThread (SloshProxy.cpp:146-161, 339-737).
 * Emission, the periodic spatial sort, CFL substep count and all substeps of one frame. */
SLOSH_API slosh_status slosh_step_frame(void* ctx, const slosh_frame_input_t* input);
/* Batched tanks (no reference counterpart; the plugin steps one proxy per volume): one frame of each of
 * `count` independent contexts. All frames are enqueued on the contexts' own streams before any is
 * waited for, so small tanks overlap on the device. statuses (optional, count entries) receives each
 * context's frame status; the return value is the first non-OK one. */
/* Autotuner of the brick passes' launch shape (extension): steps `frames` frames of `input` for each
 * candidate number of CTAs per SM (2, 4, 8, 12, 16; capped at one CTA per pool brick), times them on the
 * device and leaves the context on the fastest per substep. The simulation advances by those frames;
 * results never depend on the shape (every brick pass is a grid-stride loop). Default: 8 per SM. */
typedef struct slosh_autotune_result_t {
    uint32_t num_candidates;
    uint32_t ctas_per_sm[8];
    float ms_per_substep[8];
    uint32_t best_ctas_per_sm;
    uint32_t brick_ctas;        /* the chosen grid of the brick passes */
} slosh_autotune_result_t;
SLOSH_API slosh_status slosh_autotune(void* ctx, const slosh_frame_input_t* input, uint32_t frames, slosh_autotune_result_t* out);
SLOSH_API slosh_status slosh_set_ctas_per_sm(void* ctx, uint32_t ctas_per_sm);
/* CTAs per SM of the level-0 MGPCG passes (one warp per brick; default 3); results do not depend on it. */
SLOSH_API slosh_status slosh_set_mg_ctas_per_sm(void* ctx, uint32_t ctas_per_sm);
SLOSH_API slosh_status slosh_step_frames(void* const* ctxs, const slosh_frame_input_t* inputs, uint32_t count,
                                         slosh_status* statuses);
/* Split form of slosh_step_frame for per-substep harnesses: begin_frame does the frame prologue
 * (settings, emission, sort) and returns the substep count and dt; substep(i) runs one substep. */
SLOSH_API slosh_status slosh_begin_frame(void* ctx, const slosh_frame_input_t* input,
                                         int32_t* out_substeps, float* out_dt);
SLOSH_API slosh_status slosh_substep(void* ctx, int32_t step_index);
SLOSH_API slosh_status slosh_end_frame(void* ctx);

/* ---- individual phases (harness control; SloshProxy.cpp:1022-1087, 582-592) ---- */
/* Spatial sort + compaction of the particle buffer (AddSpatialSort). */
SLOSH_API slosh_status slosh_sort_particles(void* ctx);
/* Allocation-free spatial sort of caller-owned device particles. No counterpart in the reference
 * (whose sort, AddSpatialSort, only runs on the proxy's own buffers): it is for hosts that must not
 * allocate device memory while they run. Same keys, order and outputs as slosh_sort_particles, on
 * the current device, enqueued on cuda_stream (NULL = default stream) without waiting for it.
 * Scratch is one static device array per device, sized for SLOSH_STATIC_SORT_MAX_PARTICLES particles
 * and SLOSH_STATIC_SORT_MAX_KEYS sort keys (grids up to 256^3); larger inputs return
 * SLOSH_ERR_CAPACITY. The array's address differs per CUDA context; each call looks up the current
 * context's and resolves it on the first call in that context. That first call also loads the library's
 * device code into the context if CUDA has not loaded it yet (lazy module loading is the default), which
 * commits about 7.4 MB of device memory for the scratch, and it is the only call that allocates: make it
 * at start-up, before any stream capture begins in that context (CUDA_MODULE_LOADING=EAGER moves the
 * load to context creation). Once loaded, the scratch stays resident on that device until the process
 * exits. Overlapping calls on one device race on the shared scratch: order them. particles_out must not
 * alias particles_in; perm_out (count words), key_offsets_out (sort-key count words) and live_count_out
 * (1 word) are optional device outputs. */
#define SLOSH_STATIC_SORT_MAX_PARTICLES 262144u
#define SLOSH_STATIC_SORT_MAX_KEYS (262144u + 1u)
SLOSH_API slosh_status slosh_sort_particles_static(const slosh_particle_t* particles_in, slosh_particle_t* particles_out,
                                                   uint32_t count, const int32_t grid_dim[3], float cell_size,
                                                   uint32_t* perm_out, uint32_t* key_offsets_out, uint32_t* live_count_out,
                                                   void* cuda_stream);
/* One emission request (EmitReserveCS + EmitParticlesCS, Slosh.usf:272-358). */
SLOSH_API slosh_status slosh_emit(void* ctx, const slosh_emit_request_t* request);
/* Sets the proxy's emission seed counter (FSloshProxy::EmitSeed, SloshProxy.h:80; starts at 1
 * and increments once per emission, SloshProxy.cpp:529). */
SLOSH_API slosh_status slosh_set_emit_seed(void* ctx, uint32_t seed);

/* ---- particle data: replaces GetParticleBuffer_RenderThread / GetNumParticles_RenderThread
 * (SloshProxy.h:41-42). The reference has no upload; it is added for seeded scenes. */
SLOSH_API slosh_status slosh_upload_particles(void* ctx, const slosh_particle_t* particles, uint32_t count);
SLOSH_API slosh_status slosh_download_particles(void* ctx, slosh_particle_t* out, uint32_t capacity, uint32_t* out_count);
SLOSH_API slosh_status slosh_particle_device_ptr(void* ctx, void** out_ptr, uint32_t* out_count);

/* ---- results: replaces GetResults (SloshProxy.cpp:177-183) + PollReadbacks decode (:739-805) ---- */
SLOSH_API slosh_status slosh_get_results(void* ctx, slosh_results_t* out);
SLOSH_API slosh_status slosh_get_layout(void* ctx, slosh_layout_t* out);

/* ---- state export / import (checkpoint and parity; the reference has none) ---- */
SLOSH_API slosh_status slosh_buffer_bytes(void* ctx, int32_t buffer_id, size_t* out_bytes);
SLOSH_API slosh_status slosh_read_buffer(void* ctx, int32_t buffer_id, void* host_dst, size_t bytes);
SLOSH_API slosh_status slosh_write_buffer(void* ctx, int32_t buffer_id, const void* host_src, size_t bytes);

/* ---- timing (CUDA events on the context's stream): per-phase device milliseconds of the
 * last frame, summed over substeps. Phases: 0 sort, 1 pool, 2 p2g, 3 grid (mark, normalize,
 * divergence), 4 pressure, 5 project+residual, 6 density projection, 7 extrapolate, 8 g2p. */
#define SLOSH_NUM_PHASES 9
SLOSH_API slosh_status slosh_enable_phase_timing(void* ctx, int32_t enable);
SLOSH_API slosh_status slosh_get_phase_ms(void* ctx, float* out_ms, int32_t n);
/* Number of kernel launches this library issued since creation. */
SLOSH_API uint64_t slosh_launch_count(void* ctx);
/* Bytes this context copied host->device and device->host since creation (frame inputs,
 * results, solver residual checks, particle uploads and downloads, buffer reads and writes). */
SLOSH_API slosh_status slosh_transfer_bytes(void* ctx, uint64_t* out_h2d, uint64_t* out_d2h);

/* ---- headless liquid surface: the renderer's density field and surface nets (SloshSurface.usf:54-470,
 * SloshRenderer.cpp:118-170), written into device buffers of the context instead of UE textures and
 * vertex buffers. Particles are splatted as spheres (the renderer's Anisotropy = 0). */
typedef struct slosh_surface_params_t {
    float field_resolution;      /* FSloshRenderSettings::FieldResolution: field voxels per solver cell (0.5-3) */
    float surface_smoothing;     /* SurfaceSmoothing: kernel radius in splat radii (0.5-6) */
    float particle_radius_scale; /* ParticleRadiusScale: splat radius in cells */
    float iso_level;             /* IsoLevel (0.02-0.98): 0.5 = surface at the particle radius */
    uint32_t build_mesh;         /* 0: field and brick occupancy only; 1: also the surface-nets mesh */
    uint32_t max_vertices;       /* capacity of the vertex buffers */
    uint32_t max_indices;        /* capacity of the index buffer */
} slosh_surface_params_t;
typedef struct slosh_surface_info_t {
    int32_t field_dim[3];
    int32_t brick_dim[3];
    float voxel_size;            /* sim metres */
    uint32_t vertices_requested; /* surface cells found (can exceed max_vertices) */
    uint32_t num_vertices;       /* vertices written: min(requested, max_vertices) */
    uint32_t indices_requested;
    uint32_t num_indices;        /* min(requested, max_indices) in whole quads (6 indices): only those are written */
} slosh_surface_info_t;
SLOSH_API void slosh_surface_params_default(slosh_surface_params_t* out);
/* Builds the field (and mesh) from the current particles on the context's stream and waits for it.
 * Vertices and triangles are numbered in cell order (deterministic). */
SLOSH_API slosh_status slosh_build_surface(void* ctx, const slosh_surface_params_t* params, slosh_surface_info_t* out);
/* Device pointers of the last build (valid until the next build or slosh_destroy); any may be NULL. */
SLOSH_API slosh_status slosh_surface_device_ptrs(void* ctx, void** field_f16, void** positions, void** normals, void** tangents,
                                                 void** indices);

/* ---- learned warm start (extension; no counterpart in the reference) ----------------------------
 * A 3-D convolutional U-Net (4 levels, 16/32/64/64 channels, 3x3x3 kernels, BF16 weights and
 * activations, FP32 accumulation) maps (divergence / scale, fluid mask, solid mask) on the dense grid
 * to pressure / scale, scale = max |divergence| over the fluid cells. With settings.warm_start =
 * SLOSH_WARM_START_LEARNED and a network attached, the pressure solve of every substep starts from the
 * network's guess on the fluid cells (zero elsewhere) and still runs to the same stopping test; without
 * a network LEARNED starts from zero. Training pairs come from the plain solver (capture after a
 * substep). Parameters: per convolution W[27][cout][cin] (tap = (dz+1) 9 + (dy+1) 3 + (dx+1)) then
 * bias[cout], in network order; then the head's 16 weights and its bias. */
typedef struct slosh_unet_config_t {
    uint32_t dim[3];      /* grid (x, y, z), each a multiple of 8 and tileable into 128-voxel boxes per level */
    uint32_t batch;       /* samples per training step (slots) */
    uint32_t seed;        /* He-normal initialisation */
    float learning_rate;  /* Adam */
    float beta1, beta2, eps;
} slosh_unet_config_t;
SLOSH_API void slosh_unet_config_default(slosh_unet_config_t* out);
SLOSH_API slosh_status slosh_unet_create(const slosh_unet_config_t* config, int32_t device, void** out_net);
SLOSH_API void slosh_unet_destroy(void* net);
SLOSH_API const char* slosh_unet_last_error(void);
SLOSH_API uint64_t slosh_unet_num_params(void* net);
SLOSH_API slosh_status slosh_unet_get_params(void* net, float* host, uint64_t count);
SLOSH_API slosh_status slosh_unet_set_params(void* net, const float* host, uint64_t count);  /* also resets Adam */
/* Sample `slot` from host arrays: input [D][H][W][16] BF16 bits (channels as above, 3..15 zero),
 * target [D][H][W] (pressure / scale, 0 outside the fluid; may be NULL), its fluid voxel count. */
SLOSH_API slosh_status slosh_unet_set_sample(void* net, uint32_t slot, const uint16_t* input_bf16, const float* target,
                                             uint32_t fluid_voxels);
/* Sample `slot` from a simulation context: its divergence, cell types and current pressure (the
 * solution of the last substep's solve), on the device. */
SLOSH_API slosh_status slosh_unet_capture_sample(void* net, void* sim_ctx, uint32_t slot);
/* Forward pass over all slots; host_guess [B][D][H][W] (pressure / scale) may be NULL. */
SLOSH_API slosh_status slosh_unet_forward(void* net, float* host_guess);
/* After slosh_unet_forward: loss and parameter gradients (host_grads [num_params] may be NULL). */
SLOSH_API slosh_status slosh_unet_backward(void* net, float* out_loss, float* host_grads);
/* Forward, backward and one Adam step. */
SLOSH_API slosh_status slosh_unet_train_step(void* net, float* out_loss);
SLOSH_API uint64_t slosh_unet_launch_count(void* net);
/* Attaches (or with NULL detaches) the network used when warm_start = LEARNED; the network's grid
 * must equal the context's and its slot 0 is overwritten by each solve. */
SLOSH_API slosh_status slosh_set_warm_start_network(void* ctx, void* net);
/* One 3x3x3 convolution through the network's kernels (test entry): y = relu(conv(x) + bias) as BF16,
 * the data gradient dx (per K-block, BF16) of dz = dy, dW [27][cout][cin] and db (FP32). Arrays are
 * dense [batch][z][y][x][channels]; block channels and cout are 16, 32 or 64. */
typedef struct slosh_conv_test_t {
    uint32_t dim[3], batch;
    uint32_t nblocks;
    uint32_t cin[2];
    uint32_t cout;
    const uint16_t* x[2];
    const float* w;
    const float* bias;
    const uint16_t* dy;
    uint16_t* y;
    uint16_t* dx[2];
    float* dw;
    float* db;
} slosh_conv_test_t;
SLOSH_API slosh_status slosh_unet_conv_test(const slosh_conv_test_t* t);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SLOSH_CUDA_H */
