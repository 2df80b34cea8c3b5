// Host-side launch wrappers of the Slosh substep kernels. Each wrapper enqueues on `stream` and
// returns the number of kernels it launched.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace slosh {

// Launch shape shared by the brick passes: a grid-stride loop over the active-brick list, so the
// shape never depends on the (device-resident) active count.
struct Shape {
    int brick_ctas;     // CTAs of a brick pass (multiple of the SM count)
    int mg_ctas;        // CTAs of the level-0 MGPCG passes (one warp per brick; 3 per SM measured best)
    int particle_ctas;  // upper bound for particle passes is computed per call
    int num_sms;
};

// Launches kernel k on stream s, with programmatic stream serialisation unless SLOSH_PDL=0: the kernel may be
// scheduled before its predecessor in the stream completes, and must call pdl_entry() before anything else.
// The attribute survives stream capture as a programmatic edge of the graph.
bool pdl_enabled();
template <typename... P, typename... A>
inline cudaError_t launch_k(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
}

// ---- brick pool (Slosh.usf:1719-1831) ----
int launch_pool_update(const Dev& d, cudaStream_t s);
size_t pool_scratch_words(uint32_t num_bricks);
int launch_clear_new_slots(const Dev& d, const Shape& sh, cudaStream_t s);

// ---- grid passes ----
int launch_mark_cells(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s);
int launch_normalize_faces(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s);
int launch_viscosity(const Dev& d, const Pass& p, const float* ustar, const float* src, float* dst, const Shape& sh, cudaStream_t s);
int launch_divergence(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s);
int launch_rbgs(const Dev& d, float* pres, const float* rhs, uint32_t parity, float omega, const Shape& sh, cudaStream_t s);
int launch_project(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s);
int launch_residual(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s);
// Two-way collider coupling after the projection (wetted faces, binary force, seepage contacts and, with
// smooth coupling, the SDF-weighted force), and the per-frame submerged-cell estimate.
int launch_coupling(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s);
int launch_submerged(const Dev& d, const Shape& sh, cudaStream_t s);
int launch_density_rhs(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s);
int launch_density_displacement(const Dev& d, float* dst, const Shape& sh, cudaStream_t s);
// One layer of ExtrapolateFace, in place.
int launch_extrapolate(const Dev& d, float* vel, uint32_t iteration, const Shape& sh, cudaStream_t s);

// ---- particles ----
int launch_emit_reserve(uint32_t* particle_count, uint32_t count, cudaStream_t s);
int launch_emit(const Dev& d, slosh_particle_t* particles, const uint32_t* particle_count, const slosh_emit_request_t& em,
                uint32_t count, uint32_t bound, uint32_t capacity, uint32_t seed, cudaStream_t s);
int launch_touch_particles(const Dev& d, const slosh_particle_t* particles, uint32_t n, cudaStream_t s);
// unsorted: many particles were placed since the last sort (their order is emission order): the wider tile.
int launch_p2g(const Dev& d, const Pass& p, const slosh_particle_t* particles, uint32_t n, bool unsorted, cudaStream_t s);
int launch_g2p(const Dev& d, const Pass& p, slosh_particle_t* particles, uint32_t n, const float* vel, const float* disp,
               bool apply_density, cudaStream_t s);
// P2G as a per-brick gather (opt-in, SLOSH_P2G_GATHER=1): a per-cell particle index rebuilt every launch (counts
// into cell_count with the rank of each particle in its cell, an exclusive scan, a scatter of particle ids), then
// one CTA per active brick that visits the particles of the brick's cells and of the one-cell layer around it and
// writes the brick's 512 nodes x 6 sums with plain stores. Particles in cells of unallocated bricks (pool
// overflow) are added by a last pass with global adds.
struct P2GGather {
    uint32_t* rank;      // capacity: rank of the particle within its cell (~0u: dead or in an unallocated brick)
    uint32_t* index;     // capacity: particle ids in pool-cell order
    uint32_t* offsets;   // pool cells: exclusive scan of the counts
    uint32_t* overflow;  // capacity + 1: [0] count, then the ids of live particles in unallocated bricks
    uint32_t* scan_tmp;  // exclusive_scan_tmp_size(pool cells)
};
int launch_p2g_gather(const Dev& d, const Pass& p, const P2GGather& g, const slosh_particle_t* particles, uint32_t n,
                      cudaStream_t s);

// ---- spatial sort (SloshSort.usf) ----
struct SortBuffers {
    uint32_t* keys[2];
    uint32_t* vals[2];
    uint32_t* tile_hist;     // 256 x num_tiles
    uint32_t* scan_tmp;      // block sums of the scans
    uint32_t* counts;        // num_sort_keys
    uint32_t* offsets;       // num_sort_keys
    uint32_t* perm;          // capacity
    uint32_t* particle_count;
    size_t tile_hist_capacity;
    size_t scan_tmp_capacity;
};
int3 sort_brick_dim(int3 grid);
int launch_sort(const Dev& d, const SortBuffers& b, const slosh_particle_t* in, slosh_particle_t* out, uint32_t n,
                uint32_t num_sort_keys, int3 sort_dim, cudaStream_t s);
size_t sort_tile_hist_size(uint32_t capacity);
// Exclusive prefix sum of n u32 (in place allowed); tmp holds exclusive_scan_tmp_size(n) words.
int launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s);
size_t exclusive_scan_tmp_size(uint32_t n);
size_t sort_scan_tmp_size(uint32_t capacity, uint32_t num_sort_keys);

// ---- MGPCG (SloshPressureMG.usf) ----
struct MGLevel {
    int3 dim;
    uint32_t cells;
    uint32_t* type;
    float* x;
    float* b;
    uint16_t* word;   // per-solve stencil word: bits 0-5 fluid neighbour, 6 fluid, 7 red, 8-13 non-solid neighbour
    uint32_t prec;    // storage of x and b: SLOSH_PRECISION_FP32, _FP16_STORAGE (2-byte halves) or _BF16_STORAGE
};
struct MGState {
    int num_levels;
    MGLevel lv[SLOSH_MAX_MG_LEVELS];
    float* r;
    float* z;
    float* dvec;
    float* q;
    double* partials;     // one per brick entry, two dots (capacity 2 x num_pool_bricks)
    double* scalars;      // [0] rho, [2] d.Ad, [3] previous rho, [4] ||b||^2, [5] ||r||^2, [6..7] true residual, [8] tol,
                          // [9] r.z_prev (flexible PCG)
    uint32_t* counters;   // last-CTA counters, one per reduction kind
    uint32_t* ctl;        // [0] completed iterations, [1] limit, [2] tolerance mode, [3] done, [4] frame: a solve hit its limit
    uint8_t* word;        // level-0 stencil word per pool cell (fluid neighbours, fluid, red)
    uint32_t* nbr_slots;  // 8 per active-brick entry: slots of the 6 face-neighbour bricks
    float* dvec2;         // second search-direction buffer (d alternates by iteration parity)
    uint32_t* tail_list;  // per tail level: red fluid cells, then black fluid cells (dense indices)
    uint32_t* tail_meta;  // per level: [red offset, red count, black offset, black count]
    unsigned char* tail_image;  // per solve: the tail kernel's shared memory minus x and b (mg_tail_smem bytes)
    float restrict_scale;       // factor of the restriction's fluid-child sum: 0.25 x mg_correction_scale
    int sweeps;                 // red-black sweep pairs per pre- and post-smoothing (mg_smoothing_sweeps)
    uint32_t flexible;          // flexible PCG: UpdatePR also reduces r_{k+1}.z_k into scalars[9]
    float smooth_weight;        // over-relaxation of level 0's red-black sweeps (mg_smoother_weight; 1 = reference)
};
int launch_mg_words(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s);
int launch_mg_tail_lists(const MGState& m, cudaStream_t s);
size_t mg_tail_smem(const MGState& m);
// First level handled by the single-CTA tail kernel of the V-cycle.
int mg_tail_level(const MGState& m);
int launch_mg_setup(const MGState& m, uint32_t limit, bool tol_mode, double tol, cudaStream_t s);
int launch_mg_build_type(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s);
// Every coarse level's types and words (levels 1-3 fused: one launch for the types, one for the words).
int launch_mg_coarse_setup(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s);
// handle: the WHILE node's condition when the solve runs as a CUDA graph, 0 otherwise.
int launch_pcg_init(const Dev& d, const MGState& m, const float* p, const float* div, unsigned long long handle, const Shape& sh,
                    cudaStream_t s, bool words = true);
int launch_vcycle(const Dev& d, const MGState& m, int coarse_iterations, const Shape& sh, cudaStream_t s);
int launch_pcg_apply_a(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s);
int launch_pcg_update_pr(const Dev& d, const MGState& m, float* p, unsigned long long handle, const Shape& sh, cudaStream_t s);
int launch_pcg_update_d(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s);
int launch_true_residual(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s);

// ---- headless surface (SloshSurface.usf): density field and surface nets ----
struct SurfaceDev {
    int3 dim;               // field voxels
    int3 bdim;              // 8^3-voxel bricks of the field
    float inv_voxel, voxel; // voxels per sim metre, sim metres per voxel
    float support;          // SupportScale: kernel radius in splat radii
    float max_footprint;    // MaxFootprint (voxels)
    float radius_voxels;    // ParticleRadiusVoxels
    float splat_radius;     // SplatRadiusSim (sim metres)
    float iso;              // IsoLevel
    uint32_t max_vertices, max_indices;
    int32_t* accum;         // 5 fixed-point moments per voxel
    uint16_t* field;        // f16 field per voxel
    uint32_t* bricks;       // occupancy per field brick
    uint32_t* vflag;        // per cell (dim - 1)^3: has a vertex
    uint32_t* vbase;        // exclusive scan of vflag
    uint32_t* cell_vertex;  // vertex index or 0xFFFFFFFF
    uint32_t* qflag;        // quads per cell
    uint32_t* qbase;        // exclusive scan of qflag
    uint32_t* scan_tmp;
    float* positions;       // 3 per vertex (sim metres)
    float* normals;         // 3 per vertex
    float* tangents;        // 3 per vertex
    uint32_t* indices;      // 6 per quad
    uint32_t* counters;     // [0] vertices requested, [1] indices requested
};
// Splat, resolve and (with mesh) surface nets of the first n particle records.
int launch_surface(const SurfaceDev& s, const slosh_particle_t* particles, uint32_t n, bool mesh, cudaStream_t st);

}  // namespace slosh
