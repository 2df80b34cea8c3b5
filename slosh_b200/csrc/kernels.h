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
    int particle_ctas;  // upper bound for particle passes is computed per call
    int num_sms;
};

// ---- brick pool (Slosh.usf:1719-1831) ----
int launch_pool_update(const Dev& d, cudaStream_t s);
int launch_clear_new_slots(const Dev& d, const Shape& sh, cudaStream_t s);

// ---- grid passes ----
int launch_mark_cells(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s);
int launch_normalize_faces(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s);
int launch_viscosity(const Dev& d, const Pass& p, const float* ustar, const float* src, float* dst, const Shape& sh, cudaStream_t s);
int launch_divergence(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s);
int launch_rbgs(const Dev& d, float* pres, const float* rhs, uint32_t parity, float omega, const Shape& sh, cudaStream_t s);
int launch_project(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s);
int launch_residual(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s);
int launch_density_rhs(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s);
int launch_density_displacement(const Dev& d, float* dst, const Shape& sh, cudaStream_t s);
int launch_extrapolate(const Dev& d, const float* src, float* dst, uint32_t iteration, const Shape& sh, cudaStream_t s);

// ---- particles ----
int launch_emit_reserve(uint32_t* particle_count, uint32_t count, cudaStream_t s);
int launch_emit(const Dev& d, slosh_particle_t* particles, const uint32_t* particle_count, const slosh_emit_request_t& em,
                uint32_t count, uint32_t bound, uint32_t capacity, uint32_t seed, cudaStream_t s);
int launch_touch_particles(const Dev& d, const slosh_particle_t* particles, uint32_t n, cudaStream_t s);
int launch_p2g(const Dev& d, const Pass& p, const slosh_particle_t* particles, uint32_t n, cudaStream_t s);
int launch_g2p(const Dev& d, const Pass& p, slosh_particle_t* particles, uint32_t n, const float* vel, const float* disp,
               bool apply_density, cudaStream_t s);

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
size_t sort_scan_tmp_size(uint32_t capacity, uint32_t num_sort_keys);

// ---- MGPCG (SloshPressureMG.usf) ----
struct MGLevel {
    int3 dim;
    uint32_t cells;
    uint32_t* type;
    float* x;
    float* b;
};
struct MGState {
    int num_levels;
    MGLevel lv[SLOSH_MAX_MG_LEVELS];
    float* r;
    float* z;
    float* dvec;
    float* q;
    double* partials;     // one per brick entry (capacity num_pool_bricks)
    double* scalars;      // [0] rho, [1] scratch, [2] d.Ad, [3] previous rho, [4] ||b||^2, [5] ||r||^2, [6] true
    uint32_t* counters;   // last-CTA counters, one per reduction kind
};
int launch_mg_build_type(const Dev& d, const MGState& m, int l, cudaStream_t s);
int launch_pcg_init(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s);
int launch_mg_smooth(const Dev& d, const MGState& m, int l, uint32_t parity, bool dot, const Shape& sh, cudaStream_t s);
int launch_mg_restrict(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s);
int launch_mg_coarse_solve(const Dev& d, const MGState& m, int l, int iterations, cudaStream_t s);
int launch_mg_prolong(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s);
int launch_pcg_apply_a(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s);
int launch_pcg_update_pr(const Dev& d, const MGState& m, float* p, const Shape& sh, cudaStream_t s);
int launch_pcg_update_d(const Dev& d, const MGState& m, bool first, const Shape& sh, cudaStream_t s);
int launch_true_residual(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s);
// rho shift after a V-cycle: scalars[3] = scalars[0]; scalars[0] = scalars[1] (the r.z just reduced)
int launch_shift_rho(const MGState& m, cudaStream_t s);

}  // namespace slosh
