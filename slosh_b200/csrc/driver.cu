// Host driver and C ABI of the B200-native Slosh substep.
//
// Replaces FSloshProxy (PLUG/Source/SloshCore/Public/SloshProxy.h:23-147,
// PLUG/Source/SloshCore/Private/SloshProxy.cpp): Allocate (:185-306), EnsureParticleCapacity
// (:308-337), Step_RenderThread (:339-737), PollReadbacks_RenderThread's decode (:739-805),
// AddPressureSolveMGPCG (:807-1020) and AddSpatialSort (:1022-1087). Device work is issued on one CUDA
// stream; kernels read counts (active bricks, new slots, particle count) on the device, so a substep
// enqueues without host round trips except for the optional relative-residual test of MGPCG.
//
// Differences from the reference's host code, by design:
//   * results are read back synchronously at the end of each frame (the reference polls a 4-slot ring
//     2-4 frames late); the substep count therefore uses the previous frame's exact max speed;
//   * particle storage is sized to particle_capacity when the layout is allocated, and grows if the
//     capacity is raised;
//   * the three face-velocity buffers rotate roles instead of copying the final field into buffer 0
//     (SloshProxy.cpp:709-712); slosh_read_buffer(SLOSH_BUF_VEL) returns the current field;
//   * the grid and particle caps are raised (2048 cells per axis, 2^28 particles).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"

namespace slosh {
namespace unet {
struct Net;
int warm_start(Net* net, const Dev& d, const float* divergence, float* pressure, cudaStream_t s);  // unet.cu
}  // namespace unet
}  // namespace slosh

namespace slosh {
namespace {
// P2G as a per-brick gather instead of the shared-memory scatter (SLOSH_P2G_GATHER=1; read once per process).
bool p2g_gather_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("SLOSH_P2G_GATHER");
        return e != nullptr && std::atoi(e) != 0;
    }();
    return on;
}

thread_local std::string g_error;

struct CudaError {
    cudaError_t code;
    const char* what;
};
#define CK(call)                                                      \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) throw CudaError{e_, #call};            \
    } while (0)

struct StatusError {
    slosh_status code;
    std::string what;
};

constexpr uint32_t MG_COARSEST_MAX_CELLS = 512u;
constexpr int MG_MAX_LEVELS = 8;
constexpr int NUM_PHASES = SLOSH_NUM_PHASES;

slosh_settings_t defaults() {
    slosh_settings_t s;
    std::memset(&s, 0, sizeof(s));
    s.grid_dim[0] = 64; s.grid_dim[1] = 64; s.grid_dim[2] = 48;
    s.cell_size = 0.05f;
    s.particle_capacity = 262144u;
    s.transfer_mode = SLOSH_TRANSFER_APIC;
    s.flip_ratio = 0.95f;
    s.density = 1000.0f;
    s.adhesion_distance = 0.025f;
    s.density_correction = 0.15f;
    s.density_deadband = 0.05f;
    s.two_sided_density_projection = 1u;
    s.density_relaxation = 0.5f;
    s.density_projection_iterations = 30;
    s.density_projection_interval = 1;
    s.sparse_bricks = 1u;
    s.sparse_max_active_fraction = 0.5f;
    s.sparse_storage_budget = 1.0f;
    s.particle_radius_cells = 0.25f;
    s.gravity[2] = -9.81f;
    s.pressure_solver = SLOSH_SOLVER_MGPCG;
    s.pressure_iterations = 60;
    s.sor_weight = 1.7f;
    s.pcg_iterations = 8;
    s.mg_coarse_iterations = 16;
    s.sort_interval = 4;
    s.smooth_coupling_force = 1u;
    s.ghost_fluid = 1u;
    s.viscosity_iterations = 12;
    s.extrapolation_layers = 2;
    s.min_substeps = 1;
    s.max_substeps = 4;
    s.max_frame_dt = 1.0f / 30.0f;
    s.cfl = 2.0f;
    s.max_speed = 20.0f;
    s.tolerance = 0.0f;
    s.max_iterations = 200;
    s.precision_mode = SLOSH_PRECISION_FP32;
    s.warm_start = SLOSH_WARM_START_PREVIOUS;
    s.mg_correction_scale = 1.0f;
    s.mg_smoothing_sweeps = 1;
    s.pcg_flexible = 0u;
    s.mg_smoother_weight = 1.0f;
    return s;
}

inline float clampf_h(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }
inline int clampi_h(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

slosh_settings_t clamp_settings(slosh_settings_t s) {  // SloshProxy.cpp:344-347 (caps raised)
    for (int a = 0; a < 3; ++a) s.grid_dim[a] = clampi_h(s.grid_dim[a], 4, 2048);
    s.particle_capacity = std::min(std::max(s.particle_capacity, 1024u), 1u << 28);
    s.cell_size = std::max(s.cell_size, 1e-3f);
    return s;
}
bool layout_equals(const slosh_settings_t& a, const slosh_settings_t& b) {
    return a.grid_dim[0] == b.grid_dim[0] && a.grid_dim[1] == b.grid_dim[1] && a.grid_dim[2] == b.grid_dim[2] &&
           a.sparse_storage_budget == b.sparse_storage_budget;
}

struct Ctx {
    int device = 0;
    slosh::unet::Net* warm_net = nullptr;  // learned warm start (not owned)
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    slosh_settings_t S{};
    bool allocated = false;

    // layout
    int3 grid{}, brick_dim{}, sort_dim{};
    uint32_t num_cells = 0, num_bricks = 0, num_pool_bricks = 0, pool_cells = 0, total_faces = 0, num_sort_keys = 0;
    int num_levels = 0;
    int3 level_dim[MG_MAX_LEVELS]{};
    uint32_t level_cells[MG_MAX_LEVELS]{};

    // device memory
    std::vector<void*> grid_allocs;
    std::vector<void*> particle_allocs;
    uint64_t grid_bytes = 0, particle_bytes = 0;
    slosh_particle_t* particles[2] = {nullptr, nullptr};
    int pbuf = 0;
    uint32_t capacity = 0;
    float* vel[3] = {nullptr, nullptr, nullptr};
    int vmap[3] = {0, 1, 2};
    int disp_phys = 2;
    float* vel_old = nullptr;
    int32_t* accum = nullptr;
    uint32_t* face_flags = nullptr;
    float* face_weight = nullptr;
    uint32_t* cell_type = nullptr;
    int32_t* cell_count = nullptr;
    float *pressure = nullptr, *divergence = nullptr, *cell_diag = nullptr, *density_q = nullptr, *density_rhs = nullptr;
    uint32_t *brick_table = nullptr, *slot_brick = nullptr, *free_slots = nullptr, *brick_touch = nullptr;
    uint32_t *brick_want = nullptr, *new_slots = nullptr, *active_bricks = nullptr, *pool_scratch = nullptr;
    uint32_t* stats = nullptr;
    int32_t* coupling = nullptr;
    slosh_collider_t* colliders_d = nullptr;
    slosh_manipulator_t* manipulators_d = nullptr;
    uint32_t* particle_count = nullptr;
    SortBuffers sortb{};
    P2GGather gather{};  // the per-cell particle index of the gather P2G (allocated only when it is on)
    MGState mg{};

    // pinned host staging
    slosh_collider_t* h_colliders = nullptr;
    slosh_manipulator_t* h_manipulators = nullptr;
    uint32_t* h_stats = nullptr;     // [0..15] stats, [16..19] particle count
    double* h_scalars = nullptr;     // [0..7] device scalars, [8..9] ||b||^2, ||r||^2 of the last pressure solve
    int32_t* h_coupling = nullptr;

    // simulation state on the host
    uint32_t num_particles = 0;
    uint64_t placed_since_sort = 0;  // particles emitted or uploaded since the last sort (in placement order)
    uint64_t total_emitted = 0, sim_frame = 0;
    uint32_t emit_seed = 1;
    float prev_dt = 0.0f, last_max_speed = 0.0f;
    Pass P{};
    Shape shape{};
    uint32_t num_colliders = 0, num_manipulators = 0;
    int substeps = 0;
    float dt = 0.0f;
    bool density_frame = false;
    int last_iterations = 0;
    float last_rel = 0.0f, last_true_rel = 0.0f;
    bool last_converged = true;
    uint32_t mg_prec = SLOSH_PRECISION_FP32;  // storage precision of the coarse MG levels (precision_mode)
    bool pool_overflow_seen = false;
    bool rel_pending = false;
    bool solve_tol_mode = false;
    float solve_tol = 0.0f;

    // MGPCG solves as CUDA graphs: pre-nodes, then a WHILE node whose body is one PCG iteration
    struct SolveGraph {
        float* p;
        const float* div;
        uint32_t limit;
        bool tol_mode;
        float tol;
        int coarse;
        bool setup;
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        int pre_nodes, body_nodes;
    };
    std::vector<SolveGraph> graphs;
    cudaStream_t cap_stream = nullptr, body_stream = nullptr;
    bool use_graphs = true;
    uint32_t* h_ctl = nullptr;          // pinned: [0..3] ctl of the pressure solve, [4..7] of the density solve
    struct SolveRecord { int pre, body, slot; };
    std::vector<SolveRecord> frame_solves;

    // timing
    bool timing = false;
    std::vector<cudaEvent_t> event_pool;
    size_t event_next = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> phase_events;
    float phase_ms[NUM_PHASES] = {};
    uint64_t launches = 0;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;

    // ---------------------------------------------------------------------------------------------
    template <class T>
    T* dalloc(size_t count, bool particle, uint64_t* bytes_out = nullptr) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw StatusError{SLOSH_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes failed"};
        }
        (particle ? particle_allocs : grid_allocs).push_back(p);
        (particle ? particle_bytes : grid_bytes) += bytes;
        (void)bytes_out;
        return static_cast<T*>(p);
    }
    void free_list(std::vector<void*>& v) {
        for (void* p : v) cudaFree(p);
        v.clear();
    }
    // CTAs of the brick passes: a multiple of the SM count, at most one per pool brick. The solve graphs
    // hold the grid sizes, so a change re-captures them. Every brick pass is a grid-stride loop whose
    // results do not depend on the grid size.
    uint32_t ctas_per_sm = 8;
    int brick_ctas_for(uint32_t per_sm) const {
        return std::max(1, std::min<int>(int(num_pool_bricks > 1u ? num_pool_bricks - 1u : 1u), num_sms * int(per_sm)));
    }
    uint32_t mg_ctas_per_sm = 3;  // = the CTAs of these 80-register kernels resident per SM: one wave
    void set_mg_ctas_per_sm(uint32_t per_sm) {
        per_sm = std::max(1u, std::min(per_sm, 32u));
        mg_ctas_per_sm = per_sm;
        if (!allocated) return;
        const int bc = brick_ctas_for(per_sm);
        if (bc != shape.mg_ctas) {
            CK(cudaStreamSynchronize(stream));
            destroy_graphs();
            shape.mg_ctas = bc;
        }
    }
    void set_ctas_per_sm(uint32_t per_sm) {
        per_sm = std::max(1u, std::min(per_sm, 32u));
        ctas_per_sm = per_sm;
        if (!allocated) return;
        const int bc = brick_ctas_for(per_sm);
        if (bc != shape.brick_ctas) {
            CK(cudaStreamSynchronize(stream));
            destroy_graphs();
            shape.brick_ctas = bc;
        }
    }
    void destroy_graphs() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
        }
        graphs.clear();
    }
    // ---- headless surface (SloshSurface.usf) ----
    SurfaceDev surf{};
    std::vector<void*> surface_allocs;
    uint64_t surf_voxels_cap = 0, surf_cells_cap = 0, surf_bricks_cap = 0, surf_vert_cap = 0, surf_idx_cap = 0;
    slosh_surface_info_t surf_info{};
    uint32_t* h_surf = nullptr;  // pinned: the two counters
    template <class T>
    T* salloc(uint64_t count) {
        void* p = nullptr;
        const size_t bytes = size_t(std::max<uint64_t>(count, 1)) * sizeof(T);
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            throw StatusError{SLOSH_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes for the surface failed"};
        }
        surface_allocs.push_back(p);
        return static_cast<T*>(p);
    }
    void build_surface(const slosh_surface_params_t& q);

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        destroy_graphs();
        free_list(grid_allocs);
        free_list(particle_allocs);
        free_list(surface_allocs);
        surf_voxels_cap = surf_cells_cap = surf_bricks_cap = surf_vert_cap = surf_idx_cap = 0;
        surf = SurfaceDev{};
        surf_info = slosh_surface_info_t{};
        grid_bytes = particle_bytes = 0;
        allocated = false;
    }

    void compute_layout(const slosh_settings_t& s) {
        grid = make_int3(s.grid_dim[0], s.grid_dim[1], s.grid_dim[2]);
        num_cells = uint32_t(grid.x) * uint32_t(grid.y) * uint32_t(grid.z);
        brick_dim = make_int3((grid.x + 7) / 8, (grid.y + 7) / 8, (grid.z + 7) / 8);
        num_bricks = uint32_t(brick_dim.x) * uint32_t(brick_dim.y) * uint32_t(brick_dim.z);
        const double budget = double(clampf_h(s.sparse_storage_budget, 0.0f, 1.0f));
        uint32_t slots = uint32_t(std::ceil(budget * double(num_bricks)));
        slots = std::min(std::max(slots, 1u), num_bricks);
        num_pool_bricks = slots + 1u;
        pool_cells = num_pool_bricks * BRICK_CELLS;
        total_faces = 3u * pool_cells;
        sort_dim = sort_brick_dim(grid);
        num_sort_keys = uint32_t(sort_dim.x) * uint32_t(sort_dim.y) * uint32_t(sort_dim.z) + 1u;
        num_levels = 1;
        level_dim[0] = grid;
        level_cells[0] = num_cells;
        while (level_cells[num_levels - 1] > MG_COARSEST_MAX_CELLS && num_levels < MG_MAX_LEVELS) {
            const int3 p = level_dim[num_levels - 1];
            const int3 dd = make_int3((p.x + 1) / 2, (p.y + 1) / 2, (p.z + 1) / 2);
            level_dim[num_levels] = dd;
            level_cells[num_levels] = uint32_t(dd.x) * uint32_t(dd.y) * uint32_t(dd.z);
            ++num_levels;
        }
    }

    void alloc_particles(uint32_t cap) {
        free_list(particle_allocs);
        particle_bytes = 0;
        capacity = cap;
        particles[0] = dalloc<slosh_particle_t>(cap, true);
        particles[1] = dalloc<slosh_particle_t>(cap, true);
        sortb.keys[0] = dalloc<uint32_t>(cap, true);
        sortb.keys[1] = dalloc<uint32_t>(cap, true);
        sortb.vals[0] = dalloc<uint32_t>(cap, true);
        sortb.vals[1] = dalloc<uint32_t>(cap, true);
        sortb.perm = dalloc<uint32_t>(cap, true);
        sortb.tile_hist_capacity = sort_tile_hist_size(cap);
        sortb.tile_hist = dalloc<uint32_t>(sortb.tile_hist_capacity, true);
        sortb.scan_tmp_capacity = sort_scan_tmp_size(cap, num_sort_keys);
        sortb.scan_tmp = dalloc<uint32_t>(sortb.scan_tmp_capacity, true);
        if (p2g_gather_enabled()) {
            gather.rank = dalloc<uint32_t>(cap, true);
            gather.index = dalloc<uint32_t>(cap, true);
            gather.overflow = dalloc<uint32_t>(size_t(cap) + 1u, true);
        }
        pbuf = 0;
    }

    // Allocate (SloshProxy.cpp:185-306).
    void allocate(const slosh_settings_t& s) {
        release();
        S = s;
        compute_layout(s);
        alloc_particles(s.particle_capacity);
        num_particles = 0;
        placed_since_sort = 0;
        const size_t tf = total_faces, pc = pool_cells;
        for (int i = 0; i < 3; ++i) vel[i] = dalloc<float>(tf, false);
        vmap[0] = 0; vmap[1] = 1; vmap[2] = 2;
        disp_phys = 2;
        vel_old = dalloc<float>(tf, false);
        accum = dalloc<int32_t>(2 * tf, false);
        face_flags = dalloc<uint32_t>(tf, false);
        face_weight = dalloc<float>(tf, false);
        cell_type = dalloc<uint32_t>(pc, false);
        cell_count = dalloc<int32_t>(pc, false);
        if (p2g_gather_enabled()) {
            gather.offsets = dalloc<uint32_t>(pc, false);
            gather.scan_tmp = dalloc<uint32_t>(exclusive_scan_tmp_size(pc), false);
        }
        pressure = dalloc<float>(pc, false);
        divergence = dalloc<float>(pc, false);
        cell_diag = dalloc<float>(pc, false);
        density_q = dalloc<float>(pc, false);
        density_rhs = dalloc<float>(pc, false);
        coupling = dalloc<int32_t>(SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE, false);
        stats = dalloc<uint32_t>(SLOSH_NUM_STATS, false);
        particle_count = dalloc<uint32_t>(4, false);
        active_bricks = dalloc<uint32_t>(num_bricks + 1u, false);
        brick_table = dalloc<uint32_t>(num_bricks, false);
        brick_touch = dalloc<uint32_t>(num_bricks, false);
        brick_want = dalloc<uint32_t>(num_bricks, false);
        pool_scratch = dalloc<uint32_t>(pool_scratch_words(num_bricks), false);
        new_slots = dalloc<uint32_t>(num_pool_bricks + 1u, false);
        slot_brick = dalloc<uint32_t>(num_pool_bricks, false);
        free_slots = dalloc<uint32_t>(num_pool_bricks, false);
        colliders_d = dalloc<slosh_collider_t>(SLOSH_MAX_COLLIDERS, false);
        manipulators_d = dalloc<slosh_manipulator_t>(SLOSH_MAX_MANIPULATORS, false);
        sortb.counts = dalloc<uint32_t>(num_sort_keys, false);
        sortb.offsets = dalloc<uint32_t>(num_sort_keys, false);
        sortb.particle_count = particle_count;
        mg.num_levels = num_levels;
        for (int l = 0; l < num_levels; ++l) {
            mg.lv[l].dim = level_dim[l];
            mg.lv[l].cells = level_cells[l];
            if (l > 0) {
                mg.lv[l].type = dalloc<uint32_t>(level_cells[l], false);
                mg.lv[l].x = dalloc<float>((level_cells[l] + 3u) & ~3u, false);  // padded: read as 16-byte chunks
                mg.lv[l].b = dalloc<float>((level_cells[l] + 3u) & ~3u, false);
                mg.lv[l].word = dalloc<uint16_t>(level_cells[l], false);
                mg.lv[l].prec = mg_prec;
            } else {
                mg.lv[l].type = nullptr; mg.lv[l].x = nullptr; mg.lv[l].b = nullptr; mg.lv[l].word = nullptr;
                mg.lv[l].prec = SLOSH_PRECISION_FP32;  // level 0 (the pool) is always FP32
            }
        }
        mg.r = dalloc<float>(pc, false);
        mg.z = dalloc<float>(pc, false);
        mg.dvec = dalloc<float>(pc, false);
        mg.dvec2 = dalloc<float>(pc, false);
        mg.word = dalloc<uint8_t>(pc, false);
        mg.nbr_slots = dalloc<uint32_t>(8 * size_t(num_pool_bricks), false);
        mg.q = dalloc<float>(pc, false);
        mg.partials = dalloc<double>(2 * size_t(num_pool_bricks), false);
        mg.scalars = dalloc<double>(16, false);
        mg.counters = dalloc<uint32_t>(8, false);
        mg.ctl = dalloc<uint32_t>(8, false);
        {
            size_t tail_cells = 0;
            for (int l = 1; l < num_levels; ++l) tail_cells += level_cells[l];
            mg.tail_list = dalloc<uint32_t>(tail_cells + 1, false);
            mg.tail_meta = dalloc<uint32_t>(4 * SLOSH_MAX_MG_LEVELS, false);
            mg.tail_image = dalloc<unsigned char>(mg_tail_smem(mg) + 16, false);
        }
        // zero everything (AddClearUAVPass of every buffer), then the free stack and the slot table
        zero_all();
        std::vector<uint32_t> free_init(num_pool_bricks);
        const uint32_t pool_slots = num_pool_bricks - 1u;
        free_init[0] = pool_slots;
        for (uint32_t sl = 1; sl <= pool_slots; ++sl) free_init[sl] = sl;
        CK(cudaMemcpy(free_slots, free_init.data(), sizeof(uint32_t) * num_pool_bricks, cudaMemcpyHostToDevice));
        CK(cudaMemset(slot_brick, 0xFF, sizeof(uint32_t) * num_pool_bricks));
        // The clears above run on the legacy default stream, which the context's non-blocking streams do
        // not wait for: finish them before any frame work is issued.
        CK(cudaDeviceSynchronize());
        total_emitted = 0;
        prev_dt = 0.0f;
        last_max_speed = 0.0f;
        shape.num_sms = num_sms;
        shape.brick_ctas = brick_ctas_for(ctas_per_sm);
        shape.mg_ctas = brick_ctas_for(mg_ctas_per_sm);
        allocated = true;
    }
    void zero_all() {
        const size_t tf = total_faces, pc = pool_cells;
        for (int i = 0; i < 3; ++i) CK(cudaMemset(vel[i], 0, tf * 4));
        CK(cudaMemset(vel_old, 0, tf * 4));
        CK(cudaMemset(accum, 0, 2 * tf * 4));
        CK(cudaMemset(face_flags, 0, tf * 4));
        CK(cudaMemset(face_weight, 0, tf * 4));
        for (void* p : {(void*)cell_type, (void*)cell_count, (void*)pressure, (void*)divergence, (void*)cell_diag, (void*)density_q,
                        (void*)density_rhs, (void*)mg.r, (void*)mg.z, (void*)mg.dvec, (void*)mg.dvec2, (void*)mg.q})
            CK(cudaMemset(p, 0, pc * 4));
        CK(cudaMemset(mg.word, 0, pc));
        CK(cudaMemset(mg.nbr_slots, 0, 8 * size_t(num_pool_bricks) * 4));
        CK(cudaMemset(coupling, 0, SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE * 4));
        CK(cudaMemset(stats, 0, SLOSH_NUM_STATS * 4));
        CK(cudaMemset(particle_count, 0, 16));
        CK(cudaMemset(active_bricks, 0, (num_bricks + 1) * 4));
        CK(cudaMemset(brick_table, 0, num_bricks * 4));
        CK(cudaMemset(brick_touch, 0, num_bricks * 4));
        CK(cudaMemset(brick_want, 0, num_bricks * 4));
        CK(cudaMemset(new_slots, 0, (num_pool_bricks + 1) * 4));
        CK(cudaMemset(sortb.counts, 0, num_sort_keys * 4));
        CK(cudaMemset(sortb.offsets, 0, num_sort_keys * 4));
        for (int l = 1; l < num_levels; ++l) {
            CK(cudaMemset(mg.lv[l].type, 0, level_cells[l] * 4));
            CK(cudaMemset(mg.lv[l].x, 0, level_cells[l] * 4));
            CK(cudaMemset(mg.lv[l].b, 0, level_cells[l] * 4));
            CK(cudaMemset(mg.lv[l].word, 0, level_cells[l] * 2));
        }
        CK(cudaMemset(mg.scalars, 0, 16 * sizeof(double)));
        CK(cudaMemset(mg.counters, 0, 8 * 4));
        CK(cudaMemset(mg.ctl, 0, 8 * 4));
        CK(cudaMemset(mg.partials, 0, 2 * size_t(num_pool_bricks) * sizeof(double)));
        CK(cudaMemset(particles[0], 0, size_t(capacity) * sizeof(slosh_particle_t)));
    }

    // EnsureParticleCapacity (SloshProxy.cpp:308-337): grow, keeping the particles in use.
    void ensure_capacity(uint32_t cap) {
        if (cap <= capacity) return;
        CK(cudaStreamSynchronize(stream));
        std::vector<slosh_particle_t> keep(num_particles);
        if (num_particles)
            CK(cudaMemcpy(keep.data(), particles[pbuf], sizeof(slosh_particle_t) * num_particles, cudaMemcpyDeviceToHost));
        alloc_particles(cap);
        CK(cudaMemset(particles[0], 0, size_t(cap) * sizeof(slosh_particle_t)));
        if (num_particles)
            CK(cudaMemcpy(particles[0], keep.data(), sizeof(slosh_particle_t) * num_particles, cudaMemcpyHostToDevice));
        CK(cudaDeviceSynchronize());  // the clear (default stream) before the frame's emission (context stream)
    }

    Dev dev() const {
        Dev d;
        d.grid = grid;
        d.brick_dim = brick_dim;
        d.num_bricks = num_bricks;
        d.num_pool_bricks = num_pool_bricks;
        d.pool_cells = pool_cells;
        d.total_faces = total_faces;
        d.h = S.cell_size;
        d.inv_h = 1.0f / S.cell_size;
        d.brick_table = brick_table;
        d.brick_table_w = brick_table;
        d.slot_brick = slot_brick;
        d.free_slots = free_slots;
        d.brick_touch = brick_touch;
        d.brick_want = brick_want;
        d.pool_scratch = pool_scratch;
        d.new_slots = new_slots;
        d.active_bricks = active_bricks;
        d.cell_type = cell_type;
        d.cell_count = cell_count;
        d.pressure = pressure;
        d.divergence = divergence;
        d.cell_diag = cell_diag;
        d.density_q = density_q;
        d.density_rhs = density_rhs;
        d.accum = accum;
        d.face_flags = face_flags;
        d.face_weight = face_weight;
        d.vel_old = vel_old;
        d.stats = stats;
        d.coupling = coupling;
        d.colliders = colliders_d;
        d.manipulators = manipulators_d;
        return d;
    }

    // ---- timing ----
    cudaEvent_t next_event() {
        if (event_next == event_pool.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            event_pool.push_back(e);
        }
        return event_pool[event_next++];
    }
    struct PhaseScope {
        Ctx* c;
        int phase;
        cudaEvent_t end;
        PhaseScope(Ctx* ctx, int ph) : c(ctx), phase(ph), end(nullptr) {
            if (!c->timing) return;
            cudaEvent_t s = c->next_event();
            end = c->next_event();
            CK(cudaEventRecord(s, c->stream));
            c->phase_events.push_back({phase, {s, end}});
        }
        ~PhaseScope() {
            if (end) cudaEventRecord(end, c->stream);
        }
    };
    void count(int n) { launches += uint64_t(n); }

    // ---- pass parameters (Step_RenderThread, SloshProxy.cpp:400-483) ----
    void set_pass_params(const slosh_frame_input_t& in) {
        const slosh_settings_t& s = S;
        num_colliders = std::min<uint32_t>(in.num_colliders, SLOSH_MAX_COLLIDERS);
        num_manipulators = std::min<uint32_t>(in.num_manipulators, SLOSH_MAX_MANIPULATORS);
        if (num_colliders && !in.colliders) throw StatusError{SLOSH_ERR_INVALID_ARG, "colliders is NULL"};
        if (num_manipulators && !in.manipulators) throw StatusError{SLOSH_ERR_INVALID_ARG, "manipulators is NULL"};
        if (num_colliders) {
            std::memcpy(h_colliders, in.colliders, sizeof(slosh_collider_t) * num_colliders);
            CK(cudaMemcpyAsync(colliders_d, h_colliders, sizeof(slosh_collider_t) * num_colliders, cudaMemcpyHostToDevice, stream));
            h2d_bytes += sizeof(slosh_collider_t) * num_colliders;
        }
        if (num_manipulators) {
            std::memcpy(h_manipulators, in.manipulators, sizeof(slosh_manipulator_t) * num_manipulators);
            CK(cudaMemcpyAsync(manipulators_d, h_manipulators, sizeof(slosh_manipulator_t) * num_manipulators, cudaMemcpyHostToDevice,
                               stream));
            h2d_bytes += sizeof(slosh_manipulator_t) * num_manipulators;
        }
        const float h = s.cell_size;
        P.num_colliders = num_colliders;
        P.num_manipulators = num_manipulators;
        for (int a = 0; a < 3; ++a) P.gravity[a] = s.gravity[a];
        P.flip_ratio = clampf_h(s.flip_ratio, 0.0f, 1.0f);
        P.use_apic = s.transfer_mode == SLOSH_TRANSFER_APIC ? 1u : 0u;
        P.max_speed = std::max(s.max_speed, 0.1f);
        P.friction = clampf_h(s.boundary_friction, 0.0f, 1.0f);
        const float gmag = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
        P.adhesion_accel = std::max(s.adhesion, 0.0f) * 1.5f * gmag;
        P.adhesion_range = std::max(s.adhesion_distance, 1e-4f);
        P.particle_radius = s.particle_radius_cells * h;
        P.density_correction = s.two_sided_density_projection ? 0.0f : std::max(s.density_correction, 0.0f);
        P.target_ppc = 8.0f;
        P.density_deadband = std::max(s.density_deadband, 0.0f);
        P.warm_start_scale = 1.0f;
        P.ghost_fluid = s.ghost_fluid ? 1u : 0u;
        P.smooth_coupling = s.smooth_coupling_force ? 1u : 0u;
        const int interval = clampi_h(s.density_projection_interval, 1, 8);
        P.density_relaxation = 1.0f - std::pow(1.0f - clampf_h(s.density_relaxation, 0.0f, 1.0f), float(interval));
    }

    // ---- emission (Step_RenderThread :485-541) ----
    void emit(const slosh_emit_request_t& em) {
        uint64_t cnt = em.count;
        if (em.shape == SLOSH_EMIT_FILL_CELLS)
            cnt = uint64_t(std::max(em.cell_dims[0], 0)) * uint64_t(std::max(em.cell_dims[1], 0)) * uint64_t(std::max(em.cell_dims[2], 0)) * 8ull;
        cnt = std::min<uint64_t>(cnt, uint64_t(capacity) - std::min(num_particles, capacity));
        if (cnt == 0) return;
        const uint32_t bound = num_particles;
        const Dev d = dev();
        count(launch_emit_reserve(particle_count, uint32_t(cnt), stream));
        count(launch_emit(d, particles[pbuf], particle_count, em, uint32_t(cnt), bound, capacity, emit_seed++, stream));
        total_emitted += cnt;
        num_particles += uint32_t(cnt);
        placed_since_sort += cnt;
    }

    void sort_particles() {
        PhaseScope ps(this, 0);
        count(launch_sort(dev(), sortb, particles[pbuf], particles[pbuf ^ 1], num_particles, num_sort_keys, sort_dim, stream));
        pbuf ^= 1;
        placed_since_sort = 0;
    }

    // ---- MGPCG driver (AddPressureSolveMGPCG, SloshProxy.cpp:807-1020) ----
    // Sequence of one solve: setup, coarse cell types, PCGInit, then while the device says so:
    // V-cycle, UpdateD, ApplyA, UpdatePR. This is the reference's order (init, V-cycle, UpdateD(first),
    // then per iteration ApplyA, UpdatePR and -- unless it was the last -- V-cycle, UpdateD).
    // setup: build the per-solve structure (coarse types, stencil words, tail lists) from the cell types; the
    // density solve of the frame's last substep runs on the types its pressure solve just used and skips it.
    int enqueue_pre(const Dev& d, float* p, const float* div, uint32_t limit, bool tol_mode, float tol, unsigned long long handle,
                    cudaStream_t s, bool setup) {
        int n = launch_mg_setup(mg, limit, tol_mode, double(tol), s);
        if (setup) {
            n += launch_mg_coarse_setup(d, mg, shape, s);
            n += launch_mg_tail_lists(mg, s);
        }
        n += launch_pcg_init(d, mg, p, div, handle, shape, s, setup);
        return n;
    }
    int enqueue_body(const Dev& d, float* p, int coarse, unsigned long long handle, cudaStream_t s) {
        int n = launch_vcycle(d, mg, coarse, shape, s);
        n += launch_pcg_update_d(d, mg, shape, s);
        n += launch_pcg_apply_a(d, mg, shape, s);
        n += launch_pcg_update_pr(d, mg, p, handle, shape, s);
        return n;
    }
    SolveGraph* solve_graph(float* p, const float* div, uint32_t limit, bool tol_mode, float tol, int coarse, bool setup) {
        for (auto& g : graphs)
            if (g.p == p && g.div == div && g.limit == limit && g.tol_mode == tol_mode && g.tol == tol && g.coarse == coarse && g.setup == setup)
                return &g;
        const Dev d = dev();
        SolveGraph G{p, div, limit, tol_mode, tol, coarse, setup, nullptr, nullptr, 0, 0};
        CK(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t cg = nullptr;
        try {
            cudaStreamCaptureStatus st;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            CK(cudaStreamGetCaptureInfo(cap_stream, &st, nullptr, &cg, &deps, &nd));
            cudaGraphConditionalHandle h;
            CK(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
            G.pre_nodes = enqueue_pre(d, p, div, limit, tol_mode, tol, h, cap_stream, setup);
            CK(cudaStreamGetCaptureInfo(cap_stream, &st, nullptr, &cg, &deps, &nd));
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cn;
            CK(cudaGraphAddNode(&cn, cg, deps, nd, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            CK(cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            G.body_nodes = enqueue_body(d, p, coarse, h, body_stream);
            CK(cudaStreamEndCapture(body_stream, &body));
            CK(cudaStreamUpdateCaptureDependencies(cap_stream, &cn, 1, cudaStreamSetCaptureDependencies));
            CK(cudaStreamEndCapture(cap_stream, &G.graph));
            CK(cudaGraphInstantiate(&G.exec, G.graph, 0));
        } catch (...) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(body_stream, &junk);
            if (junk) cudaGraphDestroy(junk);
            junk = nullptr;
            cudaStreamEndCapture(cap_stream, &junk);
            if (junk) cudaGraphDestroy(junk);
            if (G.graph) cudaGraphDestroy(G.graph);
            cudaGetLastError();
            throw;
        }
        graphs.push_back(G);
        return &graphs.back();
    }
    // slot 0: the pressure solve, whose statistics are read back at the end of the frame; slot 1: the density
    // solve, which follows slot 0's solve in the same substep on the same cell types and reuses its setup.
    void mgpcg(float* p, const float* div, int fixed_iterations, float tolerance, int max_iterations, int coarse_iterations,
               int slot) {
        const bool tol_mode = fixed_iterations <= 0;
        const uint32_t limit = tol_mode ? uint32_t(std::max(max_iterations, 1)) : uint32_t(std::min(std::max(fixed_iterations, 1), 100));
        const Dev d = dev();
        SolveGraph* G = nullptr;
        if (use_graphs) {
            try {
                G = solve_graph(p, div, limit, tol_mode, tolerance, coarse_iterations, slot == 0);
            } catch (const CudaError& e) {
                std::fprintf(stderr, "slosh: CUDA graph capture of the solve failed (%s: %s); issuing kernels directly\n", e.what,
                             cudaGetErrorString(e.code));
                use_graphs = false;
                destroy_graphs();
            }
        }
        if (G) {
            CK(cudaGraphLaunch(G->exec, stream));
            frame_solves.push_back({G->pre_nodes, G->body_nodes, slot});
        } else {
            int pre = enqueue_pre(d, p, div, limit, tol_mode, tolerance, 0ull, stream, slot == 0);
            int body = 0;
            for (uint32_t it = 0; it < limit; ++it) {
                CK(cudaMemcpyAsync(h_ctl + 4 * slot, mg.ctl, 16, cudaMemcpyDeviceToHost, stream));
                d2h_bytes += 16;
                CK(cudaStreamSynchronize(stream));
                if (h_ctl[4 * slot + 3]) break;
                body = enqueue_body(d, p, coarse_iterations, 0ull, stream);
            }
            frame_solves.push_back({pre, body, slot});
        }
        CK(cudaMemcpyAsync(h_ctl + 4 * slot, mg.ctl, 16, cudaMemcpyDeviceToHost, stream));
        d2h_bytes += 16;
        if (slot == 0) {
            CK(cudaMemcpyAsync(h_scalars + 8, mg.scalars + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
            d2h_bytes += 2 * sizeof(double);
            rel_pending = true;
            solve_tol_mode = tol_mode;
            solve_tol = tolerance;
        }
    }

    // ---- frame prologue (Step_RenderThread :339-562) ----
    int begin_frame(const slosh_frame_input_t& in) {
        const slosh_settings_t s = clamp_settings(in.settings);
        if (in.reset || !allocated || !layout_equals(s, S)) allocate(s);
        ensure_capacity(s.particle_capacity);
        S = s;
        {  // storage precision of the coarse MG levels; the solve graphs hold the level descriptors
            const uint32_t prec = s.precision_mode <= uint32_t(SLOSH_PRECISION_BF16_STORAGE) ? s.precision_mode : uint32_t(SLOSH_PRECISION_FP32);
            if (prec != mg_prec) {
                CK(cudaStreamSynchronize(stream));
                destroy_graphs();
                mg_prec = prec;
                for (int l = 1; l < mg.num_levels; ++l) mg.lv[l].prec = prec;
            }
            // preconditioner options (the solve graphs hold the MGState by value)
            const float restrict_scale = 0.25f * clampf_h(s.mg_correction_scale, 0.5f, 1.95f);
            const int sweeps = clampi_h(s.mg_smoothing_sweeps, 1, 4);
            const uint32_t flexible = s.pcg_flexible ? 1u : 0u;
            const float smooth_weight = clampf_h(s.mg_smoother_weight, 0.5f, 1.9f);
            if (restrict_scale != mg.restrict_scale || sweeps != mg.sweeps || flexible != mg.flexible ||
                smooth_weight != mg.smooth_weight) {
                CK(cudaStreamSynchronize(stream));
                destroy_graphs();
                mg.restrict_scale = restrict_scale;
                mg.sweeps = sweeps;
                mg.flexible = flexible;
                mg.smooth_weight = smooth_weight;
            }
        }
        ++sim_frame;
        event_next = 0;
        phase_events.clear();
        frame_solves.clear();
        set_pass_params(in);
        bool has_drain = false;
        for (uint32_t m = 0; m < num_manipulators; ++m) has_drain = has_drain || in.manipulators[m].kind == 0u;
        CK(cudaMemsetAsync(coupling, 0, SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE * 4, stream));
        CK(cudaMemsetAsync(stats, 0, SLOSH_NUM_STATS * 4, stream));
        CK(cudaMemsetAsync(mg.ctl + 4, 0, 4, stream));
        if (in.num_emits && !in.emits) throw StatusError{SLOSH_ERR_INVALID_ARG, "emits is NULL"};
        for (uint32_t e = 0; e < in.num_emits; ++e) emit(in.emits[e]);
        if (num_particles > 0 &&
            ((s.sort_interval > 0 && (sim_frame % uint64_t(s.sort_interval)) == 0) || (has_drain && (sim_frame % 8ull) == 0)))
            sort_particles();
        substeps = 0;
        density_frame = false;
        if (!in.paused && num_particles > 0) {
            const float frame_dt = clampf_h(in.delta_time, 1e-4f, clampf_h(s.max_frame_dt, 1.0f / 240.0f, 1.0f / 10.0f));
            const float gmag = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
            const float speed_estimate = std::max(last_max_speed, 1.0f) + gmag * frame_dt;
            substeps = clampi_h(int(std::ceil(speed_estimate * frame_dt / (std::max(s.cfl, 0.1f) * s.cell_size))),
                                std::max(s.min_substeps, 1), std::max(s.max_substeps, 1));
            dt = frame_dt / float(substeps);
            P.dt = dt;
            P.viscosity_alpha = s.kinematic_viscosity * dt / (s.cell_size * s.cell_size);
            P.pressure_to_pascal = s.density * s.cell_size / dt;
            const int interval = clampi_h(s.density_projection_interval, 1, 8);
            density_frame = s.two_sided_density_projection && P.density_relaxation > 0.0f && (sim_frame % uint64_t(interval)) == 0;
        }
        return substeps;
    }

    // ---- one substep (Step_RenderThread :564-713) ----
    void substep(int step) {
        const bool last = step == substeps - 1;
        // Warm start of the pressure solve: the previous solution rescaled by dt / dt_prev
        // (MarkCellsCS), or a zero initial guess (ZERO, and LEARNED before the network's guess).
        P.warm_start_scale = S.warm_start == uint32_t(SLOSH_WARM_START_PREVIOUS) ? (prev_dt > 0.0f ? P.dt / prev_dt : 1.0f) : 0.0f;
        prev_dt = P.dt;
        P.frame_seed = uint32_t(sim_frame * 16ull + uint64_t(step));
        const Dev d = dev();
        {
            PhaseScope ps(this, 1);
            count(launch_pool_update(d, stream));
            count(launch_clear_new_slots(d, shape, stream));
        }
        float* V[3] = {vel[vmap[0]], vel[vmap[1]], vel[vmap[2]]};
        {
            PhaseScope ps(this, 2);
            if (p2g_gather_enabled()) {
                count(launch_p2g_gather(d, P, gather, particles[pbuf], num_particles, stream));
            } else {
                // more than an eighth of the particles in placement order: the wider P2G tile
                count(launch_p2g(d, P, particles[pbuf], num_particles, placed_since_sort * 8u > num_particles, stream));
            }
        }
        int c = 0;
        {
            PhaseScope ps(this, 3);
            count(launch_mark_cells(d, P, shape, stream));
            count(launch_normalize_faces(d, P, V[0], shape, stream));
            if (P.viscosity_alpha > 0.0f && S.viscosity_iterations > 0) {
                CK(cudaMemcpyAsync(V[1], V[0], size_t(total_faces) * 4, cudaMemcpyDeviceToDevice, stream));
                int src = 1;
                for (int it = 0; it < S.viscosity_iterations; ++it) {
                    const int dst = src == 1 ? 2 : 1;
                    count(launch_viscosity(d, P, V[0], V[src], V[dst], shape, stream));
                    src = dst;
                }
                c = src;
            }
            count(launch_divergence(d, P, V[c], shape, stream));
        }
        {
            PhaseScope ps(this, 4);
            if (S.warm_start == uint32_t(SLOSH_WARM_START_LEARNED) && warm_net)
                count(slosh::unet::warm_start(warm_net, d, divergence, pressure, stream));
            if (S.pressure_solver == SLOSH_SOLVER_MGPCG) {
                const int coarse = clampi_h(S.mg_coarse_iterations, 1, 200);
                if (S.tolerance > 0.0f) mgpcg(pressure, divergence, 0, S.tolerance, S.max_iterations, coarse, 0);
                else mgpcg(pressure, divergence, S.pcg_iterations, 0.0f, 0, coarse, 0);
            } else {
                const float omega = clampf_h(S.sor_weight, 0.5f, 1.95f);
                for (int it = 0; it < S.pressure_iterations; ++it)
                    for (uint32_t colour = 0; colour < 2u; ++colour) count(launch_rbgs(d, pressure, divergence, colour, omega, shape, stream));
                last_iterations = S.pressure_iterations;
                last_converged = true;
            }
            if (last) count(launch_true_residual(d, mg, pressure, divergence, shape, stream));
        }
        {
            PhaseScope ps(this, 5);
            count(launch_project(d, P, V[c], shape, stream));
            count(launch_coupling(d, P, V[c], shape, stream));
            if (last) count(launch_residual(d, P, V[c], shape, stream));
        }
        const bool density = density_frame && last;
        if (density) {
            PhaseScope ps(this, 6);
            count(launch_density_rhs(d, P, shape, stream));
            if (S.pressure_solver == SLOSH_SOLVER_MGPCG) {
                mgpcg(density_q, density_rhs, 2, 0.0f, 0, clampi_h(S.mg_coarse_iterations, 1, 200), 1);
            } else {
                for (int it = 0; it < std::max(S.density_projection_iterations, 1); ++it)
                    for (uint32_t colour = 0; colour < 2u; ++colour)
                        count(launch_rbgs(d, density_q, density_rhs, colour, 1.7f, shape, stream));
            }
        }
        {
            PhaseScope ps(this, 7);
            // in place (the reference passes the field from buffer to buffer; the values are the same)
            for (int it = 0; it < S.extrapolation_layers; ++it) count(launch_extrapolate(d, V[c], uint32_t(it), shape, stream));
            if (density) count(launch_density_displacement(d, V[(c + 2) % 3], shape, stream));
        }
        {
            PhaseScope ps(this, 8);
            count(launch_g2p(d, P, particles[pbuf], num_particles, V[c], V[(c + 2) % 3], density, stream));
        }
        // The field of logical buffer c becomes logical buffer 0 for the next substep.
        const int nm[3] = {vmap[c], vmap[(c + 1) % 3], vmap[(c + 2) % 3]};
        disp_phys = vmap[(c + 2) % 3];
        vmap[0] = nm[0]; vmap[1] = nm[1]; vmap[2] = nm[2];
        CK(cudaGetLastError());
    }

    // ---- frame epilogue: AccumulateStatsCS + the readback decode ----
    void end_frame() {
        end_frame_enqueue();
        end_frame_finish();
    }
    void end_frame_enqueue();  // frame epilogue and result copies on the stream
    void end_frame_finish();   // waits for them and decodes
};

__global__ void k_accumulate_stats(uint32_t* stats, uint32_t* pc) {  // AccumulateStatsCS (Slosh.usf:264-270)
    pc[2] += stats[15];
    stats[14] = pc[0];
    stats[15] = pc[2];
}

void Ctx::end_frame_enqueue() {
    if (num_colliders > 0 && substeps > 0) count(launch_submerged(dev(), shape, stream));  // SloshProxy.cpp:715-718
    k_accumulate_stats<<<1, 1, 0, stream>>>(stats, particle_count);
    count(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_stats, stats, SLOSH_NUM_STATS * 4, cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(h_stats + SLOSH_NUM_STATS, particle_count, 16, cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(h_scalars, mg.scalars, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(h_ctl + 8, mg.ctl + 4, 4, cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(h_coupling, coupling, SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE * 4, cudaMemcpyDeviceToHost, stream));
    d2h_bytes += SLOSH_NUM_STATS * 4 + 16 + 8 * sizeof(double) + SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE * 4;
}

void Ctx::end_frame_finish() {
    CK(cudaStreamSynchronize(stream));
    if (substeps > 0) {
        float ms;
        std::memcpy(&ms, &h_stats[0], 4);
        last_max_speed = std::isfinite(ms) ? ms : 0.0f;
        const double num = h_scalars[6], den = h_scalars[7];
        last_true_rel = float(den > 0.0 ? std::sqrt(num / den) : 0.0);
        if (S.pressure_solver != SLOSH_SOLVER_MGPCG) last_rel = last_true_rel;
    }
    if (rel_pending) {
        last_rel = float(h_scalars[8] > 0.0 ? std::sqrt(h_scalars[9] / h_scalars[8]) : 0.0);
        last_iterations = int(h_ctl[0]);
        last_converged = !solve_tol_mode || double(last_rel) <= double(solve_tol);
        rel_pending = false;
    }
    for (const auto& r : frame_solves) launches += uint64_t(r.pre) + uint64_t(r.body) * uint64_t(h_ctl[4 * r.slot]);
    if (h_ctl[8] != 0u) last_converged = false;  // some substep's solve stopped at its iteration limit
    num_particles = std::min(num_particles, h_stats[SLOSH_NUM_STATS + 0]);
    pool_overflow_seen = h_stats[8] != 0u;
    if (timing) {
        std::fill(phase_ms, phase_ms + NUM_PHASES, 0.0f);
        for (auto& pe : phase_events) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) phase_ms[pe.first] += ms;
        }
    }
}

// Field and mesh sizes as BuildDensityField / FillFieldParameters derive them (SloshRenderer.cpp:118-170).
void Ctx::build_surface(const slosh_surface_params_t& q) {
    const float res = clampf_h(q.field_resolution, 0.5f, 3.0f);
    const float cell = S.cell_size;
    SurfaceDev& d = surf;
    d.voxel = cell / res;
    d.inv_voxel = 1.0f / d.voxel;
    d.dim = make_int3(int(std::ceil(float(grid.x) * res)), int(std::ceil(float(grid.y) * res)), int(std::ceil(float(grid.z) * res)));
    d.bdim = make_int3((d.dim.x + 7) / 8, (d.dim.y + 7) / 8, (d.dim.z + 7) / 8);
    d.support = clampf_h(q.surface_smoothing, 0.5f, 6.0f);
    d.max_footprint = 4.0f;
    d.radius_voxels = q.particle_radius_scale * res;
    d.splat_radius = cell * q.particle_radius_scale;
    d.iso = clampf_h(q.iso_level, 0.02f, 0.98f);
    d.max_vertices = q.max_vertices;
    d.max_indices = q.max_indices;
    const uint64_t nv = uint64_t(d.dim.x) * uint64_t(d.dim.y) * uint64_t(d.dim.z);
    const uint64_t nb = uint64_t(d.bdim.x) * uint64_t(d.bdim.y) * uint64_t(d.bdim.z);
    const uint64_t nc = uint64_t(std::max(d.dim.x - 1, 0)) * uint64_t(std::max(d.dim.y - 1, 0)) * uint64_t(std::max(d.dim.z - 1, 0));
    if (nv * 5u > 0xFFFFFFFFull) throw StatusError{SLOSH_ERR_INVALID_ARG, "surface field too large"};
    if (nv > surf_voxels_cap || nb > surf_bricks_cap || nc > surf_cells_cap || q.max_vertices > surf_vert_cap || q.max_indices > surf_idx_cap) {
        CK(cudaStreamSynchronize(stream));
        free_list(surface_allocs);
        surf_voxels_cap = nv; surf_bricks_cap = nb; surf_cells_cap = nc; surf_vert_cap = q.max_vertices; surf_idx_cap = q.max_indices;
        d.accum = salloc<int32_t>(nv * 5u);
        d.field = salloc<uint16_t>(nv);
        d.bricks = salloc<uint32_t>(nb);
        d.vflag = salloc<uint32_t>(nc);
        d.vbase = salloc<uint32_t>(nc);
        d.cell_vertex = salloc<uint32_t>(nc);
        d.qflag = salloc<uint32_t>(nc);
        d.qbase = salloc<uint32_t>(nc);
        d.scan_tmp = salloc<uint32_t>(exclusive_scan_tmp_size(uint32_t(nc)));
        d.positions = salloc<float>(3ull * q.max_vertices);
        d.normals = salloc<float>(3ull * q.max_vertices);
        d.tangents = salloc<float>(3ull * q.max_vertices);
        d.indices = salloc<uint32_t>(q.max_indices);
        d.counters = salloc<uint32_t>(2);
    }
    count(launch_surface(d, particles[pbuf], num_particles, q.build_mesh != 0u, stream));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_surf, d.counters, 8, cudaMemcpyDeviceToHost, stream));
    d2h_bytes += 8;
    CK(cudaStreamSynchronize(stream));
    slosh_surface_info_t& o = surf_info;
    o = slosh_surface_info_t{};
    o.field_dim[0] = d.dim.x; o.field_dim[1] = d.dim.y; o.field_dim[2] = d.dim.z;
    o.brick_dim[0] = d.bdim.x; o.brick_dim[1] = d.bdim.y; o.brick_dim[2] = d.bdim.z;
    o.voxel_size = d.voxel;
    if (q.build_mesh) {
        o.vertices_requested = h_surf[0];
        o.num_vertices = std::min(h_surf[0], q.max_vertices);
        o.indices_requested = h_surf[1];
        // Whole quads only: a quad is written only when all six of its indices fit (SurfaceNetsFacesCS); the
        // reference's argument pass rounds to triangles and so can draw up to three indices never written.
        const uint32_t ni = std::min(h_surf[1], q.max_indices);
        o.num_indices = ni - ni % 6u;
    }
}

void decode_results(const Ctx& c, slosh_results_t* out) {
    std::memset(out, 0, sizeof(*out));
    const uint32_t* st = c.h_stats;
    const float inv_sub = 1.0f / float(std::max(c.substeps, 1));
    const float inv_scale = 1.0f / 1024.0f;
    out->num_colliders = c.num_colliders;
    for (uint32_t k = 0; k < c.num_colliders; ++k) {
        const int32_t* cc = c.h_coupling + k * SLOSH_COUPLING_STRIDE;
        slosh_collider_feedback_t& o = out->colliders[k];
        for (int a = 0; a < 3; ++a) {
            o.pressure_force[a] = float(cc[a]) * (inv_scale * inv_sub);
            o.pressure_torque[a] = float(cc[3 + a]) * (inv_scale * inv_sub);
            o.submerged_centroid_offset[a] = cc[7] > 0 ? float(cc[12 + a]) * (inv_scale / float(cc[7])) : 0.0f;
            o.mean_fluid_velocity[a] = cc[6] > 0 ? float(cc[8 + a]) * (inv_scale / float(cc[6])) : 0.0f;
        }
        o.wetted_faces = int32_t(std::lround(double(cc[6]) * inv_sub));
        o.submerged_cells = cc[7];
        o.solid_cells = cc[11];
    }
    float ms;
    std::memcpy(&ms, &st[0], 4);
    out->max_particle_speed = std::isfinite(ms) ? ms : 0.0f;
    out->fluid_cells = int32_t(std::lround(double(st[1]) * inv_sub));
    std::memcpy(&out->max_divergence, &st[2], 4);
    out->mean_divergence = st[4] > 0 ? float(double(st[3]) * 1e-3 / double(st[4])) : 0.0f;
    out->mean_interior_density = st[6] > 0 ? float(1.0 + double(int32_t(st[5])) * 1e-4 / double(st[6])) : 0.0f;
    out->interior_cells = int32_t(st[6]);
    out->active_brick_fraction = c.num_bricks > 0 ? float(st[7]) / float(c.num_bricks) : -1.0f;
    out->pool_usage = c.num_pool_bricks > 1 ? float(st[7]) / float(c.num_pool_bricks - 1) : -1.0f;
    out->pool_overflow_bricks = int32_t(st[8]);
    out->clamped_particles = int32_t(st[9]);
    out->clamped_in_solid = int32_t(st[13]);
    for (int a = 0; a < 3; ++a) out->clamped_centroid[a] = st[9] > 0 ? float(st[10 + a]) * (0.01f / float(st[9])) : 0.0f;
    out->grid_memory_mb = float(double(c.grid_bytes) / (1024.0 * 1024.0));
    out->particle_memory_mb = float(double(c.particle_bytes) / (1024.0 * 1024.0));
    out->allocated_particle_capacity = int32_t(c.capacity);
    out->live_particles = int32_t(st[14]);
    out->drained_particles = int64_t(st[15]);
    out->substeps = c.substeps;
    out->sim_frame = c.sim_frame;
    out->last_solve_iterations = c.last_iterations;
    out->last_solve_rel_residual = c.last_rel;
    out->last_solve_true_rel_residual = c.last_true_rel;
    std::memcpy(out->raw_stats, st, sizeof(out->raw_stats));
}

// Buffer export/import map.
struct BufView {
    void* ptr = nullptr;
    size_t bytes = 0;
};
BufView buffer_view(Ctx& c, int id) {
    BufView v;
    const size_t tf = c.total_faces, pc = c.pool_cells;
    switch (id) {
        case SLOSH_BUF_PARTICLES: v = {c.particles[c.pbuf], size_t(c.num_particles) * sizeof(slosh_particle_t)}; break;
        case SLOSH_BUF_VEL: v = {c.vel[c.vmap[0]], tf * 4}; break;
        case SLOSH_BUF_VEL_OLD: v = {c.vel_old, tf * 4}; break;
        case SLOSH_BUF_FACE_FLAGS: v = {c.face_flags, tf * 4}; break;
        case SLOSH_BUF_FACE_WEIGHT: v = {c.face_weight, tf * 4}; break;
        case SLOSH_BUF_CELL_TYPE: v = {c.cell_type, pc * 4}; break;
        case SLOSH_BUF_CELL_COUNT: v = {c.cell_count, pc * 4}; break;
        case SLOSH_BUF_PRESSURE: v = {c.pressure, pc * 4}; break;
        case SLOSH_BUF_DIVERGENCE: v = {c.divergence, pc * 4}; break;
        case SLOSH_BUF_CELL_DIAG: v = {c.cell_diag, pc * 4}; break;
        case SLOSH_BUF_DENSITY_Q: v = {c.density_q, pc * 4}; break;
        case SLOSH_BUF_DENSITY_RHS: v = {c.density_rhs, pc * 4}; break;
        case SLOSH_BUF_BRICK_TABLE: v = {c.brick_table, size_t(c.num_bricks) * 4}; break;
        case SLOSH_BUF_SLOT_BRICK: v = {c.slot_brick, size_t(c.num_pool_bricks) * 4}; break;
        case SLOSH_BUF_FREE_SLOTS: v = {c.free_slots, size_t(c.num_pool_bricks) * 4}; break;
        case SLOSH_BUF_ACTIVE_BRICKS: v = {c.active_bricks, size_t(c.num_bricks + 1) * 4}; break;
        case SLOSH_BUF_NEW_SLOTS: v = {c.new_slots, size_t(c.num_pool_bricks + 1) * 4}; break;
        case SLOSH_BUF_BRICK_TOUCH: v = {c.brick_touch, size_t(c.num_bricks) * 4}; break;
        case SLOSH_BUF_STATS: v = {c.stats, SLOSH_NUM_STATS * 4}; break;
        case SLOSH_BUF_SORT_COUNTS: v = {c.sortb.counts, size_t(c.num_sort_keys) * 4}; break;
        case SLOSH_BUF_SORT_OFFSETS: v = {c.sortb.offsets, size_t(c.num_sort_keys) * 4}; break;
        case SLOSH_BUF_SORT_PERM: v = {c.sortb.perm, size_t(c.num_particles) * 4}; break;
        case SLOSH_BUF_PARTICLE_COUNT: v = {c.particle_count, 16}; break;
        case SLOSH_BUF_ACCUM: v = {c.accum, 2 * tf * 4}; break;
        case SLOSH_BUF_VEL_EXTRAP: v = {c.vel[c.disp_phys], tf * 4}; break;
        case SLOSH_BUF_COUPLING: v = {c.coupling, size_t(SLOSH_MAX_COLLIDERS) * SLOSH_COUPLING_STRIDE * 4}; break;
        case SLOSH_BUF_SURFACE_FIELD:
            v = {c.surf.field, c.surf.field ? size_t(c.surf_info.field_dim[0]) * c.surf_info.field_dim[1] * c.surf_info.field_dim[2] * 2 : 0};
            break;
        case SLOSH_BUF_SURFACE_BRICKS:
            v = {c.surf.bricks, c.surf.bricks ? size_t(c.surf_info.brick_dim[0]) * c.surf_info.brick_dim[1] * c.surf_info.brick_dim[2] * 4 : 0};
            break;
        case SLOSH_BUF_SURFACE_POSITIONS: v = {c.surf.positions, size_t(c.surf_info.num_vertices) * 12}; break;
        case SLOSH_BUF_SURFACE_NORMALS: v = {c.surf.normals, size_t(c.surf_info.num_vertices) * 12}; break;
        case SLOSH_BUF_SURFACE_TANGENTS: v = {c.surf.tangents, size_t(c.surf_info.num_vertices) * 12}; break;
        case SLOSH_BUF_SURFACE_INDICES: v = {c.surf.indices, size_t(c.surf_info.num_indices) * 4}; break;
        default: break;
    }
    return v;
}

template <class Fn>
slosh_status guarded(Fn fn) {
    try {
        return fn();
    } catch (const CudaError& e) {
        g_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return SLOSH_ERR_CUDA;
    } catch (const StatusError& e) {
        g_error = e.what;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return SLOSH_ERR_OUT_OF_MEMORY;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return SLOSH_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        g_error = e.what();
        return SLOSH_ERR_CUDA;
    } catch (...) {
        g_error = "unknown error";
        return SLOSH_ERR_CUDA;
    }
}

Ctx* as_ctx(void* p) {
    if (!p) throw StatusError{SLOSH_ERR_INVALID_ARG, "context is NULL"};
    Ctx* c = static_cast<Ctx*>(p);
    CK(cudaSetDevice(c->device));
    return c;
}

}  // namespace
// Error text for entry points defined in other files of the library.
void set_last_error(const char* message) { g_error = message ? message : ""; }

}  // namespace slosh

using namespace slosh;

namespace slosh {
namespace unet {
// The simulation state the warm-start network reads and writes (unet.cu).
void* sim_ctx_dev(void* ctx, Dev* out, float** divergence, float** pressure, cudaStream_t* stream) {
    if (!ctx) return nullptr;
    Ctx* c = static_cast<Ctx*>(ctx);
    if (!c->allocated) return nullptr;
    *out = c->dev();
    *divergence = c->divergence;
    *pressure = c->pressure;
    *stream = c->stream;
    return ctx;
}
}  // namespace unet
}  // namespace slosh

extern "C" {

SLOSH_API uint32_t slosh_abi_version(void) { return SLOSH_ABI_VERSION; }
SLOSH_API void slosh_settings_default(slosh_settings_t* out) {
    if (out) *out = defaults();
}
SLOSH_API const char* slosh_last_error_string(void) { return g_error.c_str(); }

SLOSH_API slosh_status slosh_create(const slosh_settings_t* settings, int32_t device, void** out_ctx) {
    return guarded([&]() -> slosh_status {
        if (!settings || !out_ctx) throw StatusError{SLOSH_ERR_INVALID_ARG, "settings or out_ctx is NULL"};
        *out_ctx = nullptr;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            throw StatusError{SLOSH_ERR_NO_DEVICE, "no CUDA device: the Slosh substep runs only on the GPU"};
        }
        int dev = device;
        if (dev < 0) CK(cudaGetDevice(&dev));
        if (dev >= count) throw StatusError{SLOSH_ERR_INVALID_ARG, "device index out of range"};
        CK(cudaSetDevice(dev));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, dev));
        if (prop.major < 10) throw StatusError{SLOSH_ERR_NO_DEVICE, "this library is built for sm_100a (B200)"};
        Ctx* c = new Ctx();
        c->device = dev;
        c->num_sms = prop.multiProcessorCount;
        try {
            CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking));
            CK(cudaMallocHost(&c->h_ctl, 16 * sizeof(uint32_t)));
            CK(cudaMallocHost(&c->h_surf, 2 * sizeof(uint32_t)));
            std::memset(c->h_ctl, 0, 16 * sizeof(uint32_t));
            const char* ng = std::getenv("SLOSH_NO_GRAPHS");
            c->use_graphs = !(ng && ng[0] == '1');
            c->stream = c->own_stream;
            CK(cudaMallocHost(&c->h_colliders, sizeof(slosh_collider_t) * SLOSH_MAX_COLLIDERS));
            CK(cudaMallocHost(&c->h_manipulators, sizeof(slosh_manipulator_t) * SLOSH_MAX_MANIPULATORS));
            CK(cudaMallocHost(&c->h_stats, 4 * (SLOSH_NUM_STATS + 4)));
            CK(cudaMallocHost(&c->h_scalars, 16 * sizeof(double)));
            CK(cudaMallocHost(&c->h_coupling, 4 * SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE));
            std::memset(c->h_stats, 0, 4 * (SLOSH_NUM_STATS + 4));
            std::memset(c->h_scalars, 0, 16 * sizeof(double));
            std::memset(c->h_coupling, 0, 4 * SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE);
            c->allocate(clamp_settings(*settings));
            CK(cudaDeviceSynchronize());
        } catch (...) {
            slosh_destroy(c);
            throw;
        }
        *out_ctx = c;
        return SLOSH_OK;
    });
}

SLOSH_API void slosh_destroy(void* ctx) {
    if (!ctx) return;
    Ctx* c = static_cast<Ctx*>(ctx);
    cudaSetDevice(c->device);
    c->release();
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    if (c->h_colliders) cudaFreeHost(c->h_colliders);
    if (c->h_manipulators) cudaFreeHost(c->h_manipulators);
    if (c->h_stats) cudaFreeHost(c->h_stats);
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    if (c->h_coupling) cudaFreeHost(c->h_coupling);
    if (c->h_surf) cudaFreeHost(c->h_surf);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->body_stream) cudaStreamDestroy(c->body_stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

SLOSH_API slosh_status slosh_set_stream(void* ctx, void* cuda_stream) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        CK(cudaStreamSynchronize(c->stream));
        c->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c->own_stream;
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_synchronize(void* ctx) {
    return guarded([&]() -> slosh_status {
        CK(cudaStreamSynchronize(as_ctx(ctx)->stream));
        return SLOSH_OK;
    });
}

static slosh_status frame_status(const Ctx* c) {
    if (c->pool_overflow_seen) return SLOSH_WARN_POOL_OVERFLOW;
    if (!c->last_converged) return SLOSH_ERR_NOT_CONVERGED;
    return SLOSH_OK;
}

SLOSH_API slosh_status slosh_begin_frame(void* ctx, const slosh_frame_input_t* input, int32_t* out_substeps, float* out_dt) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!input) throw StatusError{SLOSH_ERR_INVALID_ARG, "input is NULL"};
        const int n = c->begin_frame(*input);
        if (out_substeps) *out_substeps = n;
        if (out_dt) *out_dt = c->dt;
        CK(cudaGetLastError());
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_substep(void* ctx, int32_t step_index) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (step_index < 0 || step_index >= c->substeps) throw StatusError{SLOSH_ERR_INVALID_ARG, "substep index out of range"};
        c->substep(step_index);
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_end_frame(void* ctx) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        c->end_frame();
        return frame_status(c);
    });
}
SLOSH_API slosh_status slosh_step_frame(void* ctx, const slosh_frame_input_t* input) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!input) throw StatusError{SLOSH_ERR_INVALID_ARG, "input is NULL"};
        const int n = c->begin_frame(*input);
        for (int s = 0; s < n; ++s) c->substep(s);
        c->end_frame();
        return frame_status(c);
    });
}

// Autotuner of the brick-pass launch shape: steps `frames` frames of `input` per candidate CTAs-per-SM
// count, times them on the device (events on the context's stream), and leaves the context on the
// fastest per substep. The simulation advances by all these frames; results do not depend on the shape.
SLOSH_API slosh_status slosh_autotune(void* ctx, const slosh_frame_input_t* input, uint32_t frames, slosh_autotune_result_t* out) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!input) throw StatusError{SLOSH_ERR_INVALID_ARG, "input is NULL"};
        const uint32_t cand[] = {2u, 4u, 8u, 12u, 16u};
        const uint32_t nc = uint32_t(sizeof(cand) / sizeof(cand[0]));
        slosh_autotune_result_t r;
        std::memset(&r, 0, sizeof(r));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 0.0f;
        slosh_status worst = SLOSH_OK;
        try {
            for (uint32_t k = 0; k < nc; ++k) {
                c->set_ctas_per_sm(cand[k]);
                // one untimed frame captures the solve graphs of this shape
                int n = c->begin_frame(*input);
                for (int sidx = 0; sidx < n; ++sidx) c->substep(sidx);
                c->end_frame();
                CK(cudaEventRecord(e0, c->stream));
                int substeps = 0;
                for (uint32_t f = 0; f < std::max(frames, 1u); ++f) {
                    n = c->begin_frame(*input);
                    for (int sidx = 0; sidx < n; ++sidx) c->substep(sidx);
                    c->end_frame();
                    substeps += n;
                    const slosh_status st = frame_status(c);
                    if (st != SLOSH_OK && worst == SLOSH_OK) worst = st;
                }
                CK(cudaEventRecord(e1, c->stream));
                CK(cudaEventSynchronize(e1));
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                const float per = substeps > 0 ? ms / float(substeps) : ms;
                r.ctas_per_sm[k] = cand[k];
                r.ms_per_substep[k] = per;
                if (k == 0 || per < best) {
                    best = per;
                    r.best_ctas_per_sm = cand[k];
                }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        r.num_candidates = nc;
        c->set_ctas_per_sm(r.best_ctas_per_sm);
        r.brick_ctas = uint32_t(c->shape.brick_ctas);
        if (out) *out = r;
        return worst == SLOSH_OK ? SLOSH_OK : worst;
    });
}
SLOSH_API slosh_status slosh_set_mg_ctas_per_sm(void* ctx, uint32_t ctas_per_sm) {
    return guarded([&]() -> slosh_status {
        if (ctas_per_sm == 0u) throw StatusError{SLOSH_ERR_INVALID_ARG, "ctas_per_sm must be positive"};
        as_ctx(ctx)->set_mg_ctas_per_sm(ctas_per_sm);
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_set_ctas_per_sm(void* ctx, uint32_t ctas_per_sm) {
    return guarded([&]() -> slosh_status {
        if (ctas_per_sm == 0u) throw StatusError{SLOSH_ERR_INVALID_ARG, "ctas_per_sm must be positive"};
        as_ctx(ctx)->set_ctas_per_sm(ctas_per_sm);
        return SLOSH_OK;
    });
}

// Several independent tanks one frame each (batched tanks). Every context's frame is enqueued on its own
// stream before any is waited for, so small tanks overlap on the device; then each frame is finished and
// decoded in order. statuses (optional) receives each context's status; the return value is the first
// status that is not SLOSH_OK (a warning or an error), else SLOSH_OK.
SLOSH_API slosh_status slosh_step_frames(void* const* ctxs, const slosh_frame_input_t* inputs, uint32_t count,
                                         slosh_status* statuses) {
    return guarded([&]() -> slosh_status {
        if (count && (!ctxs || !inputs)) throw StatusError{SLOSH_ERR_INVALID_ARG, "ctxs or inputs is NULL"};
        for (uint32_t i = 0; i < count; ++i) {
            Ctx* c = as_ctx(ctxs[i]);
            const int n = c->begin_frame(inputs[i]);
            for (int k = 0; k < n; ++k) c->substep(k);
            c->end_frame_enqueue();
        }
        slosh_status first = SLOSH_OK;
        for (uint32_t i = 0; i < count; ++i) {
            Ctx* c = as_ctx(ctxs[i]);
            c->end_frame_finish();
            const slosh_status st = frame_status(c);
            if (statuses) statuses[i] = st;
            if (first == SLOSH_OK) first = st;
        }
        return first;
    });
}

SLOSH_API slosh_status slosh_sort_particles(void* ctx) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        c->sort_particles();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->stream));
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_emit(void* ctx, const slosh_emit_request_t* request) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!request) throw StatusError{SLOSH_ERR_INVALID_ARG, "request is NULL"};
        c->emit(*request);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->stream));
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_set_emit_seed(void* ctx, uint32_t seed) {
    return guarded([&]() -> slosh_status {
        as_ctx(ctx)->emit_seed = seed;
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_upload_particles(void* ctx, const slosh_particle_t* particles, uint32_t count) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!particles && count) throw StatusError{SLOSH_ERR_INVALID_ARG, "particles is NULL"};
        if (count > c->capacity) throw StatusError{SLOSH_ERR_CAPACITY, "more particles than particle_capacity"};
        if (count)
            CK(cudaMemcpyAsync(c->particles[c->pbuf], particles, sizeof(slosh_particle_t) * count, cudaMemcpyHostToDevice, c->stream));
        c->num_particles = count;
        c->placed_since_sort = count;
        uint32_t pcv[2] = {count, 0u};
        CK(cudaMemcpyAsync(c->particle_count, pcv, 8, cudaMemcpyHostToDevice, c->stream));
        c->h2d_bytes += sizeof(slosh_particle_t) * count + 8;
        c->count(launch_touch_particles(c->dev(), c->particles[c->pbuf], count, c->stream));
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->stream));
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_download_particles(void* ctx, slosh_particle_t* out, uint32_t capacity, uint32_t* out_count) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (out_count) *out_count = c->num_particles;
        if (!out) return SLOSH_OK;
        const uint32_t n = std::min(capacity, c->num_particles);
        if (n) CK(cudaMemcpyAsync(out, c->particles[c->pbuf], sizeof(slosh_particle_t) * n, cudaMemcpyDeviceToHost, c->stream));
        c->d2h_bytes += sizeof(slosh_particle_t) * n;
        CK(cudaStreamSynchronize(c->stream));
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_particle_device_ptr(void* ctx, void** out_ptr, uint32_t* out_count) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (out_ptr) *out_ptr = c->particles[c->pbuf];
        if (out_count) *out_count = c->num_particles;
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_get_results(void* ctx, slosh_results_t* out) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!out) throw StatusError{SLOSH_ERR_INVALID_ARG, "out is NULL"};
        decode_results(*c, out);
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_get_layout(void* ctx, slosh_layout_t* out) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!out) throw StatusError{SLOSH_ERR_INVALID_ARG, "out is NULL"};
        std::memset(out, 0, sizeof(*out));
        out->grid_dim[0] = c->grid.x; out->grid_dim[1] = c->grid.y; out->grid_dim[2] = c->grid.z;
        out->brick_dim[0] = c->brick_dim.x; out->brick_dim[1] = c->brick_dim.y; out->brick_dim[2] = c->brick_dim.z;
        out->num_bricks = c->num_bricks;
        out->num_pool_bricks = c->num_pool_bricks;
        out->pool_cells = c->pool_cells;
        out->total_faces = c->total_faces;
        out->sort_brick_dim[0] = c->sort_dim.x; out->sort_brick_dim[1] = c->sort_dim.y; out->sort_brick_dim[2] = c->sort_dim.z;
        out->num_sort_keys = c->num_sort_keys;
        out->num_mg_levels = uint32_t(c->num_levels);
        for (int l = 0; l < c->num_levels; ++l) {
            out->mg_dim[l][0] = c->level_dim[l].x; out->mg_dim[l][1] = c->level_dim[l].y; out->mg_dim[l][2] = c->level_dim[l].z;
        }
        out->num_particles = c->num_particles;
        out->particle_capacity = c->capacity;
        out->current_vel = uint32_t(c->vmap[0]);
        return SLOSH_OK;
    });
}

SLOSH_API void slosh_surface_params_default(slosh_surface_params_t* out) {
    if (!out) return;
    // FSloshRenderSettings defaults (SloshRenderer.h:34-46); capacities for a 256^3 domain's surface.
    out->field_resolution = 1.0f;
    out->surface_smoothing = 2.0f;
    out->particle_radius_scale = 0.6f;
    out->iso_level = 0.5f;
    out->build_mesh = 1u;
    out->max_vertices = 1u << 22;
    out->max_indices = 1u << 24;
}

SLOSH_API slosh_status slosh_set_warm_start_network(void* ctx, void* net) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        c->warm_net = static_cast<slosh::unet::Net*>(net);
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_build_surface(void* ctx, const slosh_surface_params_t* params, slosh_surface_info_t* out) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!params) throw StatusError{SLOSH_ERR_INVALID_ARG, "params is NULL"};
        c->build_surface(*params);
        if (out) *out = c->surf_info;
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_surface_device_ptrs(void* ctx, void** field_f16, void** positions, void** normals, void** tangents,
                                                 void** indices) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (field_f16) *field_f16 = c->surf.field;
        if (positions) *positions = c->surf.positions;
        if (normals) *normals = c->surf.normals;
        if (tangents) *tangents = c->surf.tangents;
        if (indices) *indices = c->surf.indices;
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_buffer_bytes(void* ctx, int32_t buffer_id, size_t* out_bytes) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!out_bytes || buffer_id < 0 || buffer_id >= SLOSH_BUF_COUNT_) throw StatusError{SLOSH_ERR_INVALID_ARG, "bad buffer id"};
        *out_bytes = buffer_view(*c, buffer_id).bytes;
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_read_buffer(void* ctx, int32_t buffer_id, void* host_dst, size_t bytes) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (buffer_id < 0 || buffer_id >= SLOSH_BUF_COUNT_) throw StatusError{SLOSH_ERR_INVALID_ARG, "bad buffer id"};
        const BufView v = buffer_view(*c, buffer_id);
        if (bytes < v.bytes || (!host_dst && v.bytes)) throw StatusError{SLOSH_ERR_INVALID_ARG, "destination too small"};
        CK(cudaStreamSynchronize(c->stream));
        if (v.bytes) CK(cudaMemcpy(host_dst, v.ptr, v.bytes, cudaMemcpyDeviceToHost));
        c->d2h_bytes += v.bytes;
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_write_buffer(void* ctx, int32_t buffer_id, const void* host_src, size_t bytes) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (buffer_id < 0 || buffer_id >= SLOSH_BUF_COUNT_) throw StatusError{SLOSH_ERR_INVALID_ARG, "bad buffer id"};
        CK(cudaStreamSynchronize(c->stream));
        if (buffer_id == SLOSH_BUF_PARTICLES) {
            const size_t n = bytes / sizeof(slosh_particle_t);
            if (n > c->capacity) throw StatusError{SLOSH_ERR_CAPACITY, "more particles than particle_capacity"};
            if (n) CK(cudaMemcpy(c->particles[c->pbuf], host_src, n * sizeof(slosh_particle_t), cudaMemcpyHostToDevice));
            c->num_particles = uint32_t(n);
            c->placed_since_sort = n;
            return SLOSH_OK;
        }
        const BufView v = buffer_view(*c, buffer_id);
        if (bytes != v.bytes || (!host_src && v.bytes)) throw StatusError{SLOSH_ERR_INVALID_ARG, "size mismatch"};
        if (v.bytes) CK(cudaMemcpy(v.ptr, host_src, v.bytes, cudaMemcpyHostToDevice));
        return SLOSH_OK;
    });
}

SLOSH_API slosh_status slosh_enable_phase_timing(void* ctx, int32_t enable) {
    return guarded([&]() -> slosh_status {
        as_ctx(ctx)->timing = enable != 0;
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_get_phase_ms(void* ctx, float* out_ms, int32_t n) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (!out_ms) throw StatusError{SLOSH_ERR_INVALID_ARG, "out_ms is NULL"};
        for (int i = 0; i < std::min<int>(n, NUM_PHASES); ++i) out_ms[i] = c->phase_ms[i];
        return SLOSH_OK;
    });
}
SLOSH_API uint64_t slosh_launch_count(void* ctx) { return ctx ? static_cast<Ctx*>(ctx)->launches : 0; }
SLOSH_API slosh_status slosh_transfer_bytes(void* ctx, uint64_t* out_h2d, uint64_t* out_d2h) {
    return guarded([&]() -> slosh_status {
        Ctx* c = as_ctx(ctx);
        if (out_h2d) *out_h2d = c->h2d_bytes;
        if (out_d2h) *out_d2h = c->d2h_bytes;
        return SLOSH_OK;
    });
}

}  // extern "C"
