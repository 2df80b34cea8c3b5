// TEST INFRASTRUCTURE -- C entry points of the CPU oracle (slosh_oracle.hpp) for the Python tests and
// the cpu_baseline leg of bench.py. The calls mirror the product's C ABI (include/slosh_cuda.h) so a
// parity test drives both sides the same way.
#include <cstdio>
#include <cstring>
#include <memory>

#include "slosh_oracle.hpp"

#define ORACLE_API extern "C" __attribute__((visibility("default")))

using namespace slosh_oracle;

namespace {

struct Handle {
    int fp64 = 0;
    std::unique_ptr<Sim<float>> f;
    std::unique_ptr<Sim<double>> d;
};

template <class Fn>
int dispatch(void* h, Fn fn) {
    if (!h) return SLOSH_ERR_INVALID_ARG;
    Handle* H = static_cast<Handle*>(h);
    if (H->fp64) return fn(*H->d);
    return fn(*H->f);
}

// Decode of the stats/coupling buffers, PollReadbacks_RenderThread (SloshProxy.cpp:751-795).
template <class R>
void decode_results(const Sim<R>& s, slosh_results_t* out) {
    std::memset(out, 0, sizeof(*out));
    const uint32_t* st = s.stats;
    const float inv_sub = 1.0f / float(std::max(s.substeps, 1));
    const float inv_scale = 1.0f / 1024.0f;
    out->num_colliders = s.P.num_colliders;
    for (uint32_t k = 0; k < s.P.num_colliders; ++k) {
        const int32_t* c = s.coupling + k * SLOSH_COUPLING_STRIDE;
        slosh_collider_feedback_t& o = out->colliders[k];
        for (int a = 0; a < 3; ++a) {
            o.pressure_force[a] = float(c[a]) * (inv_scale * inv_sub);
            o.pressure_torque[a] = float(c[3 + a]) * (inv_scale * inv_sub);
            o.submerged_centroid_offset[a] = c[7] > 0 ? float(c[12 + a]) * (inv_scale / float(c[7])) : 0.0f;
            o.mean_fluid_velocity[a] = c[6] > 0 ? float(c[8 + a]) * (inv_scale / float(c[6])) : 0.0f;
        }
        o.wetted_faces = int32_t(std::lround(double(c[6]) * inv_sub));
        o.submerged_cells = c[7];
        o.solid_cells = c[11];
    }
    const float ms = bits_f32(st[0]);
    out->max_particle_speed = std::isfinite(ms) ? ms : 0.0f;
    out->fluid_cells = int32_t(std::lround(double(st[1]) * inv_sub));
    out->max_divergence = bits_f32(st[2]);
    out->mean_divergence = st[4] > 0 ? float(double(st[3]) * 1e-3 / double(st[4])) : 0.0f;
    out->mean_interior_density = st[6] > 0 ? float(1.0 + double(int32_t(st[5])) * 1e-4 / double(st[6])) : 0.0f;
    out->interior_cells = int32_t(st[6]);
    out->active_brick_fraction = s.L.num_bricks > 0 ? float(st[7]) / float(s.L.num_bricks) : -1.0f;
    out->pool_usage = s.L.num_pool_bricks > 1 ? float(st[7]) / float(s.L.num_pool_bricks - 1) : -1.0f;
    out->pool_overflow_bricks = int32_t(st[8]);
    out->clamped_particles = int32_t(st[9]);
    out->clamped_in_solid = int32_t(st[13]);
    for (int a = 0; a < 3; ++a) out->clamped_centroid[a] = st[9] > 0 ? float(st[10 + a]) * (0.01f / float(st[9])) : 0.0f;
    out->allocated_particle_capacity = int32_t(s.particles.size());
    out->live_particles = int32_t(st[14]);
    out->drained_particles = int64_t(st[15]);
    out->substeps = s.substeps;
    out->sim_frame = s.sim_frame;
    out->last_solve_iterations = s.last_solve_iterations;
    out->last_solve_rel_residual = s.last_solve_rel_residual;
    out->last_solve_true_rel_residual = s.last_solve_true_rel_residual;
    std::memcpy(out->raw_stats, st, sizeof(out->raw_stats));
}

template <class R>
void fill_layout(const Sim<R>& s, slosh_layout_t* out) {
    std::memset(out, 0, sizeof(*out));
    const Layout& L = s.L;
    for (int a = 0; a < 3; ++a) {
        out->grid_dim[a] = L.grid[a];
        out->brick_dim[a] = L.brick_dim[a];
        out->sort_brick_dim[a] = L.sort_brick_dim[a];
    }
    out->num_bricks = L.num_bricks;
    out->num_pool_bricks = L.num_pool_bricks;
    out->pool_cells = L.pool_cells;
    out->total_faces = L.total_faces;
    out->num_sort_keys = L.num_sort_keys;
    out->num_mg_levels = uint32_t(L.num_levels);
    for (int l = 0; l < L.num_levels; ++l)
        for (int a = 0; a < 3; ++a) out->mg_dim[l][a] = L.level_dim[l][a];
    out->num_particles = s.num_particles;
    out->particle_capacity = uint32_t(s.particles.size());
    out->current_vel = uint32_t(s.cur);
}

// Raw view of one buffer: pointer, element count, element size; float buffers report is_real.
template <class R>
struct View {
    void* ptr = nullptr;
    size_t count = 0;
    size_t elem = 0;
    bool is_real = false;
};
template <class R>
View<R> view(Sim<R>& s, int id) {
    View<R> v;
    auto u32 = [&](std::vector<uint32_t>& b, size_t n) { v.ptr = b.data(); v.count = n; v.elem = 4; };
    auto i32 = [&](std::vector<int32_t>& b, size_t n) { v.ptr = b.data(); v.count = n; v.elem = 4; };
    auto real = [&](std::vector<R>& b) { v.ptr = b.data(); v.count = b.size(); v.elem = sizeof(R); v.is_real = true; };
    switch (id) {
        case SLOSH_BUF_PARTICLES: v.ptr = s.particles.data(); v.count = s.num_particles; v.elem = sizeof(slosh_particle_t); break;
        case SLOSH_BUF_VEL: real(s.vel[s.cur]); break;
        case SLOSH_BUF_VEL_OLD: real(s.vel_old); break;
        case SLOSH_BUF_FACE_FLAGS: u32(s.face_flags, s.face_flags.size()); break;
        case SLOSH_BUF_FACE_WEIGHT: real(s.face_weight); break;
        case SLOSH_BUF_CELL_TYPE: u32(s.cell_type, s.cell_type.size()); break;
        case SLOSH_BUF_CELL_COUNT: i32(s.cell_count, s.cell_count.size()); break;
        case SLOSH_BUF_PRESSURE: real(s.pressure); break;
        case SLOSH_BUF_DIVERGENCE: real(s.divergence); break;
        case SLOSH_BUF_CELL_DIAG: real(s.cell_diag); break;
        case SLOSH_BUF_DENSITY_Q: real(s.density_q); break;
        case SLOSH_BUF_DENSITY_RHS: real(s.density_rhs); break;
        case SLOSH_BUF_BRICK_TABLE: u32(s.brick_table, s.brick_table.size()); break;
        case SLOSH_BUF_SLOT_BRICK: u32(s.slot_brick, s.slot_brick.size()); break;
        case SLOSH_BUF_FREE_SLOTS: u32(s.free_slots, s.free_slots.size()); break;
        case SLOSH_BUF_ACTIVE_BRICKS: u32(s.active_bricks, s.active_bricks.size()); break;
        case SLOSH_BUF_NEW_SLOTS: u32(s.new_slots, s.new_slots.size()); break;
        case SLOSH_BUF_BRICK_TOUCH: u32(s.brick_touch, s.brick_touch.size()); break;
        case SLOSH_BUF_STATS: v.ptr = s.stats; v.count = NUM_STATS; v.elem = 4; break;
        case SLOSH_BUF_SORT_COUNTS: u32(s.sort_counts, s.sort_counts.size()); break;
        case SLOSH_BUF_SORT_OFFSETS: u32(s.sort_offsets, s.sort_offsets.size()); break;
        case SLOSH_BUF_SORT_PERM: u32(s.sort_perm, s.num_particles); break;
        case SLOSH_BUF_PARTICLE_COUNT: v.ptr = s.particle_count; v.count = 4; v.elem = 4; break;
        case SLOSH_BUF_ACCUM: i32(s.accum, s.accum.size()); break;
        case SLOSH_BUF_VEL_EXTRAP: real(s.vel[s.last_disp_index]); break;
        case SLOSH_BUF_COUPLING: v.ptr = s.coupling; v.count = SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE; v.elem = 4; break;
        case SLOSH_BUF_SURFACE_FIELD: v.ptr = s.surface.field.data(); v.count = s.surface.field.size(); v.elem = 2; break;
        case SLOSH_BUF_SURFACE_BRICKS: u32(s.surface.bricks, s.surface.bricks.size()); break;
        case SLOSH_BUF_SURFACE_POSITIONS: v.ptr = s.surface.positions.data(); v.count = 3u * s.surface.num_vertices; v.elem = 4; break;
        case SLOSH_BUF_SURFACE_NORMALS: v.ptr = s.surface.normals.data(); v.count = 3u * s.surface.num_vertices; v.elem = 4; break;
        case SLOSH_BUF_SURFACE_TANGENTS: v.ptr = s.surface.tangents.data(); v.count = 3u * s.surface.num_vertices; v.elem = 4; break;
        case SLOSH_BUF_SURFACE_INDICES: u32(s.surface.indices, s.surface.num_indices); break;
        default: break;
    }
    return v;
}

}  // namespace

ORACLE_API void oracle_settings_default(slosh_settings_t* out) { settings_default(out); }
ORACLE_API uint16_t oracle_f32_to_f16(float f) { return f32_to_f16(f); }
ORACLE_API uint16_t oracle_f32_to_bf16(float f) { return f32_to_bf16(f); }
ORACLE_API float oracle_f16_to_f32(uint16_t h) { return f16_to_f32(h); }
ORACLE_API uint32_t oracle_pcg_hash(uint32_t v) { return pcg_hash(v); }
ORACLE_API float oracle_hash_to_unit(uint32_t v) { return hash_to_unit(v); }
ORACLE_API double oracle_reduce_final(const double* p, uint32_t n) { return reduce_final(p, n); }
ORACLE_API double oracle_reduce_brick(const double* v) { return reduce_brick(v); }

ORACLE_API int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

ORACLE_API int oracle_create(const slosh_settings_t* settings, int fp64, void** out) {
    if (!settings || !out) return SLOSH_ERR_INVALID_ARG;
    Handle* h = new Handle();
    h->fp64 = fp64 ? 1 : 0;
    slosh_settings_t s = clamp_settings(*settings);
    if (h->fp64) { h->d.reset(new Sim<double>()); h->d->allocate(s); }
    else { h->f.reset(new Sim<float>()); h->f->allocate(s); }
    *out = h;
    return SLOSH_OK;
}
ORACLE_API void oracle_destroy(void* h) { delete static_cast<Handle*>(h); }

ORACLE_API int oracle_set_emit_seed(void* h, uint32_t seed) {
    return dispatch(h, [&](auto& s) { s.emit_seed = seed; return int(SLOSH_OK); });
}
// Frame input for the calls that need one but whose caller only has settings.
ORACLE_API int oracle_begin_frame(void* h, const slosh_frame_input_t* in, int32_t* out_substeps, float* out_dt) {
    if (!in) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) {
        int n = s.begin_frame(*in, out_dt);
        if (out_substeps) *out_substeps = n;
        return int(SLOSH_OK);
    });
}
ORACLE_API int oracle_substep(void* h, int32_t step) {
    return dispatch(h, [&](auto& s) {
        if (step < 0 || step >= s.substeps) return int(SLOSH_ERR_INVALID_ARG);
        s.substep(step);
        return int(SLOSH_OK);
    });
}
ORACLE_API int oracle_end_frame(void* h) {
    return dispatch(h, [&](auto& s) { s.end_frame(); return int(SLOSH_OK); });
}
ORACLE_API int oracle_step_frame(void* h, const slosh_frame_input_t* in) {
    if (!in) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) { s.step_frame(*in); return int(SLOSH_OK); });
}
ORACLE_API int oracle_emit(void* h, const slosh_emit_request_t* em) {
    if (!em) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) { s.emit(*em); return int(SLOSH_OK); });
}
ORACLE_API int oracle_sort_particles(void* h) {
    return dispatch(h, [&](auto& s) { s.sort_particles(); return int(SLOSH_OK); });
}
ORACLE_API int oracle_upload_particles(void* h, const slosh_particle_t* p, uint32_t n) {
    return dispatch(h, [&](auto& s) {
        if (n > s.particles.size()) return int(SLOSH_ERR_CAPACITY);
        s.upload(p, n);
        return int(SLOSH_OK);
    });
}
ORACLE_API int oracle_get_layout(void* h, slosh_layout_t* out) {
    if (!out) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) { fill_layout(s, out); return int(SLOSH_OK); });
}
ORACLE_API int oracle_get_results(void* h, slosh_results_t* out) {
    if (!out) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) { decode_results(s, out); return int(SLOSH_OK); });
}
// Bytes of a buffer as exported: float-valued buffers are exported as f32 (rounded from FP64).
ORACLE_API int oracle_buffer_bytes(void* h, int id, size_t* out) {
    if (!out) return SLOSH_ERR_INVALID_ARG;
    return dispatch(h, [&](auto& s) {
        auto v = view(s, id);
        if (!v.ptr && v.count) return int(SLOSH_ERR_INVALID_ARG);
        if (id < 0 || id >= SLOSH_BUF_COUNT_) return int(SLOSH_ERR_INVALID_ARG);
        *out = v.count * (v.is_real ? 4 : v.elem);
        return int(SLOSH_OK);
    });
}
ORACLE_API int oracle_read_buffer(void* h, int id, void* dst, size_t bytes) {
    return dispatch(h, [&](auto& s) {
        using R = typename std::remove_reference<decltype(s)>::type::Real_;
        auto v = view(s, id);
        if (id < 0 || id >= SLOSH_BUF_COUNT_) return int(SLOSH_ERR_INVALID_ARG);
        const size_t need = v.count * (v.is_real ? 4 : v.elem);
        if (bytes < need) return int(SLOSH_ERR_INVALID_ARG);
        if (v.is_real) {
            const R* src = static_cast<const R*>(v.ptr);
            float* d = static_cast<float*>(dst);
            for (size_t i = 0; i < v.count; ++i) d[i] = float(src[i]);
        } else if (need) {
            std::memcpy(dst, v.ptr, need);
        }
        return int(SLOSH_OK);
    });
}
// Float-valued buffers at the oracle's own precision, widened to double.
ORACLE_API int oracle_read_buffer_f64(void* h, int id, double* dst, size_t count) {
    return dispatch(h, [&](auto& s) {
        using R = typename std::remove_reference<decltype(s)>::type::Real_;
        auto v = view(s, id);
        if (!v.is_real || count < v.count) return int(SLOSH_ERR_INVALID_ARG);
        const R* src = static_cast<const R*>(v.ptr);
        for (size_t i = 0; i < v.count; ++i) dst[i] = double(src[i]);
        return int(SLOSH_OK);
    });
}
ORACLE_API int oracle_write_buffer(void* h, int id, const void* src, size_t bytes) {
    return dispatch(h, [&](auto& s) {
        using R = typename std::remove_reference<decltype(s)>::type::Real_;
        if (id == SLOSH_BUF_PARTICLES) {
            size_t n = bytes / sizeof(slosh_particle_t);
            if (n > s.particles.size()) return int(SLOSH_ERR_CAPACITY);
            std::memcpy(s.particles.data(), src, n * sizeof(slosh_particle_t));
            s.num_particles = uint32_t(n);
            return int(SLOSH_OK);
        }
        auto v = view(s, id);
        if (id < 0 || id >= SLOSH_BUF_COUNT_) return int(SLOSH_ERR_INVALID_ARG);
        const size_t need = v.count * (v.is_real ? 4 : v.elem);
        if (bytes != need) return int(SLOSH_ERR_INVALID_ARG);
        if (v.is_real) {
            const float* sp = static_cast<const float*>(src);
            R* d = static_cast<R*>(v.ptr);
            for (size_t i = 0; i < v.count; ++i) d[i] = R(sp[i]);
        } else if (need) {
            std::memcpy(v.ptr, src, need);
        }
        return int(SLOSH_OK);
    });
}
// Copies the whole simulation state of src into dst (either precision): the FP64 oracle of a step
// starts from the FP32 state of the step before it.
ORACLE_API int oracle_copy_state(void* dst, void* src) {
    if (!dst || !src) return SLOSH_ERR_INVALID_ARG;
    Handle* D = static_cast<Handle*>(dst);
    Handle* S = static_cast<Handle*>(src);
    auto copy = [](auto& d, const auto& s) {
        using RD = typename std::remove_reference<decltype(d)>::type::Real_;
        auto cv = [](std::vector<RD>& out, const auto& in) { out.assign(in.begin(), in.end()); };
        d.S = s.S; d.L = s.L; d.allocated = s.allocated; d.P = s.P;
        d.particles = s.particles; d.particles_sorted = s.particles_sorted;
        d.num_particles = s.num_particles;
        std::copy(s.particle_count, s.particle_count + 4, d.particle_count);
        d.total_emitted = s.total_emitted; d.sim_frame = s.sim_frame; d.emit_seed = s.emit_seed;
        d.prev_dt = s.prev_dt; d.last_max_speed = s.last_max_speed;
        for (int i = 0; i < 3; ++i) cv(d.vel[i], s.vel[i]);
        cv(d.vel_old, s.vel_old); cv(d.face_weight, s.face_weight); cv(d.pressure, s.pressure);
        cv(d.divergence, s.divergence); cv(d.cell_diag, s.cell_diag); cv(d.density_q, s.density_q);
        cv(d.density_rhs, s.density_rhs);
        d.accum = s.accum; d.cell_count = s.cell_count; d.face_flags = s.face_flags; d.cell_type = s.cell_type;
        d.brick_table = s.brick_table; d.slot_brick = s.slot_brick; d.free_slots = s.free_slots;
        d.brick_touch = s.brick_touch; d.brick_want = s.brick_want; d.new_slots = s.new_slots;
        d.active_bricks = s.active_bricks; d.sort_counts = s.sort_counts; d.sort_offsets = s.sort_offsets;
        d.sort_perm = s.sort_perm; d.sort_keys = s.sort_keys;
        std::copy(s.stats, s.stats + NUM_STATS, d.stats);
        std::copy(s.coupling, s.coupling + SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE, d.coupling);
        d.colliders = s.colliders; d.manipulators = s.manipulators;
        d.mg.assign(s.mg.size(), {});
        for (size_t l = 0; l < s.mg.size(); ++l) {
            d.mg[l].dim = s.mg[l].dim; d.mg[l].cells = s.mg[l].cells; d.mg[l].type = s.mg[l].type;
            cv(d.mg[l].x, s.mg[l].x); cv(d.mg[l].b, s.mg[l].b);
        }
        cv(d.pcg_r, s.pcg_r); cv(d.pcg_z, s.pcg_z); cv(d.pcg_d, s.pcg_d); cv(d.pcg_q, s.pcg_q);
        std::copy(s.scalars, s.scalars + 5, d.scalars);
        d.cur = s.cur; d.substeps = s.substeps; d.frame_dt_sub = s.frame_dt_sub;
        d.density_projection_this_frame = s.density_projection_this_frame;
        d.last_disp_index = s.last_disp_index;
    };
    if (D->fp64 && S->fp64) copy(*D->d, *S->d);
    else if (D->fp64) copy(*D->d, *S->f);
    else if (S->fp64) copy(*D->f, *S->d);
    else copy(*D->f, *S->f);
    return SLOSH_OK;
}

// Headless surface of the current particles (slosh_build_surface).
ORACLE_API int oracle_build_surface(void* h, const slosh_surface_params_t* q, slosh_surface_info_t* out) {
    if (!h || !q) return int(SLOSH_ERR_INVALID_ARG);
    return dispatch(h, [&](auto& s) {
        build_surface(s.particles.data(), s.num_particles, s.L.grid, s.S.cell_size, *q, s.surface);
        if (out) {
            std::memset(out, 0, sizeof(*out));
            for (int a = 0; a < 3; ++a) { out->field_dim[a] = s.surface.dim[a]; out->brick_dim[a] = s.surface.bdim[a]; }
            out->voxel_size = s.surface.voxel;
            out->vertices_requested = s.surface.vertices_requested;
            out->num_vertices = s.surface.num_vertices;
            out->indices_requested = s.surface.indices_requested;
            out->num_indices = s.surface.num_indices;
        }
        return int(SLOSH_OK);
    });
}
