// TEST INFRASTRUCTURE -- not part of the product. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py load this code, and only as the reference the GPU results are compared
// with (or, in bench.py, as the timed CPU baseline).
//
// CPU oracle of the Slosh FLIP/APIC simulation substep: a statement-by-statement restatement of the
// reference's HLSL kernels and of the C++ schedule that dispatches them (paths relative to the
// reference project; PLUG = SloshDemo/Plugins/Slosh):
//   PLUG/Shaders/Private/SloshCommon.ush      particle packing, hashing, SDFs, ghost-fluid theta
//   PLUG/Shaders/Private/Slosh.usf            brick pool, P2G, grid passes, RBGS, projection, G2P
//   PLUG/Shaders/Private/SloshPressureMG.usf  MGPCG
//   PLUG/Shaders/Private/SloshSort.usf        counting sort
//   PLUG/Source/SloshCore/Private/SloshProxy.cpp  Allocate, Step_RenderThread, MGPCG and sort drivers
//
// Every "dispatch" runs as a loop over the linear thread id in ascending order, so each atomic of the
// reference resolves in ascending-id order. That is the canonical order for the two order-dependent
// results of the reference: the sort ranks (SloshSort.usf:73-75) and the brick-pool slot assignment
// (Slosh.usf:1754-1756,1777-1788).
//
// Arithmetic: Real = float restates the FP32 shaders; Real = double is the FP64 error reference of the
// same step. Every float expression keeps the operation order of the HLSL source; compile with
// -ffp-contract=off. Deliberate, documented deviations from the HLSL:
//   * lerp(1 - f, f, o) with o in {0, 1} is evaluated as (o ? f : 1 - f), the value the HLSL intends;
//   * PCG dot products (r.z, d.Ad) accumulate the FP32 products in FP64 through a fixed tree (one
//     partial per 8^3 brick, then one over bricks; reduce_brick / reduce_final below) instead of the
//     reference's FP32 group tree (SloshPressureMG.usf:234-251,457-492); alpha and beta are formed
//     in FP64 and rounded to FP32;
//   * MGPCG can stop at a relative residual ||r||/||b|| <= tolerance (the reference runs a fixed count,
//     SloshProxy.cpp:990-1019); with tolerance <= 0 it runs the reference's fixed count.
//
// PARITY UNPINNED BY REFERENCE TESTS: the reference has no unit tests, fixtures or golden vectors
// (Docs/Testing.md:3) and its HLSL only runs inside Unreal's D3D12 renderer, which is unavailable
// here. This restatement is pinned instead by independent checks in tests/ (numpy float16 rounding,
// numpy stable argsort, a dense scipy solve of the pressure system, analytic P2G weight sums, a
// hydrostatic pool, post-projection divergence).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/slosh_cuda.h"

namespace slosh_oracle {

// ---- constants: SloshCommon.ush:27-48, Slosh.usf:106-108 -------------------------------------
constexpr uint32_t CELL_AIR = 0u, CELL_FLUID = 1u, CELL_SOLID = 2u, CELL_TYPE_MASK = 3u;
constexpr uint32_t CELL_DENSE_FLAG = 4u, CELL_COLLIDER_SHIFT = 8u;
constexpr uint32_t FACE_VALID = 1u, FACE_SOLID = 2u, FACE_HAS_WEIGHT = 4u, FACE_EXTRAP_SHIFT = 4u;
constexpr uint32_t BRICK_CELLS = 512u, NO_BRICK = 0xFFFFFFFFu;
constexpr uint32_t COLLIDER_FLAG_TWO_WAY = 1u;
constexpr uint32_t MANIP_DRAIN = 0u, MANIP_DIRECTIONAL = 1u, MANIP_RADIAL = 2u, MANIP_SWIRL = 3u, MANIP_DRAG = 4u;
constexpr uint32_t MANIP_SHAPE_EVERYWHERE = 3u;
constexpr float P2G_FIXED_SCALE = 1048576.0f;           // SloshCommon.ush:47
constexpr float P2G_FIXED_INV = 1.0f / 1048576.0f;      // SloshCommon.ush:48
constexpr uint32_t NUM_STATS = 16u;                     // SloshProxy.cpp:17
constexpr uint32_t MG_COARSEST_MAX_CELLS = 512u;        // SloshProxy.cpp:73
constexpr int MG_MAX_LEVELS = 8;                        // SloshProxy.cpp:75

inline uint32_t f32_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bits_f32(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// f32tof16 with round-to-nearest-even, subnormals kept (SloshCommon.ush:71-74).
inline uint16_t f32_to_f16(float f) {
    const uint32_t x = f32_bits(f);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t mant = x & 0x7FFFFFu;
    if (exp == 0xFFu) return uint16_t(sign | 0x7C00u | (mant ? (0x200u | (mant >> 13)) : 0u));
    const int e = int(exp) - 112;  // half exponent field
    if (e >= 31) return uint16_t(sign | 0x7C00u);
    if (e >= 1) {
        uint32_t h = (uint32_t(e) << 10) | (mant >> 13);
        const uint32_t low = mant & 0x1FFFu;
        if (low > 0x1000u || (low == 0x1000u && (h & 1u))) h += 1u;  // carry may reach the exponent
        return uint16_t(sign | h);
    }
    if (exp == 0u) return uint16_t(sign);  // float zero / subnormal: far below half range
    const uint32_t sig = mant | 0x800000u;
    const uint32_t shift = 126u - exp;     // >= 14
    if (shift > 31u) return uint16_t(sign);
    uint32_t m = sig >> shift;
    const uint32_t rem = sig & ((1u << shift) - 1u);
    const uint32_t halfway = 1u << (shift - 1u);
    if (rem > halfway || (rem == halfway && (m & 1u))) m += 1u;
    return uint16_t(sign | m);
}

// f16tof32 (exact).
// FP32 -> BF16, round to nearest even (NaN stays NaN, quiet); BF16 -> FP32 is exact.
inline uint16_t f32_to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7FFFFFFFu) > 0x7F800000u) return uint16_t((u >> 16) | 0x40u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}
inline float bf16_to_f32(uint16_t h) {
    const uint32_t u = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline float f16_to_f32(uint16_t h) {
    const uint32_t sign = uint32_t(h & 0x8000u) << 16;
    const uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t mant = h & 0x3FFu;
    uint32_t out;
    if (exp == 0u) {
        if (mant == 0u) {
            out = sign;
        } else {
            int e = -1;
            do { mant <<= 1; ++e; } while ((mant & 0x400u) == 0u);
            out = sign | (uint32_t(127 - 15 - e) << 23) | ((mant & 0x3FFu) << 13);
        }
    } else if (exp == 0x1Fu) {
        out = sign | 0x7F800000u | (mant << 13);
    } else {
        out = sign | ((exp + 112u) << 23) | (mant << 13);
    }
    return bits_f32(out);
}

// PcgHash / HashToUnitFloat, SloshCommon.ush:255-265.
inline uint32_t pcg_hash(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline float hash_to_unit(uint32_t h) { return float(h & 0x00FFFFFFu) / 16777216.0f; }

// int(round(x)): round half to even, saturating at the int32 range, NaN -> 0 (the GPU's cvt.rni.s32).
template <class R> inline int32_t to_i32_rn(R x) {
    if (x != x) return 0;
    if (x >= R(2147483647.0)) return 2147483647;
    if (x <= R(-2147483648.0)) return int32_t(-2147483647 - 1);
    return int32_t(std::nearbyint(x));
}

// ---- small vector types ----------------------------------------------------------------------
struct I3 {
    int x, y, z;
    int& operator[](int i) { return (&x)[i]; }
    int operator[](int i) const { return (&x)[i]; }
};
inline I3 operator+(I3 a, I3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline I3 operator-(I3 a, I3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline I3 axis_offset(int a) { return {a == 0 ? 1 : 0, a == 1 ? 1 : 0, a == 2 ? 1 : 0}; }
// Neighbour N of the 6-stencil: N = 0..5 -> -x, +x, -y, +y, -z, +z (Slosh.usf:732-736).
inline I3 neighbour_offset(int n) {
    I3 d{0, 0, 0};
    d[n >> 1] = (n & 1) ? 1 : -1;
    return d;
}

template <class R>
struct V3 {
    R x, y, z;
    R& operator[](int i) { return (&x)[i]; }
    R operator[](int i) const { return (&x)[i]; }
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R clampr(R v, R lo, R hi) { return std::fmin(std::fmax(v, lo), hi); }
template <class R> inline R saturate(R v) { return clampr(v, R(0), R(1)); }
inline int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

// QuatRotate / QuatRotateInv, SloshCommon.ush:137-146.
template <class R> inline V3<R> quat_rotate(const float* q, V3<R> v) {
    V3<R> qv{R(q[0]), R(q[1]), R(q[2])};
    V3<R> t = R(2) * cross(qv, v);
    return v + R(q[3]) * t + cross(qv, t);
}
template <class R> inline V3<R> quat_rotate_inv(const float* q, V3<R> v) {
    float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    return quat_rotate<R>(qi, v);
}

// ColliderSDF / ColliderNormal / ColliderVelocityAt, SloshCommon.ush:178-235.
template <class R> inline R collider_sdf(const slosh_collider_t& c, V3<R> p) {
    V3<R> l = quat_rotate_inv<R>(c.rotation, p - V3<R>{R(c.center[0]), R(c.center[1]), R(c.center[2])});
    if (c.type == SLOSH_COLLIDER_SPHERE) return length(l) - R(c.extent[0]);
    if (c.type == SLOSH_COLLIDER_BOX) {
        V3<R> d{std::fabs(l.x) - R(c.extent[0]), std::fabs(l.y) - R(c.extent[1]), std::fabs(l.z) - R(c.extent[2])};
        V3<R> dp{std::fmax(d.x, R(0)), std::fmax(d.y, R(0)), std::fmax(d.z, R(0))};
        return length(dp) + std::fmin(std::fmax(d.x, std::fmax(d.y, d.z)), R(0));
    }
    l.z = l.z - clampr(l.z, -R(c.extent[1]), R(c.extent[1]));
    return length(l) - R(c.extent[0]);
}
template <class R> inline V3<R> collider_normal(const slosh_collider_t& c, V3<R> p, R eps) {
    V3<R> n;
    n.x = collider_sdf<R>(c, p + V3<R>{eps, R(0), R(0)}) - collider_sdf<R>(c, p - V3<R>{eps, R(0), R(0)});
    n.y = collider_sdf<R>(c, p + V3<R>{R(0), eps, R(0)}) - collider_sdf<R>(c, p - V3<R>{R(0), eps, R(0)});
    n.z = collider_sdf<R>(c, p + V3<R>{R(0), R(0), eps}) - collider_sdf<R>(c, p - V3<R>{R(0), R(0), eps});
    R len = length(n);
    return len > R(1e-8f) ? V3<R>{n.x / len, n.y / len, n.z / len} : V3<R>{R(0), R(0), R(1)};
}
template <class R> inline V3<R> collider_velocity_at(const slosh_collider_t& c, V3<R> p) {
    V3<R> w{R(c.angular_velocity[0]), R(c.angular_velocity[1]), R(c.angular_velocity[2])};
    V3<R> lin{R(c.linear_velocity[0]), R(c.linear_velocity[1]), R(c.linear_velocity[2])};
    return lin + cross(w, p - V3<R>{R(c.center[0]), R(c.center[1]), R(c.center[2])});
}
// ManipulatorSDF / ManipulatorWeight, SloshCommon.ush:207-230.
template <class R> inline R manipulator_sdf(const slosh_manipulator_t& f, V3<R> p) {
    if (f.shape == MANIP_SHAPE_EVERYWHERE) return R(-1);
    slosh_collider_t c{};
    std::memcpy(c.center, f.center, sizeof(c.center));
    c.type = f.shape;
    std::memcpy(c.rotation, f.rotation, sizeof(c.rotation));
    std::memcpy(c.extent, f.extent, sizeof(c.extent));
    return collider_sdf<R>(c, p);
}
template <class R> inline R manipulator_weight(const slosh_manipulator_t& f, V3<R> p) {
    R d = manipulator_sdf<R>(f, p);
    if (d <= R(0)) return R(1);
    return R(f.falloff) > R(0) ? saturate(R(1) - d / R(f.falloff)) : R(0);
}

// GhostTheta, SloshCommon.ush:242-252.
template <class R> inline R ghost_theta(R rho_fluid, R rho_air) {
    R denom = rho_fluid - rho_air;
    if (denom <= R(1e-4f)) return R(1);
    return clampr((rho_fluid - R(0.5f)) / denom, R(0.05f), R(1));
}

// ---- particle record: FSloshParticlePacked, SloshCommon.ush:50-105 --------------------------------
static_assert(sizeof(slosh_particle_t) == 48, "48-byte particle");
template <class R> struct ParticleU {
    V3<R> pos, vel, cx, cy, cz;
    R age;
};
inline uint32_t pack_half2(float a, float b) {
    return uint32_t(f32_to_f16(clampr(a, -65000.0f, 65000.0f))) |
           (uint32_t(f32_to_f16(clampr(b, -65000.0f, 65000.0f))) << 16);
}
template <class R> inline slosh_particle_t pack_particle(const ParticleU<R>& p) {
    slosh_particle_t s;
    s.pos[0] = float(p.pos.x); s.pos[1] = float(p.pos.y); s.pos[2] = float(p.pos.z);
    s.age = float(p.age);
    s.vel[0] = float(p.vel.x); s.vel[1] = float(p.vel.y); s.vel[2] = float(p.vel.z);
    s.c[0] = pack_half2(float(p.cx.x), float(p.cx.y));
    s.c[1] = pack_half2(float(p.cx.z), float(p.cy.x));
    s.c[2] = pack_half2(float(p.cy.y), float(p.cy.z));
    s.c[3] = pack_half2(float(p.cz.x), float(p.cz.y));
    s.c[4] = pack_half2(float(p.cz.z), 0.0f);
    return s;
}
template <class R> inline ParticleU<R> unpack_particle(const slosh_particle_t& s) {
    ParticleU<R> p;
    p.pos = {R(s.pos[0]), R(s.pos[1]), R(s.pos[2])};
    p.age = R(s.age);
    p.vel = {R(s.vel[0]), R(s.vel[1]), R(s.vel[2])};
    auto h = [&](int w, int hi) { return R(f16_to_f32(uint16_t(hi ? (s.c[w] >> 16) : (s.c[w] & 0xFFFFu)))); };
    p.cx = {h(0, 0), h(0, 1), h(1, 0)};
    p.cy = {h(1, 1), h(2, 0), h(2, 1)};
    p.cz = {h(3, 0), h(3, 1), h(4, 0)};
    return p;
}
inline slosh_particle_t dead_particle() {  // DeadParticlePacked, Slosh.usf:256-261
    ParticleU<float> d{};
    d.pos = {0, 0, 0}; d.vel = {0, 0, 0}; d.cx = {0, 0, 0}; d.cy = {0, 0, 0}; d.cz = {0, 0, 0};
    d.age = -1.0f;
    return pack_particle(d);
}
inline bool is_dead_age(float age) { return !(age >= 0.0f); }  // SloshCommon.ush:172-175

// ---- settings and layout ---------------------------------------------------------------------
inline void settings_default(slosh_settings_t* s) {  // SloshTypes.h:113-160
    std::memset(s, 0, sizeof(*s));
    s->grid_dim[0] = 64; s->grid_dim[1] = 64; s->grid_dim[2] = 48;
    s->cell_size = 0.05f;
    s->particle_capacity = 262144u;
    s->transfer_mode = SLOSH_TRANSFER_APIC;
    s->flip_ratio = 0.95f;
    s->density = 1000.0f;
    s->kinematic_viscosity = 0.0f;
    s->boundary_friction = 0.0f;
    s->adhesion = 0.0f;
    s->adhesion_distance = 0.025f;
    s->density_correction = 0.15f;
    s->density_deadband = 0.05f;
    s->two_sided_density_projection = 1u;
    s->density_relaxation = 0.5f;
    s->density_projection_iterations = 30;
    s->density_projection_interval = 1;
    s->sparse_bricks = 1u;
    s->sparse_max_active_fraction = 0.5f;
    s->sparse_storage_budget = 1.0f;
    s->particle_radius_cells = 0.25f;
    s->gravity[0] = 0.0f; s->gravity[1] = 0.0f; s->gravity[2] = -9.81f;
    s->pressure_solver = SLOSH_SOLVER_MGPCG;
    s->pressure_iterations = 60;
    s->sor_weight = 1.7f;
    s->pcg_iterations = 8;
    s->mg_coarse_iterations = 16;
    s->sort_interval = 4;
    s->smooth_coupling_force = 1u;
    s->ghost_fluid = 1u;
    s->viscosity_iterations = 12;
    s->extrapolation_layers = 2;
    s->min_substeps = 1;
    s->max_substeps = 4;
    s->max_frame_dt = 1.0f / 30.0f;
    s->cfl = 2.0f;
    s->max_speed = 20.0f;
    s->tolerance = 0.0f;
    s->max_iterations = 200;
    s->precision_mode = SLOSH_PRECISION_FP32;
    s->warm_start = SLOSH_WARM_START_PREVIOUS;
    s->mg_correction_scale = 1.0f;
    s->mg_smoothing_sweeps = 1;
    s->pcg_flexible = 0u;
    s->mg_smoother_weight = 1.0f;
}

// Step_RenderThread's clamps (SloshProxy.cpp:344-347). The grid and particle caps are raised above
// the reference's 256 cells per axis and 16M particles.
inline slosh_settings_t clamp_settings(slosh_settings_t s) {
    for (int a = 0; a < 3; ++a) s.grid_dim[a] = clampi(s.grid_dim[a], 4, 2048);
    s.particle_capacity = std::min(std::max(s.particle_capacity, 1024u), 1u << 28);
    s.cell_size = std::max(s.cell_size, 1e-3f);
    return s;
}

struct Layout {
    I3 grid{0, 0, 0}, brick_dim{0, 0, 0}, sort_brick_dim{0, 0, 0};
    uint32_t num_cells = 0, num_bricks = 0, num_pool_bricks = 0, pool_cells = 0, pool_scan_cells = 0;
    uint32_t total_faces = 0, num_sort_keys = 0;
    int num_levels = 0;
    I3 level_dim[MG_MAX_LEVELS];
    uint32_t level_cells[MG_MAX_LEVELS];
};

// FSloshProxy::Allocate sizes, SloshProxy.cpp:185-285.
inline Layout make_layout(const slosh_settings_t& s) {
    Layout L;
    L.grid = {s.grid_dim[0], s.grid_dim[1], s.grid_dim[2]};
    L.num_cells = uint32_t(L.grid.x) * uint32_t(L.grid.y) * uint32_t(L.grid.z);
    L.brick_dim = {(L.grid.x + 7) / 8, (L.grid.y + 7) / 8, (L.grid.z + 7) / 8};
    L.num_bricks = uint32_t(L.brick_dim.x) * uint32_t(L.brick_dim.y) * uint32_t(L.brick_dim.z);
    const double budget = double(clampr(s.sparse_storage_budget, 0.0f, 1.0f));
    uint32_t slots = uint32_t(std::ceil(budget * double(L.num_bricks)));
    slots = std::min(std::max(slots, 1u), L.num_bricks);
    L.num_pool_bricks = slots + 1u;
    L.pool_cells = L.num_pool_bricks * BRICK_CELLS;
    L.pool_scan_cells = slots * BRICK_CELLS;
    L.total_faces = 3u * L.pool_cells;
    L.sort_brick_dim = {(L.grid.x + 3) / 4, (L.grid.y + 3) / 4, (L.grid.z + 3) / 4};
    L.num_sort_keys = uint32_t(L.sort_brick_dim.x) * uint32_t(L.sort_brick_dim.y) * uint32_t(L.sort_brick_dim.z) + 1u;
    L.num_levels = 1;
    L.level_dim[0] = L.grid;
    L.level_cells[0] = L.num_cells;
    while (L.level_cells[L.num_levels - 1] > MG_COARSEST_MAX_CELLS && L.num_levels < MG_MAX_LEVELS) {
        I3 p = L.level_dim[L.num_levels - 1];
        I3 d{(p.x + 1) / 2, (p.y + 1) / 2, (p.z + 1) / 2};
        L.level_dim[L.num_levels] = d;
        L.level_cells[L.num_levels] = uint32_t(d.x) * uint32_t(d.y) * uint32_t(d.z);
        ++L.num_levels;
    }
    return L;
}
inline bool layout_equals(const slosh_settings_t& a, const slosh_settings_t& b) {  // SloshTypes.h:156-159
    return a.grid_dim[0] == b.grid_dim[0] && a.grid_dim[1] == b.grid_dim[1] && a.grid_dim[2] == b.grid_dim[2] &&
           a.sparse_storage_budget == b.sparse_storage_budget;
}

// Transcendentals of emission, drag and drain: evaluated in double and rounded to float, as the CUDA
// path does (float sinf/cosf/expf/powf of the C library and of CUDA differ in the last bit).
inline float sin_r(float x) { return float(std::sin(double(x))); }
inline float cos_r(float x) { return float(std::cos(double(x))); }
inline float exp_r(float x) { return float(std::exp(double(x))); }
inline float pow_r(float x, float y) { return float(std::pow(double(x), double(y))); }

// ---- canonical FP64 reduction tree of the PCG dots -------------------------------------------
// One partial per 8^3 brick (v in local order x + 8 y + 64 z): 32 lanes; in round k = 0..3 lane t owns
// the 4 cells x = 4h .. 4h + 3 of row y in plane z (h = t & 1, y = (t >> 1) & 7, z = 2k + (t >> 4)) and
// adds them round by round, x ascending, starting from 0.0; the lanes then fold with offsets 16, 8, 4,
// 2, 1 (lane j += lane j + off).
inline double reduce_brick(const double* v) {
    double s[32];
    for (int t = 0; t < 32; ++t) {
        double acc = 0.0;
        const int h = t & 1, y = (t >> 1) & 7;
        for (int k = 0; k < 4; ++k) {
            const int z = 2 * k + (t >> 4);
            for (int j = 0; j < 4; ++j) acc = acc + v[4 * h + j + 8 * y + 64 * z];
        }
        s[t] = acc;
    }
    for (int off = 16; off >= 1; off >>= 1)
        for (int j = 0; j < off; ++j) s[j] = s[j] + s[j + off];
    return s[0];
}
// Over bricks: 1024 lanes, lane t sums entries t, t + 1024, ... in order; each warp folds as above;
// the 32 warp results are added in warp order.
inline double reduce_final(const double* p, uint32_t n) {
    std::vector<double> s(1024, 0.0);
    for (uint32_t t = 0; t < 1024u; ++t) {
        double acc = 0.0;
        for (uint32_t e = t; e < n; e += 1024u) acc = acc + p[e];
        s[t] = acc;
    }
    double total = 0.0;
    for (int w = 0; w < 32; ++w) {
        double* l = s.data() + 32 * w;
        for (int off = 16; off >= 1; off >>= 1)
            for (int j = 0; j < off; ++j) l[j] = l[j] + l[j + off];
        total = (w == 0) ? l[0] : total + l[0];
    }
    return total;
}

// Per-frame pass parameters (FSloshPassParameters as filled by Step_RenderThread, SloshProxy.cpp:400-483).
struct PassParams {
    float cell_size = 0, inv_cell_size = 0, dt = 0;
    float gravity[3] = {0, 0, 0};
    float flip_ratio = 0, max_speed = 0, friction = 0, adhesion_accel = 0, adhesion_range = 0;
    float particle_radius = 0, viscosity_alpha = 0, sor_weight = 0, warm_start_scale = 1;
    float pressure_to_pascal = 0, density_correction = 0, target_ppc = 8.0f, density_deadband = 0;
    float coupling_scale = 1024.0f, density_relaxation = 0;
    uint32_t use_apic = 1, smooth_coupling = 1, ghost_fluid = 1, num_colliders = 0, num_manipulators = 0;
    uint32_t precision_mode = SLOSH_PRECISION_FP32;  // storage of the coarse MG levels
    float restrict_scale = 0.25f;  // factor of the restriction's fluid-child sum: 0.25 x mg_correction_scale
    int mg_sweeps = 1;             // red-black sweep pairs per pre- and post-smoothing (mg_smoothing_sweeps)
    uint32_t pcg_flexible = 0;     // flexible (Polak-Ribiere) beta
    float smooth_weight = 1.0f;    // over-relaxation of level 0's red-black sweeps (mg_smoother_weight)
    uint32_t frame_seed = 0;
};

// =============================================================================================
// The simulation state and its kernels.
// =============================================================================================
// ---- headless surface (SloshSurface.usf:54-470; parameters SloshRenderer.cpp:118-170) -------------------------
// Density splat of sphere-mode ellipsoids, resolve to the f16 Zhu & Bridson field with dilated brick
// occupancy, and surface nets with vertices and quads numbered in cell order (the CUDA path numbers them
// the same way through scans). Computed in FP32 from the particle records, whatever the simulation's R.
struct SurfaceOut {
    int dim[3] = {0, 0, 0}, bdim[3] = {0, 0, 0};
    float voxel = 0.0f;
    std::vector<uint16_t> field;
    std::vector<uint32_t> bricks;
    std::vector<float> positions, normals, tangents;
    std::vector<uint32_t> indices;
    uint32_t vertices_requested = 0, indices_requested = 0, num_vertices = 0, num_indices = 0;
};
inline void build_surface(const slosh_particle_t* particles, uint32_t n, I3 grid, float cell, const slosh_surface_params_t& q, SurfaceOut& o) {
    const float res = clampr(q.field_resolution, 0.5f, 3.0f);
    o.voxel = cell / res;
    const float inv_voxel = 1.0f / o.voxel;
    const int dim[3] = {int(std::ceil(float(grid.x) * res)), int(std::ceil(float(grid.y) * res)), int(std::ceil(float(grid.z) * res))};
    for (int a = 0; a < 3; ++a) { o.dim[a] = dim[a]; o.bdim[a] = (dim[a] + 7) / 8; }
    const float support = clampr(q.surface_smoothing, 0.5f, 6.0f), max_fp = 4.0f;
    const float radius_voxels = q.particle_radius_scale * res, splat_radius = cell * q.particle_radius_scale;
    const float iso = clampr(q.iso_level, 0.02f, 0.98f);
    const size_t nv = size_t(dim[0]) * dim[1] * dim[2], nb = size_t(o.bdim[0]) * o.bdim[1] * o.bdim[2];
    auto vox = [&](int x, int y, int z) { return size_t(x) + size_t(dim[0]) * (size_t(y) + size_t(dim[1]) * size_t(z)); };
    auto fbrick = [&](int x, int y, int z) {
        const int bx = clampi(x >> 3, 0, o.bdim[0] - 1), by = clampi(y >> 3, 0, o.bdim[1] - 1), bz = clampi(z >> 3, 0, o.bdim[2] - 1);
        return size_t(bx) + size_t(o.bdim[0]) * (size_t(by) + size_t(o.bdim[1]) * size_t(bz));
    };
    auto add = [](int32_t& a, int32_t v) { a = int32_t(uint32_t(a) + uint32_t(v)); };
    // DensitySplatCS
    std::vector<int32_t> acc(nv * 5, 0);
    for (uint32_t i = 0; i < n; ++i) {
        const slosh_particle_t& p = particles[i];
        if (is_dead_age(p.age)) continue;
        const V3<float> axis[3] = {{splat_radius, 0.0f, 0.0f}, {0.0f, splat_radius, 0.0f}, {0.0f, 0.0f, splat_radius}};
        const float k = support * inv_voxel;
        const V3<float> c{p.pos[0] * inv_voxel, p.pos[1] * inv_voxel, p.pos[2] * inv_voxel};
        V3<float> w[3];
        float amax = 0.0f;
        for (int a = 0; a < 3; ++a) {
            const V3<float> u{axis[a].x * k, axis[a].y * k, axis[a].z * k};
            const float aa = std::fmax(dot(u, u), 1e-8f);
            w[a] = V3<float>{u.x / aa, u.y / aa, u.z / aa};
            amax = a == 0 ? aa : std::fmax(amax, aa);
        }
        const float rr = std::fmin(std::sqrt(amax), max_fp);
        const int lo[3] = {std::max(int(std::floor(c.x - rr - 0.5f)), 0), std::max(int(std::floor(c.y - rr - 0.5f)), 0),
                           std::max(int(std::floor(c.z - rr - 0.5f)), 0)};
        const int hi[3] = {std::min(int(std::ceil(c.x + rr - 0.5f)), dim[0] - 1), std::min(int(std::ceil(c.y + rr - 0.5f)), dim[1] - 1),
                           std::min(int(std::ceil(c.z + rr - 0.5f)), dim[2] - 1)};
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    const V3<float> d{(float(x) + 0.5f) - c.x, (float(y) + 0.5f) - c.y, (float(z) + 0.5f) - c.z};
                    const V3<float> qv{dot(d, w[0]), dot(d, w[1]), dot(d, w[2])};
                    const float q2 = dot(qv, qv);
                    if (q2 < 1.0f) {
                        float wk = 1.0f - q2;
                        wk = wk * wk * wk;
                        int32_t* a = acc.data() + vox(x, y, z) * 5;
                        add(a[0], int32_t(wk * 1024.0f + 0.5f));
                        add(a[1], to_i32_rn<float>(-d.x * wk * 256.0f));
                        add(a[2], to_i32_rn<float>(-d.y * wk * 256.0f));
                        add(a[3], to_i32_rn<float>(-d.z * wk * 256.0f));
                        add(a[4], to_i32_rn<float>(radius_voxels * wk * 256.0f));
                    }
                }
    }
    // FieldResolveCS
    o.field.assign(nv, 0);
    o.bricks.assign(nb, 0u);
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x) {
                const size_t i = vox(x, y, z);
                const int32_t* a = acc.data() + i * 5;
                const float w = float(a[0]) / 1024.0f;
                float f = 0.0f;
                if (w > 1e-3f) {
                    const float den = 256.0f * w;
                    const V3<float> mo{float(a[1]) / den, float(a[2]) / den, float(a[3]) / den};
                    const float rbar = std::fmax(float(a[4]) / den, 1e-3f);
                    const float phi = std::sqrt(dot(mo, mo)) - rbar;
                    f = saturate(0.5f - 0.5f * phi / rbar);
                }
                o.field[i] = f32_to_f16(f);
                if (f <= 0.0f) continue;
                const int ib[3] = {x & 7, y & 7, z & 7};
                for (int k = 0; k < 8; ++k) {
                    const int ox = (k & 1) * 2 - 1, oy = ((k >> 1) & 1) * 2 - 1, oz = (k >> 2) * 2 - 1;
                    const int nx = x + ox * int(ib[0] == (ox < 0 ? 0 : 7)), ny = y + oy * int(ib[1] == (oy < 0 ? 0 : 7));
                    const int nz = z + oz * int(ib[2] == (oz < 0 ? 0 : 7));
                    if (nx >= 0 && ny >= 0 && nz >= 0 && nx < dim[0] && ny < dim[1] && nz < dim[2]) o.bricks[fbrick(nx, ny, nz)] |= 1u;
                }
            }
    o.positions.clear(); o.normals.clear(); o.tangents.clear(); o.indices.clear();
    o.vertices_requested = o.indices_requested = o.num_vertices = o.num_indices = 0;
    if (!q.build_mesh) return;
    auto fat = [&](int x, int y, int z) { return f16_to_f32(o.field[vox(x, y, z)]); };
    const int cd[3] = {std::max(dim[0] - 1, 0), std::max(dim[1] - 1, 0), std::max(dim[2] - 1, 0)};
    const size_t nc = size_t(cd[0]) * cd[1] * cd[2];
    auto cell_of = [&](int x, int y, int z) { return size_t(x) + size_t(cd[0]) * (size_t(y) + size_t(cd[1]) * size_t(z)); };
    auto corners = [&](int x, int y, int z, float fc[8]) {
        uint32_t mask = 0u;
        for (int k = 0; k < 8; ++k) {
            fc[k] = fat(x + (k & 1), y + ((k >> 1) & 1), z + (k >> 2));
            mask |= (fc[k] >= iso ? 1u : 0u) << k;
        }
        return mask;
    };
    auto sample = [&](float px, float py, float pz) {
        const float x = px - 0.5f, y = py - 0.5f, z = pz - 0.5f;
        const float fx0 = std::floor(x), fy0 = std::floor(y), fz0 = std::floor(z);
        const float tx = x - fx0, ty = y - fy0, tz = z - fz0;
        const int x0 = int(fx0), y0 = int(fy0), z0 = int(fz0);
        const int xs[2] = {clampi(x0, 0, dim[0] - 1), clampi(x0 + 1, 0, dim[0] - 1)};
        const int ys[2] = {clampi(y0, 0, dim[1] - 1), clampi(y0 + 1, 0, dim[1] - 1)};
        const int zs[2] = {clampi(z0, 0, dim[2] - 1), clampi(z0 + 1, 0, dim[2] - 1)};
        float cz[2];
        for (int k = 0; k < 2; ++k) {
            float cy[2];
            for (int j = 0; j < 2; ++j) {
                const float a = fat(xs[0], ys[j], zs[k]), b = fat(xs[1], ys[j], zs[k]);
                cy[j] = a + tx * (b - a);
            }
            cz[k] = cy[0] + ty * (cy[1] - cy[0]);
        }
        return cz[0] + tz * (cz[1] - cz[0]);
    };
    auto normalize_div = [](V3<float> v) {
        const float l = std::sqrt(dot(v, v));
        return V3<float>{v.x / l, v.y / l, v.z / l};
    };
    // SurfaceNetsVerticesCS in cell order
    const uint32_t NO_VERTEX = 0xFFFFFFFFu;
    std::vector<uint32_t> cell_vertex(nc, NO_VERTEX);
    uint32_t next = 0;
    for (int z = 0; z < cd[2]; ++z)
        for (int y = 0; y < cd[1]; ++y)
            for (int x = 0; x < cd[0]; ++x) {
                if (o.bricks[fbrick(x, y, z)] == 0u) continue;
                float fc[8];
                const uint32_t mask = corners(x, y, z, fc);
                if (mask == 0u || mask == 0xFFu) continue;
                const uint32_t vi = next++;
                if (vi >= q.max_vertices) continue;
                cell_vertex[cell_of(x, y, z)] = vi;
                float sx = 0.0f, sy = 0.0f, sz = 0.0f, count = 0.0f;
                for (int a = 0; a < 8; ++a)
                    for (int bit = 1; bit <= 4; bit <<= 1) {
                        if (a & bit) continue;
                        const int b = a | bit;
                        if (((mask >> a) & 1u) == ((mask >> b) & 1u)) continue;
                        const float t = saturate((iso - fc[a]) / (fc[b] - fc[a]));
                        const float px = (a & 1) == (b & 1) ? float(a & 1) : ((b & 1) ? t : 1.0f - t);
                        const float py = ((a >> 1) & 1) == ((b >> 1) & 1) ? float((a >> 1) & 1) : (((b >> 1) & 1) ? t : 1.0f - t);
                        const float pz = (a >> 2) == (b >> 2) ? float(a >> 2) : ((b >> 2) ? t : 1.0f - t);
                        sx = sx + px;
                        sy = sy + py;
                        sz = sz + pz;
                        count = count + 1.0f;
                    }
                const V3<float> pv{(float(x) + 0.5f) + sx / count, (float(y) + 0.5f) + sy / count, (float(z) + 0.5f) + sz / count};
                o.positions.push_back(pv.x * o.voxel);
                o.positions.push_back(pv.y * o.voxel);
                o.positions.push_back(pv.z * o.voxel);
                const V3<float> g{sample(pv.x + 1.0f, pv.y, pv.z) - sample(pv.x - 1.0f, pv.y, pv.z),
                                  sample(pv.x, pv.y + 1.0f, pv.z) - sample(pv.x, pv.y - 1.0f, pv.z),
                                  sample(pv.x, pv.y, pv.z + 1.0f) - sample(pv.x, pv.y, pv.z - 1.0f)};
                V3<float> nrm{0.0f, 0.0f, 1.0f};
                if (std::sqrt(dot(g, g)) > 1e-8f) {
                    const V3<float> ng = normalize_div(g);
                    nrm = V3<float>{-ng.x, -ng.y, -ng.z};
                }
                const V3<float> ref = std::fabs(nrm.z) < 0.9f ? V3<float>{0.0f, 0.0f, 1.0f} : V3<float>{1.0f, 0.0f, 0.0f};
                const V3<float> tx = normalize_div(cross(nrm, ref));
                o.normals.push_back(nrm.x); o.normals.push_back(nrm.y); o.normals.push_back(nrm.z);
                o.tangents.push_back(tx.x); o.tangents.push_back(tx.y); o.tangents.push_back(tx.z);
            }
    o.vertices_requested = next;
    o.num_vertices = std::min(next, q.max_vertices);
    // SurfaceNetsFacesCS in cell order
    uint32_t quads = 0;
    for (int z = 0; z < cd[2]; ++z)
        for (int y = 0; y < cd[1]; ++y)
            for (int x = 0; x < cd[0]; ++x) {
                if (o.bricks[fbrick(x, y, z)] == 0u) continue;
                const bool in0 = fat(x, y, z) >= iso;
                for (int axis = 0; axis < 3; ++axis) {
                    const int e[3] = {axis == 0, axis == 1, axis == 2};
                    const bool in1 = fat(x + e[0], y + e[1], z + e[2]) >= iso;
                    if (in0 == in1) continue;
                    const int eu[3] = {axis == 2, axis == 0, axis == 1}, ev[3] = {axis == 1, axis == 2, axis == 0};
                    const int c11[3] = {x - eu[0] - ev[0], y - eu[1] - ev[1], z - eu[2] - ev[2]};
                    if (c11[0] < 0 || c11[1] < 0 || c11[2] < 0) continue;
                    const uint32_t v00 = cell_vertex[cell_of(x, y, z)], v10 = cell_vertex[cell_of(x - eu[0], y - eu[1], z - eu[2])];
                    const uint32_t v11 = cell_vertex[cell_of(c11[0], c11[1], c11[2])], v01 = cell_vertex[cell_of(x - ev[0], y - ev[1], z - ev[2])];
                    if (v00 == NO_VERTEX || v10 == NO_VERTEX || v11 == NO_VERTEX || v01 == NO_VERTEX) continue;
                    const uint32_t base = 6u * quads++;
                    if (base + 6u > q.max_indices) continue;
                    const uint32_t tri[6] = {v00, in0 ? v11 : v10, in0 ? v10 : v11, v00, in0 ? v01 : v11, in0 ? v11 : v01};
                    for (int k = 0; k < 6; ++k) o.indices.push_back(tri[k]);
                }
            }
    o.indices_requested = 6u * quads;
    const uint32_t ni = std::min(o.indices_requested, q.max_indices);
    o.num_indices = ni - ni % 6u;  // whole quads (only whole quads are written)
    o.indices.resize(o.num_indices);
}

template <class R>
class Sim {
public:
    using Real_ = R;
    slosh_settings_t S{};       // clamped settings of the current layout
    Layout L;
    bool allocated = false;
    PassParams P;

    std::vector<slosh_particle_t> particles, particles_sorted;
    SurfaceOut surface;  // last build_surface
    uint32_t num_particles = 0;
    uint32_t particle_count[4] = {0, 0, 0, 0};
    uint64_t total_emitted = 0, sim_frame = 0;
    uint32_t emit_seed = 1;
    float prev_dt = 0.0f, last_max_speed = 0.0f;

    std::vector<R> vel[3], vel_old, face_weight, pressure, divergence, cell_diag, density_q, density_rhs;
    std::vector<int32_t> accum, cell_count;
    std::vector<uint32_t> face_flags, cell_type;
    std::vector<uint32_t> brick_table, slot_brick, free_slots, brick_touch, brick_want, new_slots, active_bricks;
    std::vector<uint32_t> sort_counts, sort_offsets, sort_perm, sort_keys;
    uint32_t stats[NUM_STATS] = {};
    int32_t coupling[SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE] = {};
    std::vector<slosh_collider_t> colliders;
    std::vector<slosh_manipulator_t> manipulators;

    struct Level {
        I3 dim{0, 0, 0};
        uint32_t cells = 0;
        std::vector<uint32_t> type;
        std::vector<R> x, b;
    };
    std::vector<Level> mg;                 // mg[0] is unused storage-wise (level 0 lives in the pool)
    std::vector<R> pcg_r, pcg_z, pcg_d, pcg_q;
    double scalars[5] = {0, 0, 0, 0, 0};    // rho, scratch, d.Ad, previous rho, r.z_prev (flexible PCG)
    double bb = 0.0, rr = 0.0;              // ||b||^2, ||r||^2 of the current solve
    int32_t last_solve_iterations = 0;
    float last_solve_rel_residual = 0.0f, last_solve_true_rel_residual = 0.0f;
    bool last_solve_converged = true;
    std::vector<double> brick_partials;
    std::vector<uint8_t> extrap_mark;
    int last_disp_index = 2;
    int cur = 0;                            // face-velocity buffer holding the current field
    int substeps = 0;
    float frame_dt_sub = 0.0f;
    bool density_projection_this_frame = false;

    // ---------------------------------------------------------------------------------------
    // Allocate, SloshProxy.cpp:185-306 (particle storage is sized to the capacity up front).
    void allocate(const slosh_settings_t& s) {
        S = s;
        L = make_layout(s);
        const uint32_t cap = s.particle_capacity;
        particles.assign(cap, slosh_particle_t{});
        particles_sorted.assign(cap, slosh_particle_t{});
        num_particles = 0;
        std::fill(particle_count, particle_count + 4, 0u);
        sort_counts.assign(L.num_sort_keys, 0u);
        sort_offsets.assign(L.num_sort_keys, 0u);
        sort_perm.assign(cap, 0u);
        sort_keys.assign(cap, 0u);
        for (int i = 0; i < 3; ++i) vel[i].assign(L.total_faces, R(0));
        vel_old.assign(L.total_faces, R(0));
        accum.assign(size_t(L.total_faces) * 2u, 0);
        face_flags.assign(L.total_faces, 0u);
        face_weight.assign(L.total_faces, R(0));
        cell_type.assign(L.pool_cells, 0u);
        cell_count.assign(L.pool_cells, 0);
        pressure.assign(L.pool_cells, R(0));
        divergence.assign(L.pool_cells, R(0));
        cell_diag.assign(L.pool_cells, R(0));
        density_q.assign(L.pool_cells, R(0));
        density_rhs.assign(L.pool_cells, R(0));
        std::fill(coupling, coupling + SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE, 0);
        std::fill(stats, stats + NUM_STATS, 0u);
        active_bricks.assign(L.num_bricks + 1u, 0u);
        brick_table.assign(L.num_bricks, 0u);
        brick_touch.assign(L.num_bricks, 0u);
        brick_want.assign(L.num_bricks, 0u);
        new_slots.assign(L.num_pool_bricks + 1u, 0u);
        slot_brick.assign(L.num_pool_bricks, NO_BRICK);
        free_slots.assign(L.num_pool_bricks, 0u);
        const uint32_t pool_slots = L.num_pool_bricks - 1u;
        free_slots[0] = pool_slots;  // free stack = [PoolSlots, 1, 2, ..., PoolSlots]
        for (uint32_t slot = 1; slot <= pool_slots; ++slot) free_slots[slot] = slot;
        mg.assign(L.num_levels, Level{});
        for (int l = 0; l < L.num_levels; ++l) {
            mg[l].dim = L.level_dim[l];
            mg[l].cells = L.level_cells[l];
            if (l > 0) {
                mg[l].type.assign(mg[l].cells, 0u);
                mg[l].x.assign(mg[l].cells, R(0));
                mg[l].b.assign(mg[l].cells, R(0));
            }
        }
        pcg_r.assign(L.pool_cells, R(0));
        pcg_z.assign(L.pool_cells, R(0));
        pcg_d.assign(L.pool_cells, R(0));
        pcg_q.assign(L.pool_cells, R(0));
        std::fill(scalars, scalars + 5, 0.0);
        total_emitted = 0;
        prev_dt = 0.0f;
        last_max_speed = 0.0f;
        cur = 0;
        allocated = true;
    }

    // Particle buffers grow to a raised capacity (EnsureParticleCapacity, SloshProxy.cpp:308-337).
    void ensure_capacity(uint32_t cap) {
        if (particles.size() >= cap) return;
        particles.resize(cap);
        particles_sorted.resize(cap);
        sort_perm.resize(cap);
        sort_keys.resize(cap);
    }

    // ---- addressing, Slosh.usf:110-199 ---------------------------------------------------------
    bool in_grid(I3 c) const {
        return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < L.grid.x && c.y < L.grid.y && c.z < L.grid.z;
    }
    uint32_t brick_index_of(I3 b) const {
        return uint32_t(b.x + L.brick_dim.x * (b.y + L.brick_dim.y * b.z));
    }
    I3 brick_coord_of(uint32_t brick) const {
        const uint32_t bx = uint32_t(L.brick_dim.x), by = uint32_t(L.brick_dim.y);
        return {int(brick % bx), int((brick / bx) % by), int(brick / (bx * by))};
    }
    static uint32_t local_index_of(I3 c) {
        return uint32_t((c.x & 7) + 8 * ((c.y & 7) + 8 * (c.z & 7)));
    }
    static I3 local_coord_of(uint32_t l) { return {int(l % 8u), int((l / 8u) % 8u), int(l / 64u)}; }
    uint32_t cell_index(I3 c) const {
        uint32_t slot = 0u;
        if (in_grid(c)) slot = brick_table[brick_index_of({c.x >> 3, c.y >> 3, c.z >> 3})];
        return slot * BRICK_CELLS + local_index_of(c);
    }
    static bool is_null_cell(uint32_t index) { return index < BRICK_CELLS; }
    uint32_t face_index(int axis, I3 f) const { return uint32_t(axis) * L.pool_cells + cell_index(f); }
    uint32_t get_cell_type(I3 c) const { return in_grid(c) ? cell_type[cell_index(c)] : CELL_SOLID; }
    static uint32_t type_of(uint32_t packed) { return packed & CELL_TYPE_MASK; }
    static uint32_t collider_of(uint32_t packed) { return (packed >> CELL_COLLIDER_SHIFT) & 0xFFu; }
    V3<R> face_position(int axis, I3 f) const {  // Slosh.usf:204-208
        V3<R> off{axis == 0 ? R(0) : R(0.5f), axis == 1 ? R(0) : R(0.5f), axis == 2 ? R(0) : R(0.5f)};
        R h = R(P.cell_size);
        return {(R(f.x) + off.x) * h, (R(f.y) + off.y) * h, (R(f.z) + off.z) * h};
    }
    // CellDensity, Slosh.usf:211-224.
    R cell_density(I3 c) const {
        if (!in_grid(c)) return R(0);
        R ws = R(0);
        for (int a = 0; a < 3; ++a) ws = ws + (face_weight[face_index(a, c)] + face_weight[face_index(a, c + axis_offset(a))]);
        return ws / (R(6) * R(P.target_ppc));
    }
    // AirFaceWeight, Slosh.usf:227-230.
    R air_face_weight(R rho_fluid, I3 air_cell) const {
        return P.ghost_fluid != 0u ? R(1) / ghost_theta<R>(rho_fluid, cell_density(air_cell)) : R(1);
    }
    // SolidFaceVelocity, Slosh.usf:232-241 (dot with an axis vector = that component).
    R solid_face_velocity(uint32_t solid_packed, int axis, V3<R> p) const {
        uint32_t id = collider_of(solid_packed);
        if (id == 0u) return R(0);
        V3<R> v = collider_velocity_at<R>(colliders[id - 1u], p);
        V3<R> e{axis == 0 ? R(1) : R(0), axis == 1 ? R(1) : R(0), axis == 2 ? R(1) : R(0)};
        return dot(v, e);
    }
    // CellDensityInterior, Slosh.usf:753-773.
    R cell_density_interior(I3 c) const {
        R ws = R(0), faces = R(0);
        for (int a = 0; a < 3; ++a) {
            I3 e = axis_offset(a);
            if (type_of(get_cell_type(c - e)) != CELL_SOLID) { ws = ws + face_weight[face_index(a, c)]; faces = faces + R(1); }
            if (type_of(get_cell_type(c + e)) != CELL_SOLID) { ws = ws + face_weight[face_index(a, c + e)]; faces = faces + R(1); }
        }
        return faces > R(0) ? ws / (faces * R(P.target_ppc)) : R(1);
    }

    // Visits every allocated cell in active-list order (SparseCell, Slosh.usf:155-188): fn(index, coord).
    template <class Fn> void for_active_cells(Fn fn) {
        const uint32_t active = active_bricks[0];
        #pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < int64_t(active); ++e) {
            const uint32_t brick = active_bricks[1u + uint32_t(e)];
            const uint32_t slot = brick_table[brick];
            const I3 bc = brick_coord_of(brick);
            for (uint32_t l = 0; l < BRICK_CELLS; ++l) {
                I3 lc = local_coord_of(l);
                I3 c{bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z};
                if (!in_grid(c)) continue;
                fn(slot * BRICK_CELLS + l, c);
            }
        }
    }

    // ---- emission, Slosh.usf:264-358 --------------------------------------------------------------
    void emit(const slosh_emit_request_t& em) {
        uint64_t count = em.count;
        if (em.shape == SLOSH_EMIT_FILL_CELLS)
            count = uint64_t(std::max(em.cell_dims[0], 0)) * uint64_t(std::max(em.cell_dims[1], 0)) *
                    uint64_t(std::max(em.cell_dims[2], 0)) * 8ull;
        const uint32_t cap = S.particle_capacity;
        count = std::min<uint64_t>(count, uint64_t(cap) - std::min(num_particles, cap));
        if (count == 0) return;
        const uint32_t bound = num_particles;
        // EmitReserveCS
        const uint32_t base = particle_count[0];
        particle_count[1] = base;
        particle_count[0] = base + uint32_t(count);
        const uint32_t seed = emit_seed++;
        const float h = S.cell_size, inv_h = 1.0f / h;
        const float jitter = em.fill_jitter;
        for (uint32_t i = 0; i < uint32_t(count); ++i) {
            const uint32_t fill = bound + i;
            if (fill >= base + uint32_t(count) && fill < cap) particles[fill] = dead_particle();
            const uint32_t h0 = pcg_hash(i * 3u + seed * 7919u);
            const uint32_t h1 = pcg_hash(h0);
            const uint32_t h2 = pcg_hash(h1);
            V3<float> rnd{hash_to_unit(h0), hash_to_unit(h1), hash_to_unit(h2)};
            V3<float> p;
            if (em.shape == SLOSH_EMIT_FILL_CELLS) {
                const uint32_t cell_linear = i / 8u, sub = i % 8u;
                I3 local{int(cell_linear % uint32_t(em.cell_dims[0])),
                         int((cell_linear / uint32_t(em.cell_dims[0])) % uint32_t(em.cell_dims[1])),
                         int(cell_linear / uint32_t(em.cell_dims[0] * em.cell_dims[1]))};
                V3<float> so{float(sub & 1u), float((sub >> 1u) & 1u), float((sub >> 2u) & 1u)};
                for (int a = 0; a < 3; ++a) {
                    float in_cell = ((so[a] + 0.5f) + jitter * (rnd[a] - 0.5f)) * 0.5f;
                    p[a] = (float(em.cell_min[a] + local[a]) + in_cell) * h;
                }
            } else if (em.shape == SLOSH_EMIT_SPHERE) {
                const uint32_t h3 = pcg_hash(h2);
                float cos_t = 2.0f * rnd.x - 1.0f;
                float sin_t = std::sqrt(saturate(1.0f - cos_t * cos_t));
                float phi = 6.28318530718f * rnd.y;
                float r = em.extent[0] * pow_r(std::fmax(hash_to_unit(h3), 1e-6f), 1.0f / 3.0f);
                V3<float> dir{sin_t * cos_r(phi), sin_t * sin_r(phi), cos_t};
                p = V3<float>{em.center[0], em.center[1], em.center[2]} + r * dir;
            } else {
                V3<float> q{(2.0f * rnd.x - 1.0f) * em.extent[0], (2.0f * rnd.y - 1.0f) * em.extent[1],
                            (2.0f * rnd.z - 1.0f) * em.extent[2]};
                p = V3<float>{em.center[0], em.center[1], em.center[2]} + quat_rotate<float>(em.rotation, q);
            }
            V3<float> lo{h * 1.01f, h * 1.01f, h * 1.01f};
            V3<float> hi{(float(L.grid.x) - 1.01f) * h, (float(L.grid.y) - 1.01f) * h, (float(L.grid.z) - 1.01f) * h};
            V3<float> velocity{em.velocity[0], em.velocity[1], em.velocity[2]};
            float speed = length(velocity);
            if (speed > 1e-6f && (em.velocity_spread > 0.0f || em.speed_jitter > 0.0f)) {
                const uint32_t h4 = pcg_hash(h2 ^ 0x9E3779B9u), h5 = pcg_hash(h4), h6 = pcg_hash(h5);
                V3<float> dir{velocity.x / speed, velocity.y / speed, velocity.z / speed};
                V3<float> ref = std::fabs(dir.z) < 0.9f ? V3<float>{0, 0, 1} : V3<float>{1, 0, 0};
                V3<float> t0 = cross(dir, ref);
                float t0l = length(t0);
                t0 = V3<float>{t0.x / t0l, t0.y / t0l, t0.z / t0l};
                V3<float> t1 = cross(dir, t0);
                float cos_a = 1.0f + hash_to_unit(h4) * (cos_r(em.velocity_spread) - 1.0f);
                float sin_a = std::sqrt(saturate(1.0f - cos_a * cos_a));
                float phi = 6.28318530718f * hash_to_unit(h5);
                dir = cos_a * dir + sin_a * (cos_r(phi) * t0 + sin_r(phi) * t1);
                velocity = dir * speed * std::fmax(1.0f + em.speed_jitter * (2.0f * hash_to_unit(h6) - 1.0f), 0.0f);
            }
            ParticleU<float> part;
            part.pos = {clampr(p.x, lo.x, hi.x), clampr(p.y, lo.y, hi.y), clampr(p.z, lo.z, hi.z)};
            part.vel = velocity;
            part.cx = {0, 0, 0}; part.cy = {0, 0, 0}; part.cz = {0, 0, 0};
            part.age = 0.0f;
            particles[base + i] = pack_particle(part);
            I3 c{clampi(int(std::floor(part.pos.x * inv_h)), 0, L.grid.x - 1),
                 clampi(int(std::floor(part.pos.y * inv_h)), 0, L.grid.y - 1),
                 clampi(int(std::floor(part.pos.z * inv_h)), 0, L.grid.z - 1)};
            brick_touch[brick_index_of({c.x >> 3, c.y >> 3, c.z >> 3})] = 1u;
        }
        total_emitted += count;
        num_particles += uint32_t(count);
    }

    // Uploaded particles (no reference counterpart): slots [0, n) become the particle buffer; their
    // bricks are touched like EmitParticlesCS touches them (Slosh.usf:357).
    void upload(const slosh_particle_t* src, uint32_t n) {
        std::copy(src, src + n, particles.begin());
        num_particles = n;
        particle_count[0] = n;
        particle_count[1] = 0;
        const float inv_h = 1.0f / S.cell_size;
        for (uint32_t i = 0; i < n; ++i) {
            const slosh_particle_t& p = particles[i];
            if (is_dead_age(p.age)) continue;
            I3 c{clampi(int(std::floor(p.pos[0] * inv_h)), 0, L.grid.x - 1),
                 clampi(int(std::floor(p.pos[1] * inv_h)), 0, L.grid.y - 1),
                 clampi(int(std::floor(p.pos[2] * inv_h)), 0, L.grid.z - 1)};
            brick_touch[brick_index_of({c.x >> 3, c.y >> 3, c.z >> 3})] = 1u;
        }
    }

    // ---- counting sort, SloshSort.usf:36-154 and AddSpatialSort, SloshProxy.cpp:1022-1087 --------------
    uint32_t sort_key_of(const slosh_particle_t& p) const {
        if (is_dead_age(p.age)) return L.num_sort_keys - 1u;
        const float inv_h = 1.0f / S.cell_size;
        I3 c{clampi(int(std::floor(p.pos[0] * inv_h)), 0, L.grid.x - 1),
             clampi(int(std::floor(p.pos[1] * inv_h)), 0, L.grid.y - 1),
             clampi(int(std::floor(p.pos[2] * inv_h)), 0, L.grid.z - 1)};
        I3 b{c.x >> 2, c.y >> 2, c.z >> 2};
        return std::min(uint32_t(b.x + L.sort_brick_dim.x * (b.y + L.sort_brick_dim.y * b.z)), L.num_sort_keys - 2u);
    }
    void sort_particles() {
        const uint32_t n = num_particles;
        std::fill(sort_counts.begin(), sort_counts.end(), 0u);
        std::vector<uint32_t> rank(n);
        for (uint32_t i = 0; i < n; ++i) {            // SortCountCS in ascending thread order
            const uint32_t key = sort_key_of(particles[i]);
            sort_keys[i] = key;
            rank[i] = sort_counts[key]++;
        }
        uint32_t run = 0;                             // SortScanBlocksCS + SortScanBlockSumsCS
        for (uint32_t k = 0; k < L.num_sort_keys; ++k) { sort_offsets[k] = run; run += sort_counts[k]; }
        for (uint32_t i = 0; i < n; ++i) {            // SortScatterCS
            const uint32_t dst = sort_offsets[sort_keys[i]] + rank[i];
            particles_sorted[dst] = particles[i];
            sort_perm[dst] = i;
        }
        particle_count[0] = sort_offsets[L.num_sort_keys - 1u];  // SortWriteCountCS
        std::swap(particles, particles_sorted);        // SloshProxy.cpp:1085
    }

    // ---- brick pool, Slosh.usf:1719-1831 -------------------------------------------------------------
    void brick_free() {  // BrickFreeCS
        active_bricks[0] = 0u;
        new_slots[0] = 0u;
        for (uint32_t brick = 0; brick < L.num_bricks; ++brick) {
            I3 b = brick_coord_of(brick);
            bool wanted = false;
            for (int z = -1; z <= 1; ++z)
                for (int y = -1; y <= 1; ++y)
                    for (int x = -1; x <= 1; ++x) {
                        I3 nb{b.x + x, b.y + y, b.z + z};
                        if (nb.x >= 0 && nb.y >= 0 && nb.z >= 0 && nb.x < L.brick_dim.x && nb.y < L.brick_dim.y &&
                            nb.z < L.brick_dim.z)
                            wanted = wanted || brick_touch[brick_index_of(nb)] != 0u;
                    }
            brick_want[brick] = wanted ? 1u : 0u;
            const uint32_t slot = brick_table[brick];
            if (!wanted && slot != 0u) {
                brick_table[brick] = 0u;
                slot_brick[slot] = NO_BRICK;
                const uint32_t count = free_slots[0]++;
                free_slots[1u + count] = slot;
            }
        }
    }
    void brick_alloc() {  // BrickAllocCS
        for (uint32_t brick = 0; brick < L.num_bricks; ++brick) {
            brick_touch[brick] = 0u;
            if (brick_want[brick] == 0u) continue;
            uint32_t slot = brick_table[brick];
            if (slot == 0u) {
                const uint32_t count = free_slots[0];
                free_slots[0] = count - 1u;
                if (int32_t(count) <= 0) { stats[8] += 1u; continue; }
                slot = free_slots[count];
                brick_table[brick] = slot;
                slot_brick[slot] = brick;
                const uint32_t entry = new_slots[0]++;
                new_slots[1u + entry] = slot;
            }
            const uint32_t entry = active_bricks[0]++;
            active_bricks[1u + entry] = brick;
        }
    }
    void pool_args() {  // PoolArgsCS
        if (int32_t(free_slots[0]) < 0) free_slots[0] = 0u;
        stats[7] = std::max(stats[7], active_bricks[0]);
    }
    void clear_new_slots() {  // ClearNewSlotsCS
        for (uint32_t e = 0; e < new_slots[0]; ++e) {
            const uint32_t base = new_slots[1u + e] * BRICK_CELLS;
            for (uint32_t l = 0; l < BRICK_CELLS; ++l) {
                pressure[base + l] = R(0);
                cell_count[base + l] = 0;
                density_q[base + l] = R(0);
            }
        }
    }

    // ---- BuildSolidCS, Slosh.usf:365-395 -----------------------------------------------------------
    void build_solid() {
        for_active_cells([&](uint32_t index, I3 c) {
            uint32_t packed = CELL_AIR;
            if (c.x == 0 || c.y == 0 || c.z == 0 || c.x == L.grid.x - 1 || c.y == L.grid.y - 1 || c.z == L.grid.z - 1) {
                packed = CELL_SOLID;
            } else {
                const float h = P.cell_size;
                V3<float> p{(float(c.x) + 0.5f) * h, (float(c.y) + 0.5f) * h, (float(c.z) + 0.5f) * h};
                float best = 0.0f;
                for (uint32_t k = 0; k < P.num_colliders; ++k) {
                    float d = collider_sdf<float>(colliders[k], p);
                    if (d < best) { best = d; packed = CELL_SOLID | ((k + 1u) << CELL_COLLIDER_SHIFT); }
                }
            }
            cell_type[index] = packed;
        });
    }

    // ---- P2GCS, Slosh.usf:401-563: fixed-point sums are order independent -------------------------------
    // P2GCS (Slosh.usf:448-563): per MAC component the 8 stencil nodes receive w (u_p + C_p . (x_n - x_p)) and w
    // in 2^20 fixed point. The per-node terms are formed from per-axis factors: with S = 2^20,
    // wS = w_x ((w_y w_z) S) and the affine term (u_p + C_x dx) + (C_y dy + C_z dz), then
    // mom = rn(wS term) and weight = rn(wS). Mathematically the reference's w (u + dot(C, x_n - x_p)) S and
    // w S; the GPU rounds in the same order.
    void p2g() {
        const R inv_h = R(P.inv_cell_size), h = R(P.cell_size);
        const R scale = R(P2G_FIXED_SCALE);
        const uint32_t tf = L.total_faces;
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < int64_t(num_particles); ++ii) {
            const slosh_particle_t& sp = particles[size_t(ii)];
            if (is_dead_age(sp.age)) continue;
            ParticleU<R> p = unpack_particle<R>(sp);
            I3 cell{clampi(int(std::floor(p.pos.x * inv_h)), 0, L.grid.x - 1),
                    clampi(int(std::floor(p.pos.y * inv_h)), 0, L.grid.y - 1),
                    clampi(int(std::floor(p.pos.z * inv_h)), 0, L.grid.z - 1)};
            V3<R> cs[3] = {p.cx, p.cy, p.cz};
            for (int axis = 0; axis < 3; ++axis) {
                V3<R> cp = P.use_apic ? cs[axis] : V3<R>{R(0), R(0), R(0)};
                R up = p.vel[axis];
                V3<R> off{axis == 0 ? R(0) : R(0.5f), axis == 1 ? R(0) : R(0.5f), axis == 2 ? R(0) : R(0.5f)};
                V3<R> g{p.pos.x * inv_h - off.x, p.pos.y * inv_h - off.y, p.pos.z * inv_h - off.z};
                I3 base{int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z))};
                V3<R> fr{g.x - R(base.x), g.y - R(base.y), g.z - R(base.z)};
                for (uint32_t o = 0; o < 8u; ++o) {
                    I3 oi{int(o & 1u), int((o >> 1u) & 1u), int((o >> 2u) & 1u)};
                    I3 node = base + oi;
                    if (!in_grid(node)) continue;
                    V3<R> w3{oi.x ? fr.x : R(1) - fr.x, oi.y ? fr.y : R(1) - fr.y, oi.z ? fr.z : R(1) - fr.z};
                    R ws = w3.x * ((w3.y * w3.z) * scale);
                    if (ws <= R(0)) continue;
                    V3<R> xn{(R(node.x) + off.x) * h, (R(node.y) + off.y) * h, (R(node.z) + off.z) * h};
                    V3<R> dx = xn - p.pos;
                    R term = (up + cp.x * dx.x) + (cp.y * dx.y + cp.z * dx.z);
                    int32_t mom = to_i32_rn<R>(ws * term);
                    int32_t wt = to_i32_rn<R>(ws);
                    uint32_t cidx = cell_index(node);
                    if (is_null_cell(cidx)) continue;
                    uint32_t f = uint32_t(axis) * L.pool_cells + cidx;
                    uint32_t* am = reinterpret_cast<uint32_t*>(&accum[f]);
                    uint32_t* aw = reinterpret_cast<uint32_t*>(&accum[tf + f]);
                    #pragma omp atomic
                    *am += uint32_t(mom);
                    #pragma omp atomic
                    *aw += uint32_t(wt);
                }
            }
            uint32_t ci = cell_index(cell);
            if (!is_null_cell(ci)) {
                #pragma omp atomic
                cell_count[ci] += 1;
            }
        }
    }

    // ---- MarkCellsCS, Slosh.usf:569-598 ------------------------------------------------------------
    void mark_cells() {
        uint32_t fluid = 0;
        for_active_cells([&](uint32_t index, I3) {
            uint32_t packed = cell_type[index];
            if (type_of(packed) != CELL_SOLID) {
                int32_t count = cell_count[index];
                packed = count > 0 ? CELL_FLUID : CELL_AIR;
                if (float(count) >= 0.5f * P.target_ppc) packed |= CELL_DENSE_FLAG;
                cell_type[index] = packed;
            }
            if (type_of(packed) == CELL_FLUID) {
                pressure[index] = pressure[index] * R(P.warm_start_scale);
                #pragma omp atomic
                fluid += 1u;
            } else {
                pressure[index] = R(0);
            }
        });
        stats[1] += fluid;
    }

    // ---- NormalizeFace, Slosh.usf:604-651 --------------------------------------------------------------
    void normalize_faces() {
        const uint32_t tf = L.total_faces;
        std::vector<R>& v = vel[0];
        for_active_cells([&](uint32_t index, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const uint32_t f = uint32_t(axis) * L.pool_cells + index;
                int32_t mom = accum[f], wt = accum[tf + f];
                if (mom != 0 || wt != 0) { accum[f] = 0; accum[tf + f] = 0; }
                R u = wt > 0 ? R(mom) / R(wt) : R(0);
                face_weight[f] = R(float(wt) * P2G_FIXED_INV);
                uint32_t flags = wt > 0 ? FACE_HAS_WEIGHT : 0u;
                if (P.use_apic == 0u) vel_old[f] = u;
                uint32_t a = get_cell_type(c - axis_offset(axis));
                uint32_t b = get_cell_type(c);
                if (type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID) {
                    uint32_t solid = type_of(b) == CELL_SOLID ? b : a;
                    u = solid_face_velocity(solid, axis, face_position(axis, c));
                } else if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                    uint32_t solid = type_of(b) == CELL_SOLID ? b : a;
                    u = solid_face_velocity(solid, axis, face_position(axis, c));
                    flags |= FACE_VALID | FACE_SOLID;
                } else if (type_of(a) == CELL_FLUID || type_of(b) == CELL_FLUID) {
                    u = u + R(P.gravity[axis]) * R(P.dt);
                    flags |= FACE_VALID;
                } else {
                    u = R(0);
                }
                v[f] = u;
                face_flags[f] = flags;
            }
        });
    }

    // ---- ViscosityJacobiFace, Slosh.usf:657-686 (Vel = u*, src -> dst) ----------------------------------
    void viscosity_jacobi(const std::vector<R>& ustar, const std::vector<R>& src, std::vector<R>& dst) {
        const R alpha = R(P.viscosity_alpha);
        for_active_cells([&](uint32_t index, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const uint32_t f = uint32_t(axis) * L.pool_cells + index;
                uint32_t flags = face_flags[f];
                R center = src[f];
                if ((flags & FACE_VALID) == 0u || (flags & FACE_SOLID) != 0u) { dst[f] = center; continue; }
                R sum = R(0);
                for (int n = 0; n < 6; ++n) {
                    I3 nb = c + neighbour_offset(n);
                    R value = center;
                    if (in_grid(nb)) {
                        uint32_t ni = face_index(axis, nb);
                        if ((face_flags[ni] & FACE_VALID) != 0u) value = src[ni];
                    }
                    sum = sum + value;
                }
                dst[f] = (ustar[f] + alpha * sum) / (R(1) + R(6) * alpha);
            }
        });
    }

    // ---- DivergenceCS, Slosh.usf:692-741 ---------------------------------------------------------------
    void divergence_pass(const std::vector<R>& v) {
        for_active_cells([&](uint32_t index, I3 c) {
            cell_count[index] = 0;
            if (type_of(cell_type[index]) != CELL_FLUID) { divergence[index] = R(0); cell_diag[index] = R(0); return; }
            R div = R(0);
            for (int a = 0; a < 3; ++a) div = div + (v[face_index(a, c + axis_offset(a))] - v[face_index(a, c)]);
            R ws = R(0);
            for (int a = 0; a < 3; ++a) ws = ws + (face_weight[face_index(a, c)] + face_weight[face_index(a, c + axis_offset(a))]);
            R rho = ws / (R(6) * R(P.target_ppc));
            R excess = std::fmax(rho - (R(1) + R(P.density_deadband)), R(0));
            R target = std::fmin(R(P.density_correction) * excess, R(0.5f)) * R(P.cell_size) / R(P.dt);
            divergence[index] = div - target;
            R diag = R(0);
            for (int n = 0; n < 6; ++n) {
                I3 nb = c + neighbour_offset(n);
                uint32_t nt = type_of(get_cell_type(nb));
                diag = diag + (nt == CELL_FLUID ? R(1) : (nt == CELL_AIR ? air_face_weight(rho, nb) : R(0)));
            }
            cell_diag[index] = diag;
        });
    }

    // ---- PressureRBGSCS, Slosh.usf:860-892 ------------------------------------------------------------
    void rbgs_sweep(std::vector<R>& p, const std::vector<R>& rhs, uint32_t parity, float sor_weight) {
        for_active_cells([&](uint32_t index, I3 c) {
            if (type_of(cell_type[index]) != CELL_FLUID) return;
            if ((uint32_t(c.x + c.y + c.z) & 1u) != parity) return;
            R sum = R(0);
            R diag = cell_diag[index];
            for (int n = 0; n < 6; ++n) {
                I3 nb = c + neighbour_offset(n);
                if (type_of(get_cell_type(nb)) == CELL_FLUID) sum = sum + p[cell_index(nb)];
            }
            if (diag > R(0)) {
                R gs = (sum - rhs[index]) / diag;
                R old = p[index];
                p[index] = old + R(sor_weight) * (gs - old);
            }
        });
    }

    // ---- MGPCG, SloshPressureMG.usf:58-543 with the driver of SloshProxy.cpp:807-1020 -------------------------
    static constexpr float DIAG_EPSILON = 1e-4f;  // SloshProxy.cpp:845
    static uint32_t lin(I3 c, I3 d) { return uint32_t(c.x + d.x * (c.y + d.y * c.z)); }
    static I3 coord(uint32_t i, I3 d) {
        return {int(i % uint32_t(d.x)), int((i / uint32_t(d.x)) % uint32_t(d.y)), int(i / uint32_t(d.x * d.y))};
    }
    static bool inside(I3 c, I3 d) { return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < d.x && c.y < d.y && c.z < d.z; }
    static bool is_red(I3 c) { return (uint32_t(c.x + c.y + c.z) & 1u) == 0u; }

    // Level l index of a cell (FineIndex: pooled on level 0, dense above).
    uint32_t level_index(int l, I3 c) const { return l == 0 ? cell_index(c) : lin(c, mg[l].dim); }
    uint32_t level_type_raw(int l, uint32_t i) const { return l == 0 ? cell_type[i] : mg[l].type[i]; }
    uint32_t level_type_at(int l, I3 c) const {  // FineTypeAt / CoarseTypeAt
        return inside(c, mg[l].dim) ? (level_type_raw(l, level_index(l, c)) & CELL_TYPE_MASK) : CELL_SOLID;
    }
    // FINE_STENCIL, SloshPressureMG.usf:142-157.
    void stencil(int l, const std::vector<R>& buf, I3 c, uint32_t i, const std::vector<R>* diag_f, R& out_diag, R& out_sum) const {
        out_diag = R(DIAG_EPSILON);
        out_sum = R(0);
        for (int n = 0; n < 6; ++n) {
            I3 nb = c + neighbour_offset(n);
            if (!inside(nb, mg[l].dim)) continue;
            uint32_t ni = level_index(l, nb);
            uint32_t t = level_type_raw(l, ni) & CELL_TYPE_MASK;
            if (t != CELL_SOLID) out_diag = out_diag + R(1);
            if (t == CELL_FLUID) out_sum = out_sum + buf[ni];
        }
        if (l == 0) out_diag = (*diag_f)[i] + R(DIAG_EPSILON);
    }
    // Storage precision of the coarse levels (precision_mode): every store to a level >= 1 rounds to it.
    R store_q(int l, R v) const {
        if (l == 0) return v;
        if (P.precision_mode == SLOSH_PRECISION_FP16_STORAGE) return R(f16_to_f32(f32_to_f16(float(v))));
        if (P.precision_mode == SLOSH_PRECISION_BF16_STORAGE) return R(bf16_to_f32(f32_to_bf16(float(v))));
        return v;
    }
    std::vector<R>& level_x(int l) { return l == 0 ? pcg_z : mg[l].x; }
    std::vector<R>& level_b(int l) { return l == 0 ? pcg_r : mg[l].b; }

    // Level-0 visit with one canonical FP64 partial per active brick (entry order).
    template <class Fn> double level0_dot(Fn fn) {
        const uint32_t active = active_bricks[0];
        brick_partials.assign(active, 0.0);
        #pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < int64_t(active); ++e) {
            double vals[BRICK_CELLS];
            const uint32_t brick = active_bricks[1u + uint32_t(e)];
            const uint32_t slot = brick_table[brick];
            const I3 bc = brick_coord_of(brick);
            for (uint32_t l = 0; l < BRICK_CELLS; ++l) {
                I3 lc = local_coord_of(l);
                I3 c{bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z};
                vals[l] = in_grid(c) ? fn(slot * BRICK_CELLS + l, c) : 0.0;
            }
            brick_partials[size_t(e)] = reduce_brick(vals);
        }
        return reduce_final(brick_partials.data(), active);
    }

    void mg_build_type(int l) {  // MGBuildTypeCS: level l -> l + 1
        Level& cl = mg[l + 1];
        #pragma omp parallel for schedule(static)
        for (int64_t ci = 0; ci < int64_t(cl.cells); ++ci) {
            I3 c = coord(uint32_t(ci), cl.dim);
            bool any_air = false, any_fluid = false;
            for (uint32_t o = 0; o < 8u; ++o) {
                I3 f{c.x * 2 + int(o & 1u), c.y * 2 + int((o >> 1u) & 1u), c.z * 2 + int((o >> 2u) & 1u)};
                if (inside(f, mg[l].dim)) {
                    uint32_t t = level_type_at(l, f);
                    any_air = any_air || t == CELL_AIR;
                    any_fluid = any_fluid || t == CELL_FLUID;
                }
            }
            cl.type[size_t(ci)] = any_air ? CELL_AIR : (any_fluid ? CELL_FLUID : CELL_SOLID);
        }
    }

    // MGSmoothCS on level l; with dot, returns B.X over the level-0 fluid cells (canonical tree).
    double mg_smooth(int l, uint32_t parity, bool dot) {
        std::vector<R>& xf = level_x(l);
        std::vector<R>& bf = level_b(l);
        auto cell = [&](uint32_t i, I3 c) -> double {
            double dv = 0.0;
            if ((level_type_raw(l, i) & CELL_TYPE_MASK) == CELL_FLUID) {
                if ((is_red(c) ? 0u : 1u) == parity) {
                    R diag, sum;
                    stencil(l, xf, c, i, &cell_diag, diag, sum);
                    R b = bf[i];
                    const R gs = (b + sum) / diag;
                    // level 0 over-relaxed by mg_smoother_weight: x + w (x_GS - x); 1 = the reference
                    R x = store_q(l, (l == 0 && P.smooth_weight != 1.0f) ? xf[i] + R(P.smooth_weight) * (gs - xf[i]) : gs);
                    xf[i] = x;
                    dv = double(b * x);
                } else if (dot) {
                    dv = double(bf[i] * xf[i]);
                }
            }
            return dv;
        };
        if (l == 0) {
            if (dot) return level0_dot(cell);
            for_active_cells([&](uint32_t i, I3 c) { cell(i, c); });
            return 0.0;
        }
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < int64_t(mg[l].cells); ++i) cell(uint32_t(i), coord(uint32_t(i), mg[l].dim));
        return 0.0;
    }

    // Scale of the coarse levels with 16-bit storage (1 with FP32): a power of two bringing the level-0
    // residual's norm (rr when the V-cycle starts) to about 1, applied by the restriction from level 0 and
    // undone by the prolongation to level 0.
    R coarse_scale() const {
        if (P.precision_mode == SLOSH_PRECISION_FP32) return R(1);
        int e = rr > 0.0 ? -std::ilogb(std::sqrt(rr)) : 0;
        e = std::max(-60, std::min(60, e));
        return R(std::ldexp(1.0f, e));
    }
    void mg_restrict(int l) {  // MGRestrictCS: level l -> l + 1
        std::vector<R>& xf = level_x(l);
        std::vector<R>& bf = level_b(l);
        Level& cl = mg[l + 1];
        auto coarse = [&](uint32_t ci) {
            I3 c = coord(ci, cl.dim);
            if ((cl.type[ci] & CELL_TYPE_MASK) != CELL_FLUID) { cl.b[ci] = R(0); cl.x[ci] = R(0); return; }
            R sum = R(0);
            for (uint32_t o = 0; o < 8u; ++o) {
                I3 f{c.x * 2 + int(o & 1u), c.y * 2 + int((o >> 1u) & 1u), c.z * 2 + int((o >> 2u) & 1u)};
                if (inside(f, mg[l].dim) && level_type_at(l, f) == CELL_FLUID) {
                    uint32_t fi = level_index(l, f);
                    R diag, nbsum;
                    stencil(l, xf, f, fi, &cell_diag, diag, nbsum);
                    sum = sum + (bf[fi] - (diag * xf[fi] - nbsum));
                }
            }
            R b = R(P.restrict_scale) * sum;
            if (l == 0) b = b * coarse_scale();
            cl.b[ci] = store_q(l + 1, b);
            R cdiag = R(DIAG_EPSILON);
            for (int n = 0; n < 6; ++n) {
                I3 nb = c + neighbour_offset(n);
                uint32_t t = inside(nb, cl.dim) ? (cl.type[lin(nb, cl.dim)] & CELL_TYPE_MASK) : CELL_SOLID;
                cdiag = cdiag + (t != CELL_SOLID ? R(1) : R(0));
            }
            cl.x[ci] = store_q(l + 1, is_red(c) ? b / cdiag : R(0));
        };
        if (l == 0) {
            // SparseCoarse: the 4^3 level-1 cells of every active brick.
            const uint32_t active = active_bricks[0];
            #pragma omp parallel for schedule(static)
            for (int64_t e = 0; e < int64_t(active); ++e) {
                I3 bc = brick_coord_of(active_bricks[1u + uint32_t(e)]);
                for (uint32_t lc = 0; lc < 64u; ++lc) {
                    I3 c{bc.x * 4 + int(lc % 4u), bc.y * 4 + int((lc / 4u) % 4u), bc.z * 4 + int(lc / 16u)};
                    if (!inside(c, cl.dim)) continue;
                    coarse(lin(c, cl.dim));
                }
            }
        } else {
            #pragma omp parallel for schedule(static)
            for (int64_t ci = 0; ci < int64_t(cl.cells); ++ci) coarse(uint32_t(ci));
        }
    }

    void mg_coarse_solve(int l, int iterations) {  // MGCoarseSolveCS
        std::vector<R>& xf = level_x(l);
        std::vector<R>& bf = level_b(l);
        const uint32_t cells = mg[l].cells;
        for (int it = 0; it < iterations; ++it)
            for (uint32_t colour = 0; colour < 2u; ++colour)
                for (uint32_t lin_i = 0; lin_i < cells; ++lin_i) {
                    I3 c = coord(lin_i, mg[l].dim);
                    uint32_t i = level_index(l, c);
                    if ((level_type_raw(l, i) & CELL_TYPE_MASK) == CELL_FLUID && (is_red(c) ? 0u : 1u) == colour) {
                        R diag, sum;
                        stencil(l, xf, c, i, &cell_diag, diag, sum);
                        xf[i] = store_q(l, (bf[i] + sum) / diag);
                    }
                }
    }

    void mg_prolong(int l) {  // MGProlongCS: level l + 1 -> l
        std::vector<R>& xf = level_x(l);
        Level& cl = mg[l + 1];
        const R inv_scale = R(1) / coarse_scale();
        auto fine = [&](uint32_t i, I3 c) {
            if ((level_type_raw(l, i) & CELL_TYPE_MASK) != CELL_FLUID) return;
            I3 parent{c.x / 2, c.y / 2, c.z / 2};
            uint32_t pi = lin(parent, cl.dim);
            if ((cl.type[pi] & CELL_TYPE_MASK) == CELL_FLUID) xf[i] = store_q(l, xf[i] + (l == 0 ? cl.x[pi] * inv_scale : cl.x[pi]));
        };
        if (l == 0) {
            for_active_cells(fine);
        } else {
            #pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < int64_t(mg[l].cells); ++i) fine(uint32_t(i), coord(uint32_t(i), mg[l].dim));
        }
    }

    // VCycle, SloshProxy.cpp:904-959. Returns rho = r.z. Every level above the coarsest is pre-smoothed
    // by P.mg_sweeps red-black pairs (the first red half is the red initialisation its producer wrote)
    // and post-smoothed by P.mg_sweeps black-red pairs; the reference is one pair.
    double vcycle(int coarse_iterations) {
        const int nl = L.num_levels;
        if (nl == 1) {
            mg_coarse_solve(0, coarse_iterations);
            return mg_smooth(0, 0u, true);
        }
        const int sweeps = P.mg_sweeps;
        auto pre_smooth = [&](int l) {
            mg_smooth(l, 1u, false);
            for (int k = 1; k < sweeps; ++k) {
                mg_smooth(l, 0u, false);
                mg_smooth(l, 1u, false);
            }
        };
        pre_smooth(0);
        for (int l = 0; l < nl - 1; ++l) {
            mg_restrict(l);
            if (l + 1 < nl - 1) pre_smooth(l + 1);
        }
        mg_coarse_solve(nl - 1, coarse_iterations);
        double rho = 0.0;
        for (int l = nl - 2; l >= 0; --l) {
            mg_prolong(l);
            for (int k = 0; k < sweeps; ++k) {
                mg_smooth(l, 1u, false);
                const bool last = k == sweeps - 1;
                double d = mg_smooth(l, 0u, l == 0 && last);
                if (l == 0 && last) rho = d;
            }
        }
        return rho;
    }

    // The preconditioner's red initialisation of level 0 (one red half-sweep from zero): w (r / diag) with the
    // smoother weight w, r / diag for the reference.
    R red_init(R v) const { return P.smooth_weight != 1.0f ? R(P.smooth_weight) * v : v; }

    static float ratio_f(double num, double den) {  // alpha / beta: FP64 ratio rounded to FP32
        return std::fabs(den) > 1e-30 ? float(num / den) : 0.0f;
    }

    // AddPressureSolveMGPCG. p: solution (warm start), div: the Divergence buffer (b = -div).
    // fixed_iterations > 0 runs that many iterations (reference); otherwise tolerance mode.
    int mgpcg(std::vector<R>& p, const std::vector<R>& div, int fixed_iterations, float tolerance, int max_iterations,
              int coarse_iterations) {
        const int nl = L.num_levels;
        for (int l = 0; l < nl - 1; ++l) mg_build_type(l);
        // PCGInitCS (+ ||b||^2, an extension for the relative residual)
        double bb_local = 0.0;
        double r0 = level0_dot([&](uint32_t i, I3 c) -> double {
            if (type_of(cell_type[i]) != CELL_FLUID) { pcg_r[i] = R(0); pcg_z[i] = R(0); pcg_d[i] = R(0); return 0.0; }
            R diag, sum;
            stencil(0, p, c, i, &cell_diag, diag, sum);
            R ri = -div[i] - (diag * p[i] - sum);
            pcg_r[i] = ri;
            pcg_z[i] = is_red(c) ? red_init(ri / diag) : R(0);
            return double(ri * ri);
        });
        bb_local = level0_dot([&](uint32_t i, I3) -> double {
            if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
            R b = -div[i];
            return double(b * b);
        });
        bb = bb_local;
        rr = r0;
        const bool tol_mode = fixed_iterations <= 0;
        const int iterations = tol_mode ? std::max(max_iterations, 1) : std::min(std::max(fixed_iterations, 1), 100);
        auto rel = [&]() { return bb > 0.0 ? std::sqrt(rr / bb) : 0.0; };
        if (tol_mode && rel() <= double(tolerance)) {
            last_solve_iterations = 0;
            last_solve_rel_residual = float(rel());
            last_solve_converged = true;
            return 0;
        }
        double rho = vcycle(coarse_iterations);
        scalars[3] = scalars[0];
        scalars[0] = rho;
        update_d(true);
        int done = 0;
        for (int it = 0; it < iterations; ++it) {
            // PCGApplyACS + FinalizeDot(2)
            double dq = level0_dot([&](uint32_t i, I3 c) -> double {
                if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
                R diag, sum;
                stencil(0, pcg_d, c, i, &cell_diag, diag, sum);
                R qi = diag * pcg_d[i] - sum;
                pcg_q[i] = qi;
                return double(pcg_d[i] * qi);
            });
            scalars[2] = dq;
            // PCGUpdatePRCS (+ ||r||^2)
            const R alpha = R(ratio_f(scalars[0], scalars[2]));
            if (P.pcg_flexible) {  // r_{k+1} . z_k with the new residual, before z is overwritten
                scalars[4] = level0_dot([&](uint32_t i, I3) -> double {
                    if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
                    R ri = pcg_r[i] - alpha * pcg_q[i];
                    return double(ri * pcg_z[i]);
                });
            }
            rr = level0_dot([&](uint32_t i, I3 c) -> double {
                if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
                p[i] = p[i] + alpha * pcg_d[i];
                R ri = pcg_r[i] - alpha * pcg_q[i];
                pcg_r[i] = ri;
                R diag = cell_diag[i] + R(DIAG_EPSILON);
                pcg_z[i] = is_red(c) ? red_init(ri / diag) : R(0);
                return double(ri * ri);
            });
            done = it + 1;
            if (tol_mode && rel() <= double(tolerance)) break;
            if (it + 1 < iterations) {
                rho = vcycle(coarse_iterations);
                scalars[3] = scalars[0];
                scalars[0] = rho;
                update_d(false);
            }
        }
        last_solve_iterations = done;
        last_solve_rel_residual = float(rel());
        last_solve_converged = !tol_mode || rel() <= double(tolerance);
        return done;
    }
    // PCGUpdateDCS: d = z + beta d. The first direction is d = z exactly (the reference computes
    // z + 0 * d; the two differ only in the sign of a zero or a non-finite stale d). Flexible PCG
    // subtracts r_k.z_{k-1} (scalars[4]) from rho_k, in FP64, before the ratio.
    void update_d(bool first) {
        const double num = P.pcg_flexible ? scalars[0] - scalars[4] : scalars[0];
        const R beta = first ? R(0) : R(ratio_f(num, scalars[3]));
        for_active_cells([&](uint32_t i, I3) {
            if (type_of(cell_type[i]) != CELL_FLUID) return;
            pcg_d[i] = first ? pcg_z[i] : pcg_z[i] + beta * pcg_d[i];
        });
    }
    // ||b - A p|| / ||b|| with the level-0 operator (diagnostic of a finished solve).
    // The residual is evaluated in FP64 from the stored (FP32) solution and operator -- diag_f + 1e-4 as the
    // solve forms it, the fluid neighbours in neighbour order -- so it measures the solution, not the
    // cancellation of an FP32 evaluation of A p.
    double true_rel_residual(const std::vector<R>& p, const std::vector<R>& div) {
        double num = level0_dot([&](uint32_t i, I3 c) -> double {
            if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
            R diag, sum;
            stencil(0, p, c, i, &cell_diag, diag, sum);
            double nsum = 0.0;
            for (int n = 0; n < 6; ++n) {
                I3 nb = c + neighbour_offset(n);
                if (!inside(nb, mg[0].dim)) continue;
                uint32_t ni = level_index(0, nb);
                if ((level_type_raw(0, ni) & CELL_TYPE_MASK) == CELL_FLUID) nsum = nsum + double(p[ni]);
            }
            double r = -double(div[i]) - (double(diag) * double(p[i]) - nsum);
            return r * r;
        });
        double den = level0_dot([&](uint32_t i, I3) -> double {
            if (type_of(cell_type[i]) != CELL_FLUID) return 0.0;
            R b = -div[i];
            return double(b * b);
        });
        return den > 0.0 ? std::sqrt(num / den) : 0.0;
    }

    // ---- two-way collider coupling (Slosh.usf:897-993, 1062-1216, 1316-1370) ------------------------------
    // Per-collider integer accumulators in 1/1024 fixed point (CouplingScale): the sums do not depend on
    // the order of the additions. Slots: 0-2 force, 3-5 torque, 6 wetted faces, 7 submerged cells,
    // 8-10 fluid velocity sum, 11 solid cells, 12-14 submerged centroid offset sum.
    bool two_way(uint32_t k) const { return (colliders[k].flags & COLLIDER_FLAG_TWO_WAY) != 0u; }
    // The cell loops run under OpenMP, so the additions are atomic (wrapping, as the GPU's integer atomics).
    void coupling_add_i(uint32_t k, int slot, int32_t v) {
        uint32_t* a = reinterpret_cast<uint32_t*>(&coupling[k * SLOSH_COUPLING_STRIDE + uint32_t(slot)]);
        #pragma omp atomic
        *a += uint32_t(v);
    }
    void coupling_add(uint32_t k, int slot, R v) { coupling_add_i(k, slot, to_i32_rn<R>(v * R(P.coupling_scale))); }
    void coupling_count(uint32_t k, int slot) { coupling_add_i(k, slot, 1); }
    V3<R> collider_center(uint32_t k) const { return {R(colliders[k].center[0]), R(colliders[k].center[1]), R(colliders[k].center[2])}; }
    // CellCenterVelocity, Slosh.usf:897-906.
    V3<R> cell_center_velocity(const std::vector<R>& v, I3 c) const {
        R out[3];
        for (int a = 0; a < 3; ++a) out[a] = R(0.5f) * (v[face_index(a, c)] + v[face_index(a, c + axis_offset(a))]);
        return {out[0], out[1], out[2]};
    }
    // AccumulatePressureForce, Slosh.usf:913-925.
    void accumulate_pressure_force(uint32_t k, V3<R> face_pos, V3<R> into, R p_hat) {
        const R pa = p_hat * R(P.pressure_to_pascal);
        const R h = R(P.cell_size);
        const V3<R> force = ((pa * h) * h) * into;
        const V3<R> torque = cross(face_pos - collider_center(k), force);
        coupling_add(k, 0, force.x); coupling_add(k, 1, force.y); coupling_add(k, 2, force.z);
        coupling_add(k, 3, torque.x); coupling_add(k, 4, torque.y); coupling_add(k, 5, torque.z);
    }
    // AccumulateCoupling, Slosh.usf:929-946: wetted face of a two-way collider (+ binary force when the
    // smoothed estimator is off).
    void accumulate_coupling(uint32_t k, const std::vector<R>& v, I3 fluid_cell, V3<R> face_pos, V3<R> into, R p_hat) {
        if (!two_way(k)) return;
        if (P.smooth_coupling == 0u) accumulate_pressure_force(k, face_pos, into, p_hat);
        const V3<R> fv = cell_center_velocity(v, fluid_cell);
        coupling_count(k, 6);
        coupling_add(k, 8, fv.x); coupling_add(k, 9, fv.y); coupling_add(k, 10, fv.z);
    }
    // EstimateSeepagePressure, Slosh.usf:952-977: mean pressure of the liquid first met by horizontal walks
    // (x+, x-, y+, y-; up to 16 cells) out of body `id`.
    bool seepage_pressure(I3 body, uint32_t id, R& p_hat) const {
        const I3 dirs[4] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
        R sum = R(0), count = R(0);
        for (int k = 0; k < 4; ++k) {
            I3 q = body;
            for (int step = 0; step < 16; ++step) {
                q = q + dirs[k];
                const uint32_t t = get_cell_type(q);
                if (type_of(t) != CELL_SOLID || collider_of(t) != id) {
                    if (type_of(t) == CELL_FLUID) {
                        sum = sum + pressure[cell_index(q)];
                        count = count + R(1);
                    }
                    break;
                }
            }
        }
        p_hat = count > R(0) ? sum / count : R(0);
        return count > R(0);
    }
    // AccumulateContact, Slosh.usf:979-992.
    void accumulate_contact(uint32_t solid_packed, I3 body, V3<R> face_pos, V3<R> into) {
        const uint32_t id = collider_of(solid_packed);
        if (id == 0u || !two_way(id - 1u)) return;
        R ph;
        if (seepage_pressure(body, id, ph)) accumulate_pressure_force(id - 1u, face_pos, into, ph);
    }
    // The coupling terms of ProjectFace (Slosh.usf:1004-1029), evaluated after the projection pass on the
    // projected field (the reference samples the wetted-face velocity while the same pass writes it).
    void coupling_faces(const std::vector<R>& v) {
        if (P.num_colliders == 0u) return;
        for_active_cells([&](uint32_t, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const I3 ca = c - axis_offset(axis), cb = c;
                const uint32_t a = get_cell_type(ca), b = get_cell_type(cb);
                const V3<R> e{axis == 0 ? R(1) : R(0), axis == 1 ? R(1) : R(0), axis == 2 ? R(1) : R(0)};
                const V3<R> ne{axis == 0 ? R(-1) : R(0), axis == 1 ? R(-1) : R(0), axis == 2 ? R(-1) : R(0)};
                if (type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID) {
                    if (collider_of(a) != collider_of(b)) {
                        const V3<R> fp = face_position(axis, c);
                        accumulate_contact(b, cb, fp, e);
                        accumulate_contact(a, ca, fp, ne);
                    }
                } else if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                    if (type_of(a) == CELL_FLUID && collider_of(b) != 0u)
                        accumulate_coupling(collider_of(b) - 1u, v, ca, face_position(axis, c), e, pressure[cell_index(ca)]);
                    else if (type_of(b) == CELL_FLUID && collider_of(a) != 0u)
                        accumulate_coupling(collider_of(a) - 1u, v, cb, face_position(axis, c), ne, pressure[cell_index(cb)]);
                }
            }
        });
    }
    // FluidPressureGradient, Slosh.usf:1086-1101.
    V3<R> fluid_pressure_gradient(I3 c, R pc) const {
        R g[3];
        for (int a = 0; a < 3; ++a) {
            const I3 e = axis_offset(a);
            const bool bp = type_of(get_cell_type(c + e)) == CELL_FLUID, bm = type_of(get_cell_type(c - e)) == CELL_FLUID;
            const R pp = bp ? pressure[cell_index(c + e)] : R(0);
            const R pm = bm ? pressure[cell_index(c - e)] : R(0);
            g[a] = bp && bm ? (pp - pm) * R(0.5f) : (bp ? pp - pc : (bm ? pc - pm : R(0)));
        }
        const R ih = R(P.inv_cell_size);
        return {g[0] * ih, g[1] * ih, g[2] * ih};
    }
    // BodySurfacePressure, Slosh.usf:1105-1125.
    bool body_surface_pressure(I3 c, R& p_hat) const {
        R sum = R(0), count = R(0);
        for (int n = 0; n < 6; ++n) {
            I3 d{0, 0, 0};
            d[n >> 1] = (n & 1) ? 1 : -1;
            const I3 nb = c + d;
            if (type_of(get_cell_type(nb)) == CELL_FLUID) {
                const R pn = pressure[cell_index(nb)];
                const R slope = type_of(get_cell_type(nb + d)) == CELL_FLUID ? pressure[cell_index(nb + d)] - pn : R(0);
                sum = sum + (pn - R(0.5f) * slope);
                count = count + R(1);
            }
        }
        p_hat = count > R(0) ? sum / count : R(0);
        return count > R(0);
    }
    // CouplingForceCS, Slosh.usf:1127-1216: smoothed pressure force and torque on two-way colliders.
    void coupling_force() {
        const R h = R(P.cell_size), ih = R(P.inv_cell_size);
        for_active_cells([&](uint32_t index, I3 c) {
            const uint32_t packed = cell_type[index];
            const uint32_t type = type_of(packed);
            if (type == CELL_AIR) return;
            const V3<R> x{(R(c.x) + R(0.5f)) * h, (R(c.y) + R(0.5f)) * h, (R(c.z) + R(0.5f)) * h};
            R p_hat = R(0);
            V3<R> g{R(0), R(0), R(0)};
            bool have = false;
            if (type == CELL_FLUID) {
                p_hat = pressure[index];
                g = fluid_pressure_gradient(c, p_hat);
                have = true;
            } else if (collider_of(packed) != 0u) {
                have = body_surface_pressure(c, p_hat);
            }
            if (!have) return;
            for (uint32_t k = 0; k < P.num_colliders; ++k) {
                const slosh_collider_t& col = colliders[k];
                if ((col.flags & COLLIDER_FLAG_TWO_WAY) == 0u || std::fabs(collider_sdf<R>(col, x)) > h) continue;
                if (type == CELL_SOLID && collider_of(packed) != k + 1u) continue;
                R sp = p_hat;
                if (type == CELL_FLUID) {
                    const R phi = collider_sdf<R>(col, x);
                    sp = sp + dot(g, (-phi) * collider_normal<R>(col, x, R(0.25f) * h));
                }
                const R scale = (((-sp) * R(P.pressure_to_pascal)) * h) * h;
                V3<R> force{R(0), R(0), R(0)}, torque{R(0), R(0), R(0)};
                const V3<R> center = collider_center(k);
                for (int n = 0; n < 6; ++n) {
                    V3<R> normal{R(0), R(0), R(0)};
                    I3 d{0, 0, 0};
                    const R sgn = (n & 1) ? R(1) : R(-1);
                    if (n >> 1 == 0) { normal.x = sgn; d.x = (n & 1) ? 1 : -1; }
                    else if (n >> 1 == 1) { normal.y = sgn; d.y = (n & 1) ? 1 : -1; }
                    else { normal.z = sgn; d.z = (n & 1) ? 1 : -1; }
                    const V3<R> fp = x + (R(0.5f) * h) * normal;
                    if (type == CELL_SOLID) {
                        const uint32_t nbp = get_cell_type(c + d);
                        if (type_of(nbp) == CELL_SOLID && collider_of(nbp) != k + 1u) continue;
                    }
                    const R w = saturate(R(0.5f) + collider_sdf<R>(col, fp) * ih);
                    const V3<R> df = (scale * w) * normal;
                    force = force + df;
                    torque = torque + cross(fp - center, df);
                }
                coupling_add(k, 0, force.x); coupling_add(k, 1, force.y); coupling_add(k, 2, force.z);
                coupling_add(k, 3, torque.x); coupling_add(k, 4, torque.y); coupling_add(k, 5, torque.z);
            }
        });
    }
    // SubmergedCS, Slosh.usf:1316-1370: solid cells per collider and the submerged ones (a horizontal walk out
    // of the body meets dense fluid with no air in the three cells below), with their centroid offset.
    void submerged() {
        const R h = R(P.cell_size);
        const I3 dirs[4] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
        for_active_cells([&](uint32_t index, I3 c) {
            const uint32_t packed = cell_type[index];
            const uint32_t id = collider_of(packed);
            if (type_of(packed) != CELL_SOLID || id == 0u) return;
            coupling_count(id - 1u, 11);
            bool sub = false;
            for (int k = 0; k < 4; ++k) {
                I3 q = c;
                for (int step = 0; step < 12; ++step) {
                    q = q + dirs[k];
                    const uint32_t t = get_cell_type(q);
                    if (type_of(t) != CELL_SOLID || collider_of(t) != id) {
                        bool liquid = type_of(t) == CELL_FLUID && (t & CELL_DENSE_FLAG) != 0u;
                        for (int below = 1; below <= 3; ++below)
                            liquid = liquid && type_of(get_cell_type(q - I3{0, 0, below})) != CELL_AIR;
                        sub = sub || liquid;
                        break;
                    }
                }
            }
            if (sub) {
                const V3<R> off = V3<R>{(R(c.x) + R(0.5f)) * h, (R(c.y) + R(0.5f)) * h, (R(c.z) + R(0.5f)) * h} - collider_center(id - 1u);
                coupling_count(id - 1u, 7);
                coupling_add(id - 1u, 12, off.x); coupling_add(id - 1u, 13, off.y); coupling_add(id - 1u, 14, off.z);
            }
        });
    }

    // ---- ProjectFace, Slosh.usf:995-1052 (the coupling terms are accumulated by coupling_faces) -------------
    void project(std::vector<R>& v) {
        for_active_cells([&](uint32_t index, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const uint32_t f = uint32_t(axis) * L.pool_cells + index;
                I3 ca = c - axis_offset(axis), cb = c;
                uint32_t a = get_cell_type(ca), b = get_cell_type(cb);
                uint32_t flags = face_flags[f] & FACE_HAS_WEIGHT;
                if (type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID) {
                } else if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                    flags |= FACE_VALID | FACE_SOLID;
                } else if (type_of(a) == CELL_FLUID || type_of(b) == CELL_FLUID) {
                    R pa, pb;
                    if (type_of(a) == CELL_FLUID && type_of(b) == CELL_FLUID) {
                        pa = pressure[cell_index(ca)];
                        pb = pressure[cell_index(cb)];
                    } else if (type_of(a) == CELL_FLUID) {
                        pa = pressure[cell_index(ca)];
                        pb = pa - pa * air_face_weight(cell_density(ca), cb);
                    } else {
                        pb = pressure[cell_index(cb)];
                        pa = pb - pb * air_face_weight(cell_density(cb), ca);
                    }
                    v[f] = v[f] - (pb - pa);
                    flags |= FACE_VALID;
                }
                face_flags[f] = flags;
            }
        });
    }

    // ---- ResidualCS, Slosh.usf:1222-1257 -----------------------------------------------------------
    void residual(const std::vector<R>& v) {
        uint32_t mx = stats[2], sum3 = 0, n4 = 0, sum5 = 0, n6 = 0;
        for_active_cells([&](uint32_t index, I3 c) {
            if (type_of(cell_type[index]) != CELL_FLUID) return;
            R div = R(0);
            for (int a = 0; a < 3; ++a) div = div + (v[face_index(a, c + axis_offset(a))] - v[face_index(a, c)]);
            float rate = float(std::fabs(div) * R(P.inv_cell_size));
            uint32_t bits = f32_bits(rate);
            uint32_t add3 = uint32_t(std::fmin(rate, 1.0e5f) * 1000.0f);
            bool touches_air = false;
            for (int n = 0; n < 6; ++n) touches_air = touches_air || type_of(get_cell_type(c + neighbour_offset(n))) == CELL_AIR;
            uint32_t add5 = 0, add6 = 0;
            if (!touches_air) {
                float dens = float(clampr(cell_density_interior(c), R(0), R(4)));
                add5 = uint32_t(to_i32_rn<float>((dens - 1.0f) * 10000.0f));
                add6 = 1u;
            }
            #pragma omp critical(slosh_residual)
            {
                mx = std::max(mx, bits);
                sum3 += add3; n4 += 1u; sum5 += add5; n6 += add6;
            }
        });
        stats[2] = mx; stats[3] += sum3; stats[4] += n4; stats[5] += sum5; stats[6] += n6;
    }

    // ---- DensityProjectionRhsCS, Slosh.usf:775-805 --------------------------------------------------------
    void density_rhs_pass() {
        for_active_cells([&](uint32_t index, I3 c) {
            density_q[index] = R(0);
            if (type_of(cell_type[index]) != CELL_FLUID) { density_rhs[index] = R(0); return; }
            R dev = cell_density_interior(c) - R(1);
            bool touches_air = false;
            for (int n = 0; n < 6; ++n) touches_air = touches_air || type_of(get_cell_type(c + neighbour_offset(n))) == CELL_AIR;
            if (touches_air) dev = std::fmax(dev, R(0));
            density_rhs[index] = -R(P.density_relaxation) * clampr(dev, R(-0.5f), R(0.5f));
        });
    }
    // DensityFaceDisplacement / DensityDisplacementFace, Slosh.usf:808-828.
    void density_displacement(std::vector<R>& dst) {
        for_active_cells([&](uint32_t index, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const uint32_t f = uint32_t(axis) * L.pool_cells + index;
                I3 ca = c - axis_offset(axis);
                uint32_t a = get_cell_type(ca), b = get_cell_type(c);
                R value;
                if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                    value = R(0);
                } else {
                    R qa = type_of(a) == CELL_FLUID ? density_q[cell_index(ca)] : R(0);
                    R qb = type_of(b) == CELL_FLUID ? density_q[cell_index(c)] : R(0);
                    value = -(qb - qa);
                }
                dst[f] = value;
            }
        });
    }

    // ---- ExtrapolateFace, Slosh.usf:1263-1310 -----------------------------------------------------------
    void extrapolate(const std::vector<R>& src, std::vector<R>& dst, uint32_t iteration) {
        uint32_t known = FACE_VALID;
        for (uint32_t it = 0; it < iteration; ++it) known |= 1u << (FACE_EXTRAP_SHIFT + it);
        const uint32_t new_bit = 1u << (FACE_EXTRAP_SHIFT + iteration);
        // Flags are read against bits set before this iteration only; new bits are applied after the pass.
        std::vector<uint8_t>& mark = extrap_mark;
        mark.assign(L.total_faces, 0);
        for_active_cells([&](uint32_t index, I3 c) {
            for (int axis = 0; axis < 3; ++axis) {
                const uint32_t f = uint32_t(axis) * L.pool_cells + index;
                uint32_t flags = face_flags[f];
                R center = src[f];
                if ((flags & known) != 0u) { dst[f] = center; continue; }
                R sum = R(0), count = R(0);
                for (int n = 0; n < 6; ++n) {
                    I3 nb = c + neighbour_offset(n);
                    if (!in_grid(nb)) continue;
                    uint32_t ni = face_index(axis, nb);
                    uint32_t nf = face_flags[ni];
                    if ((nf & known) != 0u && (nf & FACE_SOLID) == 0u) { sum = sum + src[ni]; count = count + R(1); }
                }
                if (count > R(0)) { dst[f] = sum / count; mark[f] = 1; } else { dst[f] = R(0); }
            }
        });
        for (uint32_t f = 0; f < L.total_faces; ++f)
            if (mark[f]) face_flags[f] |= new_bit;
    }

    // ---- G2P + advection: GatherComponent, SampleVelocityComponent, AdvectParticle, G2PAdvectCS,
    //      Slosh.usf:1376-1678 ------------------------------------------------------------------------
    // Trilinear interpolation of the 8 stencil values u[o] (o = x + 2 y + 4 z) as lerps with fused
    // multiply-adds, x then y then z, and the three partial derivatives from the same differences:
    // mathematically the reference's sum_o w_o u_o and sum_o sign_o (w3 w3) inv_h u_o (Slosh.usf:1376-1443),
    // rounded in this order on both sides of the parity (the HLSL fixes no order either: its compiler may
    // fuse a multiply-add).
    struct Lerp3 {
        R val, gx, gy, gz;
    };
    static Lerp3 lerp3(const R u[8], R fx, R fy, R fz, R inv_h, bool grad) {
        const R d00 = u[1] - u[0], d10 = u[3] - u[2], d01 = u[5] - u[4], d11 = u[7] - u[6];
        const R a00 = std::fma(fx, d00, u[0]), a10 = std::fma(fx, d10, u[2]);
        const R a01 = std::fma(fx, d01, u[4]), a11 = std::fma(fx, d11, u[6]);
        const R e0 = a10 - a00, e1 = a11 - a01;
        const R b0 = std::fma(fy, e0, a00), b1 = std::fma(fy, e1, a01);
        const R g = b1 - b0;
        Lerp3 r{std::fma(fz, g, b0), R(0), R(0), R(0)};
        if (grad) {
            r.gz = g * inv_h;
            r.gy = std::fma(fz, e1 - e0, e0) * inv_h;
            const R c0 = std::fma(fy, d10 - d00, d00), c1 = std::fma(fy, d11 - d01, d01);
            r.gx = std::fma(fz, c1 - c0, c0) * inv_h;
        }
        return r;
    }
    void gather_component(int axis, V3<R> xp, const std::vector<R>& v, R& unew, R& delta_sum, R& delta_weight, V3<R>& grad) const {
        const R inv_h = R(P.inv_cell_size);
        V3<R> off{axis == 0 ? R(0) : R(0.5f), axis == 1 ? R(0) : R(0.5f), axis == 2 ? R(0) : R(0.5f)};
        V3<R> g{xp.x * inv_h - off.x, xp.y * inv_h - off.y, xp.z * inv_h - off.z};
        I3 base{int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z))};
        V3<R> fr{g.x - R(base.x), g.y - R(base.y), g.z - R(base.z)};
        delta_sum = R(0); delta_weight = R(0);
        R u[8];
        for (uint32_t o = 0; o < 8u; ++o) {
            I3 oi{int(o & 1u), int((o >> 1u) & 1u), int((o >> 2u) & 1u)};
            I3 node{clampi(base.x + oi.x, 0, L.grid.x - 1), clampi(base.y + oi.y, 0, L.grid.y - 1), clampi(base.z + oi.z, 0, L.grid.z - 1)};
            uint32_t f = face_index(axis, node);
            u[o] = v[f];
            if (P.use_apic == 0u && (face_flags[f] & FACE_HAS_WEIGHT) != 0u) {
                V3<R> w3{oi.x ? fr.x : R(1) - fr.x, oi.y ? fr.y : R(1) - fr.y, oi.z ? fr.z : R(1) - fr.z};
                R w = w3.x * w3.y * w3.z;
                delta_sum = delta_sum + w * (u[o] - vel_old[f]);
                delta_weight = delta_weight + w;
            }
        }
        const Lerp3 l = lerp3(u, fr.x, fr.y, fr.z, inv_h, P.use_apic != 0u);
        unew = l.val;
        grad = {l.gx, l.gy, l.gz};
    }
    R sample_velocity_component(int axis, V3<R> xp, R fallback, bool check_known, const std::vector<R>& v) const {
        const uint32_t known = FACE_VALID | (0xFFFFFFFFu << FACE_EXTRAP_SHIFT);
        const R inv_h = R(P.inv_cell_size);
        V3<R> off{axis == 0 ? R(0) : R(0.5f), axis == 1 ? R(0) : R(0.5f), axis == 2 ? R(0) : R(0.5f)};
        V3<R> g{xp.x * inv_h - off.x, xp.y * inv_h - off.y, xp.z * inv_h - off.z};
        I3 base{int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z))};
        V3<R> fr{g.x - R(base.x), g.y - R(base.y), g.z - R(base.z)};
        R u[8];
        for (uint32_t o = 0; o < 8u; ++o) {
            I3 oi{int(o & 1u), int((o >> 1u) & 1u), int((o >> 2u) & 1u)};
            I3 node{clampi(base.x + oi.x, 0, L.grid.x - 1), clampi(base.y + oi.y, 0, L.grid.y - 1), clampi(base.z + oi.z, 0, L.grid.z - 1)};
            uint32_t f = face_index(axis, node);
            u[o] = v[f];
            if (check_known && (face_flags[f] & known) == 0u) u[o] = fallback;
        }
        return lerp3(u, fr.x, fr.y, fr.z, inv_h, false).val;
    }
    V3<R> sample_density_displacement(V3<R> xp, const std::vector<R>& disp) const {
        const R inv_h = R(P.inv_cell_size);
        V3<R> out;
        for (int axis = 0; axis < 3; ++axis) {
            V3<R> off{axis == 0 ? R(0) : R(0.5f), axis == 1 ? R(0) : R(0.5f), axis == 2 ? R(0) : R(0.5f)};
            V3<R> g{xp.x * inv_h - off.x, xp.y * inv_h - off.y, xp.z * inv_h - off.z};
            I3 base{int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z))};
            V3<R> fr{g.x - R(base.x), g.y - R(base.y), g.z - R(base.z)};
            R u[8];
            for (uint32_t o = 0; o < 8u; ++o) {
                I3 oi{int(o & 1u), int((o >> 1u) & 1u), int((o >> 2u) & 1u)};
                I3 node{clampi(base.x + oi.x, 0, L.grid.x - 1), clampi(base.y + oi.y, 0, L.grid.y - 1), clampi(base.z + oi.z, 0, L.grid.z - 1)};
                u[o] = disp[face_index(axis, node)];
            }
            out[axis] = lerp3(u, fr.x, fr.y, fr.z, inv_h, false).val;
        }
        R len = length(out);
        V3<R> d = len > R(0.5f) ? out * (R(0.5f) / len) : out;
        return d * R(P.cell_size);
    }

    // AdvectParticle; returns the end brick (NO_BRICK for dead / drained particles).
    uint32_t advect_particle(uint32_t i, const std::vector<R>& v, const std::vector<R>& disp, bool apply_density,
                             uint32_t& max_speed_bits, uint32_t* local_stats) {
        ParticleU<R> p = unpack_particle<R>(particles[i]);
        if (is_dead_age(float(p.age))) return NO_BRICK;
        const R h = R(P.cell_size), inv_h = R(P.inv_cell_size), dt = R(P.dt);
        V3<R> lo{h * R(1.01f), h * R(1.01f), h * R(1.01f)};
        V3<R> hi{(R(L.grid.x) - R(1.01f)) * h, (R(L.grid.y) - R(1.01f)) * h, (R(L.grid.z) - R(1.01f)) * h};
        V3<R> pic, delta, delta_w, gx, gy, gz;
        gather_component(0, p.pos, v, pic.x, delta.x, delta_w.x, gx);
        gather_component(1, p.pos, v, pic.y, delta.y, delta_w.y, gy);
        gather_component(2, p.pos, v, pic.z, delta.z, delta_w.z, gz);
        V3<R> new_vel;
        if (P.use_apic) {
            new_vel = pic;
            p.cx = gx; p.cy = gy; p.cz = gz;
        } else {
            V3<R> fd;
            for (int a = 0; a < 3; ++a) fd[a] = delta_w[a] > R(1e-4f) ? delta[a] / delta_w[a] : pic[a] - p.vel[a];
            V3<R> target = p.vel + fd;
            const R fr = R(P.flip_ratio);
            new_vel = {pic.x + fr * (target.x - pic.x), pic.y + fr * (target.y - pic.y), pic.z + fr * (target.z - pic.z)};
            p.cx = {R(0), R(0), R(0)}; p.cy = p.cx; p.cz = p.cx;
        }
        // RK2 midpoint with the Euler blend (Slosh.usf:1491-1504).
        V3<R> v1 = pic;
        const R half_dt = R(0.5f) * dt;
        V3<R> mid = p.pos + half_dt * v1;
        mid = {clampr(mid.x, lo.x, hi.x), clampr(mid.y, lo.y, hi.y), clampr(mid.z, lo.z, hi.z)};
        R mid_cells = half_dt * length(v1) * inv_h;
        V3<R> v2 = v1;
        if (mid_cells < R(2)) {
            bool check = mid_cells > R(1);
            V3<R> s{sample_velocity_component(0, mid, v1.x, check, v), sample_velocity_component(1, mid, v1.y, check, v),
                    sample_velocity_component(2, mid, v1.z, check, v)};
            R t = saturate(mid_cells - R(1));
            v2 = {s.x + t * (v1.x - s.x), s.y + t * (v1.y - s.y), s.z + t * (v1.z - s.z)};
        }
        V3<R> x = p.pos + dt * v2;
        if (apply_density) {
            V3<R> cp{clampr(p.pos.x, lo.x, hi.x), clampr(p.pos.y, lo.y, hi.y), clampr(p.pos.z, lo.z, hi.z)};
            x = x + sample_density_displacement(cp, disp);
        }
        // Pool exhausted: ballistic (Slosh.usf:1512-1521).
        I3 pc{clampi(int(std::floor(p.pos.x * inv_h)), 0, L.grid.x - 1), clampi(int(std::floor(p.pos.y * inv_h)), 0, L.grid.y - 1),
              clampi(int(std::floor(p.pos.z * inv_h)), 0, L.grid.z - 1)};
        if (is_null_cell(cell_index(pc))) {
            V3<R> g{R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
            new_vel = p.vel + g * dt;
            x = p.pos + dt * new_vel;
            p.cx = {R(0), R(0), R(0)}; p.cy = p.cx; p.cz = p.cx;
        }
        // Force-field manipulators (Slosh.usf:1523-1559).
        for (uint32_t m = 0; m < P.num_manipulators; ++m) {
            const slosh_manipulator_t& f = manipulators[m];
            if (f.kind == MANIP_DRAIN) continue;
            R w = manipulator_weight<R>(f, x);
            if (w <= R(0)) continue;
            V3<R> r = x - V3<R>{R(f.center[0]), R(f.center[1]), R(f.center[2])};
            V3<R> ax{R(f.axis[0]), R(f.axis[1]), R(f.axis[2])};
            if (f.kind == MANIP_DIRECTIONAL) {
                new_vel = new_vel + ax * (R(f.strength) * w * dt);
            } else if (f.kind == MANIP_RADIAL) {
                R rl = length(r);
                V3<R> n = rl > R(1e-5f) ? V3<R>{r.x / rl, r.y / rl, r.z / rl} : V3<R>{R(0), R(0), R(0)};
                new_vel = new_vel + n * (R(f.strength) * w * dt);
            } else if (f.kind == MANIP_SWIRL) {
                V3<R> perp = r - dot(r, ax) * ax;
                R pl = length(perp);
                if (pl > R(1e-5f)) {
                    V3<R> pn{perp.x / pl, perp.y / pl, perp.z / pl};
                    V3<R> tangent = cross(ax, pn);
                    new_vel = new_vel + (tangent - pn * R(f.param0)) * (R(f.strength) * w * dt);
                }
            } else if (f.kind == MANIP_DRAG) {
                new_vel = new_vel * R(exp_r(float(-R(f.strength) * w * dt)));
            }
        }
        // Colliders (Slosh.usf:1561-1592).
        const R radius = R(P.particle_radius), adh = R(P.adhesion_accel), adh_range = R(P.adhesion_range);
        const R friction = R(P.friction);
        for (uint32_t k = 0; k < P.num_colliders; ++k) {
            const slosh_collider_t& c = colliders[k];
            R d = collider_sdf<R>(c, x);
            if (adh > R(0) && d < radius + adh_range) {
                V3<R> n = collider_normal<R>(c, x, R(0.25f) * h);
                R w = saturate(R(1) - (d - radius) / adh_range);
                V3<R> vs = collider_velocity_at<R>(c, x);
                R vn = dot(new_vel - vs, n);
                new_vel = new_vel - n * std::fmin(adh * w * dt, std::fmax(vn, R(0)) + adh * w * dt * R(0.25f));
            }
            if (d < radius) {
                V3<R> n = collider_normal<R>(c, x, R(0.25f) * h);
                x = x + n * (radius - d);
                V3<R> vs = collider_velocity_at<R>(c, x);
                V3<R> rel = new_vel - vs;
                R vn = dot(rel, n);
                if (vn < R(0)) {
                    rel = rel - vn * n;
                    rel = rel - friction * (rel - dot(rel, n) * n);
                }
                new_vel = vs + rel;
            }
        }
        // Domain walls (Slosh.usf:1594-1623).
        uint32_t wall = 0u;
        for (int a = 0; a < 3; ++a) {
            if (x[a] < lo[a]) { x[a] = lo[a]; new_vel[a] = std::fmax(new_vel[a], R(0)); wall |= 1u << a; }
            else if (x[a] > hi[a]) { x[a] = hi[a]; new_vel[a] = std::fmin(new_vel[a], R(0)); wall |= 1u << a; }
        }
        if (wall != 0u && friction > R(0))
            for (int a = 0; a < 3; ++a)
                if ((wall & (1u << a)) == 0u) new_vel[a] = new_vel[a] * (R(1) - friction);
        R speed = length(new_vel);
        if (speed > R(P.max_speed)) {
            local_stats[9] += 1u;
            local_stats[10] += uint32_t(float(x.x * R(100)));
            local_stats[11] += uint32_t(float(x.y * R(100)));
            local_stats[12] += uint32_t(float(x.z * R(100)));
            I3 sc{int(std::floor(p.pos.x * inv_h)), int(std::floor(p.pos.y * inv_h)), int(std::floor(p.pos.z * inv_h))};
            if (type_of(get_cell_type(sc)) == CELL_SOLID) local_stats[13] += 1u;
        }
        // Drains (Slosh.usf:1639-1654).
        for (uint32_t dr = 0; dr < P.num_manipulators; ++dr) {
            const slosh_manipulator_t& f = manipulators[dr];
            if (f.kind != MANIP_DRAIN || manipulator_sdf<R>(f, x) > R(0)) continue;
            float chance = f.param0 > 0.0f ? 1.0f - exp_r(-f.param0 * P.dt) : 1.0f;
            if (chance >= 1.0f || hash_to_unit(pcg_hash(i * 2654435761u + P.frame_seed * 97u + dr)) < chance) {
                particles[i] = dead_particle();
                local_stats[15] += 1u;
                return NO_BRICK;
            }
        }
        p.pos = x;
        p.vel = new_vel;
        p.age = p.age + dt;
        particles[i] = pack_particle(p);
        max_speed_bits = std::max(max_speed_bits, f32_bits(float(speed)));
        I3 ec{clampi(int(std::floor(x.x * inv_h)), 0, L.grid.x - 1), clampi(int(std::floor(x.y * inv_h)), 0, L.grid.y - 1),
              clampi(int(std::floor(x.z * inv_h)), 0, L.grid.z - 1)};
        return brick_index_of({ec.x >> 3, ec.y >> 3, ec.z >> 3});
    }
    void g2p(const std::vector<R>& v, const std::vector<R>& disp, bool apply_density) {
        uint32_t max_bits = stats[0];
        uint32_t add[NUM_STATS] = {};
        #pragma omp parallel
        {
            uint32_t mb = 0, loc[NUM_STATS] = {};
            #pragma omp for schedule(static)
            for (int64_t i = 0; i < int64_t(num_particles); ++i) {
                uint32_t brick = advect_particle(uint32_t(i), v, disp, apply_density, mb, loc);
                if (brick != NO_BRICK) brick_touch[brick] = 1u;
            }
            #pragma omp critical(slosh_g2p)
            {
                max_bits = std::max(max_bits, mb);
                for (uint32_t s = 0; s < NUM_STATS; ++s) add[s] += loc[s];
            }
        }
        stats[0] = max_bits;
        for (uint32_t s = 9; s < NUM_STATS; ++s) stats[s] += add[s];
    }

    // =============================================================================================
    // Frame and substep schedule: Step_RenderThread, SloshProxy.cpp:339-737.
    // =============================================================================================
    void set_pass_params(const slosh_frame_input_t& in) {
        const slosh_settings_t& s = S;
        const float h = s.cell_size;
        P.cell_size = h;
        P.inv_cell_size = 1.0f / h;
        P.num_colliders = std::min<uint32_t>(in.num_colliders, SLOSH_MAX_COLLIDERS);
        colliders.assign(in.colliders, in.colliders + P.num_colliders);
        P.num_manipulators = std::min<uint32_t>(in.num_manipulators, SLOSH_MAX_MANIPULATORS);
        manipulators.assign(in.manipulators, in.manipulators + P.num_manipulators);
        for (int a = 0; a < 3; ++a) P.gravity[a] = s.gravity[a];
        P.flip_ratio = clampr(s.flip_ratio, 0.0f, 1.0f);
        P.use_apic = s.transfer_mode == SLOSH_TRANSFER_APIC ? 1u : 0u;
        P.max_speed = std::max(s.max_speed, 0.1f);
        P.friction = clampr(s.boundary_friction, 0.0f, 1.0f);
        const float gmag = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
        P.adhesion_accel = std::max(s.adhesion, 0.0f) * 1.5f * gmag;
        P.adhesion_range = std::max(s.adhesion_distance, 1e-4f);
        P.particle_radius = s.particle_radius_cells * h;
        P.sor_weight = clampr(s.sor_weight, 0.5f, 1.95f);
        P.density_correction = s.two_sided_density_projection ? 0.0f : std::max(s.density_correction, 0.0f);
        P.target_ppc = 8.0f;
        P.density_deadband = std::max(s.density_deadband, 0.0f);
        P.coupling_scale = 1024.0f;
        P.warm_start_scale = 1.0f;
        P.smooth_coupling = s.smooth_coupling_force ? 1u : 0u;
        P.precision_mode = s.precision_mode <= uint32_t(SLOSH_PRECISION_BF16_STORAGE) ? s.precision_mode : uint32_t(SLOSH_PRECISION_FP32);
        P.restrict_scale = 0.25f * clampr(s.mg_correction_scale, 0.5f, 1.95f);
        P.mg_sweeps = clampi(s.mg_smoothing_sweeps, 1, 4);
        P.pcg_flexible = s.pcg_flexible ? 1u : 0u;
        P.smooth_weight = clampr(s.mg_smoother_weight, 0.5f, 1.9f);
        P.ghost_fluid = s.ghost_fluid ? 1u : 0u;
        const int interval = clampi(s.density_projection_interval, 1, 8);
        P.density_relaxation = 1.0f - std::pow(1.0f - clampr(s.density_relaxation, 0.0f, 1.0f), float(interval));
    }

    // Frame prologue up to the substep loop. Returns the substep count (0: paused or empty).
    int begin_frame(const slosh_frame_input_t& in, float* out_dt) {
        slosh_settings_t s = clamp_settings(in.settings);
        if (in.reset || !allocated || !layout_equals(s, S)) allocate(s);
        ensure_capacity(s.particle_capacity);
        S = s;
        ++sim_frame;
        set_pass_params(in);
        bool has_drain = false;
        for (uint32_t m = 0; m < P.num_manipulators; ++m) has_drain = has_drain || manipulators[m].kind == MANIP_DRAIN;
        std::fill(coupling, coupling + SLOSH_MAX_COLLIDERS * SLOSH_COUPLING_STRIDE, 0);
        std::fill(stats, stats + NUM_STATS, 0u);
        for (uint32_t e = 0; e < in.num_emits; ++e) emit(in.emits[e]);
        if (num_particles > 0 && ((s.sort_interval > 0 && (sim_frame % uint64_t(s.sort_interval)) == 0) ||
                                  (has_drain && (sim_frame % 8ull) == 0)))
            sort_particles();
        substeps = 0;
        density_projection_this_frame = false;
        if (!in.paused && num_particles > 0) {
            const float frame_dt = clampr(in.delta_time, 1e-4f, clampr(s.max_frame_dt, 1.0f / 240.0f, 1.0f / 10.0f));
            const float gmag = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
            const float speed_estimate = std::max(last_max_speed, 1.0f) + gmag * frame_dt;
            substeps = clampi(int(std::ceil(speed_estimate * frame_dt / (std::max(s.cfl, 0.1f) * s.cell_size))),
                              std::max(s.min_substeps, 1), std::max(s.max_substeps, 1));
            frame_dt_sub = frame_dt / float(substeps);
            P.dt = frame_dt_sub;
            P.viscosity_alpha = s.kinematic_viscosity * frame_dt_sub / (s.cell_size * s.cell_size);
            P.pressure_to_pascal = s.density * s.cell_size / frame_dt_sub;
            const int interval = clampi(s.density_projection_interval, 1, 8);
            density_projection_this_frame = s.two_sided_density_projection && P.density_relaxation > 0.0f &&
                                            (sim_frame % uint64_t(interval)) == 0;
        }
        if (out_dt) *out_dt = frame_dt_sub;
        return substeps;
    }

    void substep(int step) {
        const bool last = step == substeps - 1;
        // PREVIOUS: MarkCellsCS rescales the last solution by dt / dt_prev; ZERO and LEARNED start
        // from zero (LEARNED then takes the network's guess).
        P.warm_start_scale = S.warm_start == uint32_t(SLOSH_WARM_START_PREVIOUS) ? (prev_dt > 0.0f ? P.dt / prev_dt : 1.0f) : 0.0f;
        prev_dt = P.dt;
        P.frame_seed = uint32_t(sim_frame * 16ull + uint64_t(step));
        // Brick pool
        brick_free();
        brick_alloc();
        pool_args();
        clear_new_slots();
        // Grid transfer
        build_solid();
        p2g();
        mark_cells();
        normalize_faces();
        int c = 0;
        if (P.viscosity_alpha > 0.0f && S.viscosity_iterations > 0) {
            vel[1] = vel[0];
            int src = 1;
            for (int it = 0; it < S.viscosity_iterations; ++it) {
                int dst = src == 1 ? 2 : 1;
                viscosity_jacobi(vel[0], vel[src], vel[dst]);
                src = dst;
            }
            c = src;
        }
        divergence_pass(vel[c]);
        // Pressure
        if (S.pressure_solver == SLOSH_SOLVER_MGPCG) {
            const int coarse = clampi(S.mg_coarse_iterations, 1, 200);
            if (S.tolerance > 0.0f) mgpcg(pressure, divergence, 0, S.tolerance, S.max_iterations, coarse);
            else mgpcg(pressure, divergence, S.pcg_iterations, 0.0f, 0, coarse);
        } else {
            for (int it = 0; it < S.pressure_iterations; ++it)
                for (uint32_t colour = 0; colour < 2u; ++colour) rbgs_sweep(pressure, divergence, colour, P.sor_weight);
            last_solve_iterations = S.pressure_iterations;
            last_solve_converged = true;
        }
        if (last) {  // diagnostic, once per frame
            last_solve_true_rel_residual = float(true_rel_residual(pressure, divergence));
            if (S.pressure_solver != SLOSH_SOLVER_MGPCG) last_solve_rel_residual = last_solve_true_rel_residual;
        }
        project(vel[c]);
        coupling_faces(vel[c]);
        if (P.num_colliders > 0u && P.smooth_coupling != 0u) coupling_force();
        if (last) residual(vel[c]);
        const bool density = density_projection_this_frame && last;
        if (density) {
            density_rhs_pass();
            if (S.pressure_solver == SLOSH_SOLVER_MGPCG) {
                // The projection reuses the pressure solver with 2 fixed PCG iterations (SloshProxy.cpp:664-670);
                // keep the pressure solve's statistics.
                int it = last_solve_iterations; float rel = last_solve_rel_residual; bool conv = last_solve_converged;
                mgpcg(density_q, density_rhs, 2, 0.0f, 0, clampi(S.mg_coarse_iterations, 1, 200));
                last_solve_iterations = it; last_solve_rel_residual = rel; last_solve_converged = conv;
            } else {
                for (int it = 0; it < std::max(S.density_projection_iterations, 1); ++it)
                    for (uint32_t colour = 0; colour < 2u; ++colour) rbgs_sweep(density_q, density_rhs, colour, 1.7f);
            }
        }
        for (int it = 0; it < S.extrapolation_layers; ++it) {
            const int dst = (c + 1) % 3;
            extrapolate(vel[c], vel[dst], uint32_t(it));
            c = dst;
        }
        if (density) density_displacement(vel[(c + 2) % 3]);
        g2p(vel[c], vel[(c + 2) % 3], density);
        last_disp_index = (c + 2) % 3;
        if (c != 0) vel[0] = vel[c];  // SloshProxy.cpp:709-712
        cur = 0;
    }

    void end_frame() {
        if (P.num_colliders > 0u && substeps > 0) submerged();  // once per frame, after the last substep
        // AccumulateStatsCS (Slosh.usf:264-270)
        particle_count[2] += stats[15];
        stats[14] = particle_count[0];
        stats[15] = particle_count[2];
        // Exact, unlagged readback (the reference reads back 2-4 frames late, SloshProxy.cpp:739-805).
        if (substeps > 0) {
            float ms = bits_f32(stats[0]);
            last_max_speed = std::isfinite(ms) ? ms : 0.0f;
        }
        num_particles = std::min(num_particles, particle_count[0]);
    }

    void step_frame(const slosh_frame_input_t& in) {
        float dt = 0.0f;
        int n = begin_frame(in, &dt);
        for (int s = 0; s < n; ++s) substep(s);
        end_frame();
    }
};

}  // namespace slosh_oracle
