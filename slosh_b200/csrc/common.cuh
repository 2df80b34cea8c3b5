// Device-side definitions shared by the Slosh substep kernels (sm_100a).
//
// Reference (PLUG = SloshDemo/Plugins/Slosh): cell/face flag bits, fixed-point scale and particle
// packing follow PLUG/Shaders/Private/SloshCommon.ush:27-105; sparse-brick addressing follows
// PLUG/Shaders/Private/Slosh.usf:98-199. Layout in HBM:
//   * per-cell buffers: num_pool_bricks slots of 512 cells (slot s = cells [512 s, 512 s + 512),
//     local index x + 8 (y + 8 z)); slot 0 is the null brick, all zeros, never written;
//   * per-face buffers: three planes of pool_cells faces, face (axis, F) stored with cell F;
//   * particles: 48-byte records (3 x 16-byte vectors), arrays of structures.
// All kernels are compiled with --fmad=false so every float expression rounds in source order; the
// CPU oracle uses the same order, which makes the two bit-identical.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

#include "../../include/slosh_cuda.h"

namespace slosh {

constexpr uint32_t CELL_AIR = 0u, CELL_FLUID = 1u, CELL_SOLID = 2u, CELL_TYPE_MASK = 3u;
constexpr uint32_t CELL_DENSE_FLAG = 4u, CELL_COLLIDER_SHIFT = 8u;
constexpr uint32_t COLLIDER_FLAG_TWO_WAY = 1u;  // SloshCommon.ush:42
constexpr float COUPLING_SCALE = 1024.0f;      // fixed point of the coupling accumulators (CouplingFixedScale)
constexpr uint32_t FACE_VALID = 1u, FACE_SOLID = 2u, FACE_HAS_WEIGHT = 4u, FACE_EXTRAP_SHIFT = 4u;
constexpr uint32_t BRICK_CELLS = 512u, NO_BRICK = 0xFFFFFFFFu;
constexpr float P2G_FIXED_SCALE = 1048576.0f;
constexpr float P2G_FIXED_INV = 1.0f / 1048576.0f;
constexpr float DIAG_EPSILON = 1e-4f;
constexpr uint32_t MANIP_DRAIN = 0u, MANIP_DIRECTIONAL = 1u, MANIP_RADIAL = 2u, MANIP_SWIRL = 3u, MANIP_DRAG = 4u;
constexpr uint32_t MANIP_SHAPE_EVERYWHERE = 3u;
constexpr int GRID_THREADS = 256;  // threads per CTA of a brick pass: 2 cells of a 512-cell brick each

// Everything a grid or particle kernel needs to address the state. Passed by value.
struct Dev {
    int3 grid;
    int3 brick_dim;
    uint32_t num_bricks, num_pool_bricks, pool_cells, total_faces;
    float h, inv_h;
    // brick pool
    const uint32_t* brick_table;
    uint32_t* brick_table_w;
    uint32_t* slot_brick;
    uint32_t* free_slots;
    uint32_t* brick_touch;
    uint32_t* brick_want;
    uint32_t* pool_scratch;  // the pool update's per-CTA counts and offsets (pool_scratch_words(num_bricks))
    uint32_t* new_slots;
    uint32_t* active_bricks;
    // cells
    uint32_t* cell_type;
    int32_t* cell_count;
    float* pressure;
    float* divergence;
    float* cell_diag;
    float* density_q;
    float* density_rhs;
    // faces
    int32_t* accum;
    uint32_t* face_flags;
    float* face_weight;
    float* vel_old;
    // diagnostics
    uint32_t* stats;
    int32_t* coupling;
    const slosh_collider_t* colliders;
    const slosh_manipulator_t* manipulators;
};

// Per-substep scalars (FSloshPassParameters as Step_RenderThread fills it, SloshProxy.cpp:400-562).
struct Pass {
    float dt;
    float gravity[3];
    float flip_ratio, max_speed, friction, adhesion_accel, adhesion_range, particle_radius;
    float viscosity_alpha, warm_start_scale, pressure_to_pascal, density_correction, target_ppc;
    float density_deadband, density_relaxation;
    uint32_t use_apic, ghost_fluid, num_colliders, num_manipulators, frame_seed, smooth_coupling;
};

// ---- small helpers ------------------------------------------------------------------------------
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
__device__ __forceinline__ float saturatef(float v) { return clampf(v, 0.0f, 1.0f); }
__device__ __forceinline__ int3 add3(int3 a, int3 b) { return make_int3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ int3 axis_off(int a) { return make_int3(a == 0, a == 1, a == 2); }
__device__ __forceinline__ int3 nbr_off(int n) {  // 0..5 -> -x, +x, -y, +y, -z, +z
    const int s = (n & 1) ? 1 : -1;
    const int a = n >> 1;
    return make_int3(a == 0 ? s : 0, a == 1 ? s : 0, a == 2 ? s : 0);
}
__device__ __forceinline__ int comp(int3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ float compf(float3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 addf3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 scale3(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 mul3s(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }

// ---- addressing (Slosh.usf:110-199) ------------------------------------------------------------------
__device__ __forceinline__ bool in_grid(const Dev& d, int3 c) {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < d.grid.x && c.y < d.grid.y && c.z < d.grid.z;
}
__device__ __forceinline__ uint32_t brick_index_of(const Dev& d, int3 b) {
    return uint32_t(b.x + d.brick_dim.x * (b.y + d.brick_dim.y * b.z));
}
__device__ __forceinline__ int3 brick_coord_of(const Dev& d, uint32_t brick) {
    const uint32_t bx = uint32_t(d.brick_dim.x), by = uint32_t(d.brick_dim.y);
    return make_int3(int(brick % bx), int((brick / bx) % by), int(brick / (bx * by)));
}
__device__ __forceinline__ uint32_t local_index_of(int3 c) {
    return uint32_t((c.x & 7) + 8 * ((c.y & 7) + 8 * (c.z & 7)));
}
__device__ __forceinline__ int3 local_coord_of(uint32_t l) { return make_int3(int(l & 7u), int((l >> 3) & 7u), int(l >> 6)); }
__device__ __forceinline__ uint32_t cell_index(const Dev& d, int3 c) {
    uint32_t slot = 0u;
    if (in_grid(d, c)) slot = __ldg(d.brick_table + brick_index_of(d, make_int3(c.x >> 3, c.y >> 3, c.z >> 3)));
    return slot * BRICK_CELLS + local_index_of(c);
}
__device__ __forceinline__ bool is_null_cell(uint32_t i) { return i < BRICK_CELLS; }
__device__ __forceinline__ uint32_t face_index(const Dev& d, int axis, int3 f) {
    return uint32_t(axis) * d.pool_cells + cell_index(d, f);
}
__device__ __forceinline__ uint32_t type_of(uint32_t packed) { return packed & CELL_TYPE_MASK; }
__device__ __forceinline__ uint32_t collider_of(uint32_t packed) { return (packed >> CELL_COLLIDER_SHIFT) & 0xFFu; }
__device__ __forceinline__ uint32_t get_cell_type(const Dev& d, int3 c) {
    return in_grid(d, c) ? d.cell_type[cell_index(d, c)] : CELL_SOLID;
}
// Index of neighbour n of the cell (c, index): within the brick a fixed offset of the slot, across
// a brick boundary a BrickTable lookup (SloshPressureMG.usf:121-139 does the same for level 0).
__device__ __forceinline__ uint32_t nbr_index(const Dev& d, uint32_t index, int3 c, int n) {
    const int a = n >> 1;
    const int l = comp(c, a) & 7;
    const bool plus = (n & 1) != 0;
    if (plus ? l < 7 : l > 0) {
        const uint32_t stride = a == 0 ? 1u : (a == 1 ? 8u : 64u);
        return plus ? index + stride : index - stride;
    }
    return cell_index(d, add3(c, nbr_off(n)));
}

// ---- particle record (SloshCommon.ush:61-105) ------------------------------------------------------
struct ParticleF {
    float3 pos, vel, cx, cy, cz;
    float age;
};
__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
    const __half ha = __float2half_rn(clampf(a, -65000.0f, 65000.0f));
    const __half hb = __float2half_rn(clampf(b, -65000.0f, 65000.0f));
    return uint32_t(__half_as_ushort(ha)) | (uint32_t(__half_as_ushort(hb)) << 16);
}
__device__ __forceinline__ float half_lo(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu))); }
__device__ __forceinline__ float half_hi(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }

// The 48-byte record as three 16-byte vectors: (pos, age), (vel, c0), (c1, c2, c3, c4).
__device__ __forceinline__ void load_particle_raw(const slosh_particle_t* p, uint32_t i, float4& a, float4& b, uint4& c) {
    const float4* v = reinterpret_cast<const float4*>(p + i);
    a = __ldg(v);
    b = __ldg(v + 1);
    c = __ldg(reinterpret_cast<const uint4*>(v + 2));
}
__device__ __forceinline__ ParticleF unpack_particle(float4 a, float4 b, uint4 c) {
    ParticleF p;
    p.pos = make_float3(a.x, a.y, a.z);
    p.age = a.w;
    p.vel = make_float3(b.x, b.y, b.z);
    const uint32_t c0 = __float_as_uint(b.w);
    p.cx = make_float3(half_lo(c0), half_hi(c0), half_lo(c.x));
    p.cy = make_float3(half_hi(c.x), half_lo(c.y), half_hi(c.y));
    p.cz = make_float3(half_lo(c.z), half_hi(c.z), half_lo(c.w));
    return p;
}
__device__ __forceinline__ void store_particle(slosh_particle_t* out, uint32_t i, const ParticleF& p) {
    float4* v = reinterpret_cast<float4*>(out + i);
    const uint32_t c0 = pack_half2(p.cx.x, p.cx.y);
    const uint32_t c1 = pack_half2(p.cx.z, p.cy.x);
    const uint32_t c2 = pack_half2(p.cy.y, p.cy.z);
    const uint32_t c3 = pack_half2(p.cz.x, p.cz.y);
    const uint32_t c4 = pack_half2(p.cz.z, 0.0f);
    v[0] = make_float4(p.pos.x, p.pos.y, p.pos.z, p.age);
    v[1] = make_float4(p.vel.x, p.vel.y, p.vel.z, __uint_as_float(c0));
    reinterpret_cast<uint4*>(v)[2] = make_uint4(c1, c2, c3, c4);
}
// The same record with the APIC rows already packed (c[0..4] as store_particle forms them).
__device__ __forceinline__ void store_particle_packed(slosh_particle_t* out, uint32_t i, float3 pos, float age, float3 vel,
                                                      const uint32_t (&c)[5]) {
    float4* v = reinterpret_cast<float4*>(out + i);
    v[0] = make_float4(pos.x, pos.y, pos.z, age);
    v[1] = make_float4(vel.x, vel.y, vel.z, __uint_as_float(c[0]));
    reinterpret_cast<uint4*>(v)[2] = make_uint4(c[1], c[2], c[3], c[4]);
}
__device__ __forceinline__ void store_dead(slosh_particle_t* out, uint32_t i) {  // DeadParticlePacked
    ParticleF p;
    p.pos = p.vel = p.cx = p.cy = p.cz = make_float3(0.0f, 0.0f, 0.0f);
    p.age = -1.0f;
    store_particle(out, i, p);
}
__device__ __forceinline__ bool is_dead_age(float age) { return !(age >= 0.0f); }

// Programmatic dependent launch. A kernel launched with programmatic stream serialisation (launch_k) may be
// scheduled while its predecessor in the stream is still draining; pdl_entry() first waits until that
// predecessor has completed and its writes are visible (griddepcontrol.wait), then lets the kernel's own
// successor be scheduled (griddepcontrol.launch_dependents), so a successor's CTAs take the SMs this kernel's
// CTAs release while it finishes. Both instructions are no-ops in a kernel launched without the attribute.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- hashing (SloshCommon.ush:255-265) ----------------------------------------------------------------
__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ float hash_to_unit(uint32_t h) { return float(h & 0x00FFFFFFu) / 16777216.0f; }

// ---- shapes (SloshCommon.ush:137-235) -------------------------------------------------------------
__device__ __forceinline__ float3 quat_rotate(float4 q, float3 v) {
    const float3 qv = make_float3(q.x, q.y, q.z);
    const float3 t = scale3(2.0f, cross3(qv, v));
    return addf3(addf3(v, scale3(q.w, t)), cross3(qv, t));
}
__device__ __forceinline__ float collider_sdf(const slosh_collider_t& c, float3 p) {
    const float4 q = make_float4(-c.rotation[0], -c.rotation[1], -c.rotation[2], c.rotation[3]);
    float3 l = quat_rotate(q, sub3(p, ld3(c.center)));
    if (c.type == SLOSH_COLLIDER_SPHERE) return len3(l) - c.extent[0];
    if (c.type == SLOSH_COLLIDER_BOX) {
        const float3 dd = make_float3(fabsf(l.x) - c.extent[0], fabsf(l.y) - c.extent[1], fabsf(l.z) - c.extent[2]);
        const float3 dp = make_float3(fmaxf(dd.x, 0.0f), fmaxf(dd.y, 0.0f), fmaxf(dd.z, 0.0f));
        return len3(dp) + fminf(fmaxf(dd.x, fmaxf(dd.y, dd.z)), 0.0f);
    }
    l.z = l.z - clampf(l.z, -c.extent[1], c.extent[1]);
    return len3(l) - c.extent[0];
}
__device__ __forceinline__ float3 collider_normal(const slosh_collider_t& c, float3 p, float eps) {
    float3 n;
    n.x = collider_sdf(c, addf3(p, make_float3(eps, 0.0f, 0.0f))) - collider_sdf(c, sub3(p, make_float3(eps, 0.0f, 0.0f)));
    n.y = collider_sdf(c, addf3(p, make_float3(0.0f, eps, 0.0f))) - collider_sdf(c, sub3(p, make_float3(0.0f, eps, 0.0f)));
    n.z = collider_sdf(c, addf3(p, make_float3(0.0f, 0.0f, eps))) - collider_sdf(c, sub3(p, make_float3(0.0f, 0.0f, eps)));
    const float len = len3(n);
    return len > 1e-8f ? make_float3(n.x / len, n.y / len, n.z / len) : make_float3(0.0f, 0.0f, 1.0f);
}
__device__ __forceinline__ float3 collider_velocity_at(const slosh_collider_t& c, float3 p) {
    return addf3(ld3(c.linear_velocity), cross3(ld3(c.angular_velocity), sub3(p, ld3(c.center))));
}
// The few transcendental functions of the path (emission shapes and velocity spread, drag, drain
// chance) are evaluated in double and rounded to float. The CPU restatement does the same with the C
// library's double functions, so both sides agree unless the exact value lies within a few double ulps
// of a float rounding boundary (float sinf/cosf/expf/powf of the two libraries differ in the last bit).
__device__ __forceinline__ float sin_r(float x) { return float(sin(double(x))); }
__device__ __forceinline__ float cos_r(float x) { return float(cos(double(x))); }
__device__ __forceinline__ float exp_r(float x) { return float(exp(double(x))); }
__device__ __forceinline__ float pow_r(float x, float y) { return float(pow(double(x), double(y))); }
__device__ __forceinline__ float manipulator_sdf(const slosh_manipulator_t& f, float3 p) {
    if (f.shape == MANIP_SHAPE_EVERYWHERE) return -1.0f;
    slosh_collider_t c;
    c.center[0] = f.center[0]; c.center[1] = f.center[1]; c.center[2] = f.center[2];
    c.type = f.shape;
    c.rotation[0] = f.rotation[0]; c.rotation[1] = f.rotation[1]; c.rotation[2] = f.rotation[2]; c.rotation[3] = f.rotation[3];
    c.extent[0] = f.extent[0]; c.extent[1] = f.extent[1]; c.extent[2] = f.extent[2];
    return collider_sdf(c, p);
}
__device__ __forceinline__ float manipulator_weight(const slosh_manipulator_t& f, float3 p) {
    const float dd = manipulator_sdf(f, p);
    if (dd <= 0.0f) return 1.0f;
    return f.falloff > 0.0f ? saturatef(1.0f - dd / f.falloff) : 0.0f;
}
// GhostTheta (SloshCommon.ush:244-252).
__device__ __forceinline__ float ghost_theta(float rho_fluid, float rho_air) {
    const float denom = rho_fluid - rho_air;
    if (denom <= 1e-4f) return 1.0f;
    return clampf((rho_fluid - 0.5f) / denom, 0.05f, 1.0f);
}

// ---- canonical FP64 reduction (one partial per brick, then one over bricks) ------------------------
// Brick partial: 256 threads hold v[t] + v[t + 256]; each warp folds with shfl_down 16..1; thread 0
// adds the 8 warp results in warp order. Must be called by all 256 threads of the CTA.
__device__ __forceinline__ double warp_fold(double s) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_down_sync(0xFFFFFFFFu, s, off);
    return s;
}
__device__ __forceinline__ double brick_reduce(double s, double* smem8) {
    s = warp_fold(s);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem8[warp] = s;
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0) {
        total = smem8[0];
        for (int w = 1; w < GRID_THREADS / 32; ++w) total = total + smem8[w];
    }
    __syncthreads();
    return total;  // valid in thread 0
}

}  // namespace slosh
