// Particle kernels of the Slosh substep (sm_100a): emission, P2G, G2P + advection.
//
// Reference (PLUG/Shaders/Private/Slosh.usf): EmitReserveCS / EmitParticlesCS (:272-358), P2GCS with
// ScatterComponentTiled (:448-563), GatherComponent / SampleVelocityComponent / AdvectParticle /
// G2PAdvectCS (:1376-1678).
//
// Particles are 48-byte records read and written as three 16-byte vectors per thread. P2G accumulates
// APIC momentum and weight as 2^20 fixed-point int32 (SloshCommon.ush:46-48), so the sums are exact
// and independent of the order in which particles add them.
#include <cstdlib>

#include "kernels.h"

namespace slosh {

namespace {

// ---- EmitReserveCS: base = count; count += n ---------------------------------------------------------
__global__ void k_emit_reserve(uint32_t* pc, uint32_t count) {
    const uint32_t base = pc[0];
    pc[1] = base;
    pc[0] = base + count;
}

// ---- EmitParticlesCS -----------------------------------------------------------------------------------
__global__ void k_emit(Dev d, slosh_particle_t* __restrict__ particles, const uint32_t* __restrict__ pc,
                       slosh_emit_request_t em, uint32_t count, uint32_t bound, uint32_t capacity, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t base = pc[1];
    const uint32_t fill = bound + i;
    if (fill >= base + count && fill < capacity) store_dead(particles, fill);
    const uint32_t h0 = pcg_hash(i * 3u + seed * 7919u);
    const uint32_t h1 = pcg_hash(h0);
    const uint32_t h2 = pcg_hash(h1);
    const float3 rnd = make_float3(hash_to_unit(h0), hash_to_unit(h1), hash_to_unit(h2));
    const float h = d.h;
    float3 pos;
    if (em.shape == SLOSH_EMIT_FILL_CELLS) {
        const uint32_t cell_linear = i / 8u, sub = i % 8u;
        const int lx = int(cell_linear % uint32_t(em.cell_dims[0]));
        const int ly = int((cell_linear / uint32_t(em.cell_dims[0])) % uint32_t(em.cell_dims[1]));
        const int lz = int(cell_linear / uint32_t(em.cell_dims[0] * em.cell_dims[1]));
        const float sx = float(sub & 1u), sy = float((sub >> 1u) & 1u), sz = float((sub >> 2u) & 1u);
        const float j = em.fill_jitter;
        pos.x = (float(em.cell_min[0] + lx) + ((sx + 0.5f) + j * (rnd.x - 0.5f)) * 0.5f) * h;
        pos.y = (float(em.cell_min[1] + ly) + ((sy + 0.5f) + j * (rnd.y - 0.5f)) * 0.5f) * h;
        pos.z = (float(em.cell_min[2] + lz) + ((sz + 0.5f) + j * (rnd.z - 0.5f)) * 0.5f) * h;
    } else if (em.shape == SLOSH_EMIT_SPHERE) {
        const uint32_t h3 = pcg_hash(h2);
        const float cos_t = 2.0f * rnd.x - 1.0f;
        const float sin_t = sqrtf(saturatef(1.0f - cos_t * cos_t));
        const float phi = 6.28318530718f * rnd.y;
        const float r = em.extent[0] * pow_r(fmaxf(hash_to_unit(h3), 1e-6f), 1.0f / 3.0f);
        pos = addf3(ld3(em.center), scale3(r, make_float3(sin_t * cos_r(phi), sin_t * sin_r(phi), cos_t)));
    } else {
        const float3 q = make_float3((2.0f * rnd.x - 1.0f) * em.extent[0], (2.0f * rnd.y - 1.0f) * em.extent[1],
                                     (2.0f * rnd.z - 1.0f) * em.extent[2]);
        pos = addf3(ld3(em.center), quat_rotate(make_float4(em.rotation[0], em.rotation[1], em.rotation[2], em.rotation[3]), q));
    }
    const float lo = h * 1.01f;
    const float3 hi = make_float3((float(d.grid.x) - 1.01f) * h, (float(d.grid.y) - 1.01f) * h, (float(d.grid.z) - 1.01f) * h);
    float3 velocity = ld3(em.velocity);
    const float speed = len3(velocity);
    if (speed > 1e-6f && (em.velocity_spread > 0.0f || em.speed_jitter > 0.0f)) {
        const uint32_t h4 = pcg_hash(h2 ^ 0x9E3779B9u), h5 = pcg_hash(h4), h6 = pcg_hash(h5);
        float3 dir = make_float3(velocity.x / speed, velocity.y / speed, velocity.z / speed);
        const float3 ref = fabsf(dir.z) < 0.9f ? make_float3(0.0f, 0.0f, 1.0f) : make_float3(1.0f, 0.0f, 0.0f);
        float3 t0 = cross3(dir, ref);
        const float t0l = len3(t0);
        t0 = make_float3(t0.x / t0l, t0.y / t0l, t0.z / t0l);
        const float3 t1 = cross3(dir, t0);
        const float cos_a = 1.0f + hash_to_unit(h4) * (cos_r(em.velocity_spread) - 1.0f);
        const float sin_a = sqrtf(saturatef(1.0f - cos_a * cos_a));
        const float phi = 6.28318530718f * hash_to_unit(h5);
        dir = addf3(scale3(cos_a, dir), scale3(sin_a, addf3(scale3(cos_r(phi), t0), scale3(sin_r(phi), t1))));
        velocity = mul3s(mul3s(dir, speed), fmaxf(1.0f + em.speed_jitter * (2.0f * hash_to_unit(h6) - 1.0f), 0.0f));
    }
    ParticleF p;
    p.pos = make_float3(clampf(pos.x, lo, hi.x), clampf(pos.y, lo, hi.y), clampf(pos.z, lo, hi.z));
    p.vel = velocity;
    p.cx = p.cy = p.cz = make_float3(0.0f, 0.0f, 0.0f);
    p.age = 0.0f;
    store_particle(particles, base + i, p);
    const int3 c = make_int3(clampi(int(floorf(p.pos.x * d.inv_h)), 0, d.grid.x - 1),
                             clampi(int(floorf(p.pos.y * d.inv_h)), 0, d.grid.y - 1),
                             clampi(int(floorf(p.pos.z * d.inv_h)), 0, d.grid.z - 1));
    d.brick_touch[brick_index_of(d, make_int3(c.x >> 3, c.y >> 3, c.z >> 3))] = 1u;
}

// Touch flags of uploaded particles (what EmitParticlesCS does for the particles it writes).
__global__ void k_touch(Dev d, const slosh_particle_t* __restrict__ particles, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(reinterpret_cast<const float4*>(particles + i));
    if (is_dead_age(a.w)) return;
    const int3 c = make_int3(clampi(int(floorf(a.x * d.inv_h)), 0, d.grid.x - 1), clampi(int(floorf(a.y * d.inv_h)), 0, d.grid.y - 1),
                             clampi(int(floorf(a.z * d.inv_h)), 0, d.grid.z - 1));
    d.brick_touch[brick_index_of(d, make_int3(c.x >> 3, c.y >> 3, c.z >> 3))] = 1u;
}

// ---- P2G --------------------------------------------------------------------------------------------------
// APIC P2G (Slosh.usf:448-563). One CTA takes P2G_CHUNK consecutive (spatially sorted) particles; thread t takes
// the run of P2G_PER_THREAD particles starting at t * P2G_PER_THREAD, so at any instant neighbouring lanes hold
// different particles of a cell (a lane-strided assignment would make whole warps hit the same shared-memory
// words). Every contribution is a pair of fixed-point integers (momentum, weight), so the sums are exact in any
// order and the three paths below give the same integers:
//  * CTA tile: the CTA finds the bounding box of its particles' cells; when the box plus its one-node halo fits
//    the shared-memory tile, contributions accumulate there and each non-zero tile entry is then added to global
//    memory once;
//  * warp tiles: when the CTA's box does not fit (a run that wraps from the end of one row of sort keys to the
//    start of the next, or particles that drifted since the last sort), each warp does the same with its own
//    box in an eighth of the tile;
//  * direct: a warp whose box does not fit either adds each contribution to global memory.
// The tile holds 6 planes of 32-bit sums (momentum and weight of the three MAC components) and a plane of
// per-cell particle counts indexed like the nodes (a cell and the node of the same coordinates share an index),
// so one loop flushes all seven. (One 64-bit shared atomic per node, packing weight and momentum into one word,
// measured 2.3 times slower than two 32-bit ones.) A particle whose 2x2x2 stencils all lie inside the grid (every particle the clamped
// advection leaves, all but freshly placed ones at the walls) adds its 24 pairs without per-node tests: a zero
// weight adds (0, 0).
// Measured per 256^3 launch (sorted frames): 2 particles per thread with a 1,024-node tile (28 KB), both records
// loaded before the box reduction and held in registers (64 registers, 4 CTAs per SM) 0.739 ms; the same at 48
// registers and 5 CTAs per SM (68 bytes of spills) 0.748, and reading the records again after the barrier at 5
// CTAs per SM 0.767 (0.820 before the unchecked interior path and the merged flush); the 2,048-node tile on sorted
// frames too, also at 4 CTAs per SM, 0.772; 0.857 with 4 particles per thread; 1 per thread at 6 CTAs per SM was
// slower. In the frames between a bulk emission and the first sort the particles are in emission order and most
// boxes exceed the 1,024-node tile (1.2-1.4 ms per launch on the direct path); the driver then launches the
// 2,048-node tile, which fits them: 0.78-0.80 ms.
constexpr int P2G_THREADS = 256;
constexpr int P2G_WARPS = P2G_THREADS / 32;
#ifndef P2G_MINB_ONE
#define P2G_MINB_ONE 6
#endif
#ifndef P2G_MINB_SMALL
#define P2G_MINB_SMALL 4  // 64 registers, 4 CTAs per SM with the small tile
#endif
constexpr int P2G_PER_THREAD_DEFAULT = 2;
// Tile capacity per CTA in nodes: a CTA of 2 particles per thread (512 particles, one 4^3 sort key of 8 per
// cell) covers about 64 to 180 cells once sorted. WIDE: the 2,048-node tile (56 KB, 4 CTAs per SM) for the frames
// between a bulk emission and the next sort, whose emission-ordered runs of 512 particles span two or three rows
// of cells (at 192^3, frame 2: 98.6 % of the CTA boxes fit 2,048 nodes, 10 % fit 1,024).
template <int PER, bool WIDE = false> struct P2GTile {
    static constexpr int NODES = (WIDE || PER >= 4) ? 2048 : (PER == 2 ? 1024 : 512);
    static constexpr int MINB = WIDE ? 4 : (PER >= 4 ? 1 : (PER == 2 ? P2G_MINB_SMALL : P2G_MINB_ONE));
    static constexpr int SMEM = NODES * 7 * 4;  // momentum and weight of the 3 components + counts
};

__device__ __forceinline__ int3 p2g_cell(const Dev& d, float3 pos) {
    return make_int3(clampi(int(floorf(pos.x * d.inv_h)), 0, d.grid.x - 1), clampi(int(floorf(pos.y * d.inv_h)), 0, d.grid.y - 1),
                     clampi(int(floorf(pos.z * d.inv_h)), 0, d.grid.z - 1));
}

// A tile over the cell box [mn, mx] plus a one-node halo: tile index of node c is
// (c.x - origin.x) + sy (c.y - origin.y) + sz (c.z - origin.z).
struct P2GBox {
    int3 origin;
    int sy, sz, nodes;
};
// False when the box is empty (no live particle) or its tile exceeds cap nodes.
__device__ __forceinline__ bool p2g_box(int3 mn, int3 mx, int cap, P2GBox& b) {
    if (mn.x > mx.x) return false;
    const long long nx = (long long)mx.x - mn.x + 3, ny = (long long)mx.y - mn.y + 3, nz = (long long)mx.z - mn.z + 3;
    if (nx * ny * nz > cap) return false;
    b.origin = make_int3(mn.x - 1, mn.y - 1, mn.z - 1);
    b.sy = int(nx);
    b.sz = int(nx * ny);
    b.nodes = int(nx * ny * nz);
    return true;
}

// Shared-memory reduction by 32-bit shared address (no result returned).
__device__ __forceinline__ void red_shared_add_u32(uint32_t addr, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// The 24 contributions of one particle into a tile: the momentum of component a at index l is the word at shared
// address tile + 4 (2 a plane + l), its weight the word at tile + 4 ((2 a + 1) plane + l), the count of index l
// the word at tile + 4 (6 plane + l).
// Per MAC component the 8 stencil nodes share their per-axis factors: the weights (1 - f, f), the node offsets
// x_n - x_p and their products with the APIC row, the in-grid tests and the tile index; per (y, z) pair
// (w_y w_z) 2^20 and C_y dy + C_z dz, per x u_p + C_x dx, so per node one product forms the scaled weight and one
// sum and one product the momentum: weight = rn(w_x ((w_y w_z) 2^20)), momentum = rn(that (u_p + C_x dx) +
// (C_y dy + C_z dz)) -- the oracle's order.
__device__ __forceinline__ void p2g_particle_tile(const Dev& d, bool apic, const ParticleF& part, const P2GBox& b,
                                                  uint32_t tile, int plane) {
    const uint32_t wplane = 4u * uint32_t(plane);
    const float inv_h = d.inv_h, h = d.h;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const float3 cp = apic ? (axis == 0 ? part.cx : (axis == 1 ? part.cy : part.cz)) : make_float3(0.0f, 0.0f, 0.0f);
        const float up = compf(part.vel, axis);
        const float ox = axis == 0 ? 0.0f : 0.5f, oy = axis == 1 ? 0.0f : 0.5f, oz = axis == 2 ? 0.0f : 0.5f;
        const float gx = part.pos.x * inv_h - ox, gy = part.pos.y * inv_h - oy, gz = part.pos.z * inv_h - oz;
        const int3 base = make_int3(int(floorf(gx)), int(floorf(gy)), int(floorf(gz)));
        const float fx = gx - float(base.x), fy = gy - float(base.y), fz = gz - float(base.z);
        const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
        float px[2], py[2], pz[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            px[j] = cp.x * ((float(base.x + j) + ox) * h - part.pos.x);
            py[j] = cp.y * ((float(base.y + j) + oy) * h - part.pos.y);
            pz[j] = cp.z * ((float(base.z + j) + oz) * h - part.pos.z);
        }
        const uint32_t t =
            tile + 4u * uint32_t(2 * axis * plane + (base.x - b.origin.x) + b.sy * (base.y - b.origin.y) + b.sz * (base.z - b.origin.z));
        const float upx[2] = {up + px[0], up + px[1]};
        const bool inside = unsigned(base.x) < unsigned(d.grid.x - 1) && unsigned(base.y) < unsigned(d.grid.y - 1) &&
                            unsigned(base.z) < unsigned(d.grid.z - 1);
        if (inside) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int oiy = q & 1, oiz = q >> 1;
                const float wyzs = (wy[oiy] * wz[oiz]) * P2G_FIXED_SCALE;
                const float pyz = py[oiy] + pz[oiz];
                const uint32_t tq = t + 4u * uint32_t(oiy * b.sy + oiz * b.sz);
#pragma unroll
                for (int oix = 0; oix < 2; ++oix) {
                    const float ws = wx[oix] * wyzs;
                    red_shared_add_u32(tq + 4u * oix, uint32_t(__float2int_rn(ws * (upx[oix] + pyz))));
                    red_shared_add_u32(tq + wplane + 4u * oix, uint32_t(__float2int_rn(ws)));
                }
            }
        } else {
            bool inx[2], iny[2], inz[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                inx[j] = unsigned(base.x + j) < unsigned(d.grid.x);
                iny[j] = unsigned(base.y + j) < unsigned(d.grid.y);
                inz[j] = unsigned(base.z + j) < unsigned(d.grid.z);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int oiy = q & 1, oiz = q >> 1;
                if (!(iny[oiy] && inz[oiz])) continue;
                const float wyzs = (wy[oiy] * wz[oiz]) * P2G_FIXED_SCALE;
                const float pyz = py[oiy] + pz[oiz];
                const uint32_t tq = t + 4u * uint32_t(oiy * b.sy + oiz * b.sz);
#pragma unroll
                for (int oix = 0; oix < 2; ++oix) {
                    if (!inx[oix]) continue;
                    const float ws = wx[oix] * wyzs;
                    if (ws <= 0.0f) continue;
                    red_shared_add_u32(tq + 4u * oix, uint32_t(__float2int_rn(ws * (upx[oix] + pyz))));
                    red_shared_add_u32(tq + wplane + 4u * oix, uint32_t(__float2int_rn(ws)));
                }
            }
        }
    }
    const int3 cell = p2g_cell(d, part.pos);
    red_shared_add_u32(tile + 6u * wplane + 4u * uint32_t((cell.x - b.origin.x) + b.sy * (cell.y - b.origin.y) + b.sz * (cell.z - b.origin.z)), 1u);
}

// The contributions of one particle added straight to global memory (a warp whose box fits no tile).
__device__ __forceinline__ void p2g_particle_global(const Dev& d, bool apic, const ParticleF& part) {
    const float inv_h = d.inv_h, h = d.h;
    const uint32_t tf = d.total_faces;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const float3 cp = apic ? (axis == 0 ? part.cx : (axis == 1 ? part.cy : part.cz)) : make_float3(0.0f, 0.0f, 0.0f);
        const float up = compf(part.vel, axis);
        const float ox = axis == 0 ? 0.0f : 0.5f, oy = axis == 1 ? 0.0f : 0.5f, oz = axis == 2 ? 0.0f : 0.5f;
        const float gx = part.pos.x * inv_h - ox, gy = part.pos.y * inv_h - oy, gz = part.pos.z * inv_h - oz;
        const int3 base = make_int3(int(floorf(gx)), int(floorf(gy)), int(floorf(gz)));
        const float fx = gx - float(base.x), fy = gy - float(base.y), fz = gz - float(base.z);
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const int oix = o & 1, oiy = (o >> 1) & 1, oiz = (o >> 2) & 1;
            const int3 node = make_int3(base.x + oix, base.y + oiy, base.z + oiz);
            if (!in_grid(d, node)) continue;
            const float w3x = oix ? fx : 1.0f - fx, w3y = oiy ? fy : 1.0f - fy, w3z = oiz ? fz : 1.0f - fz;
            const float ws = w3x * ((w3y * w3z) * P2G_FIXED_SCALE);
            if (ws <= 0.0f) continue;
            const float3 xn = make_float3((float(node.x) + ox) * h, (float(node.y) + oy) * h, (float(node.z) + oz) * h);
            const float3 dx = sub3(xn, part.pos);
            const float term = (up + cp.x * dx.x) + (cp.y * dx.y + cp.z * dx.z);
            const int mom = __float2int_rn(ws * term);
            const int wt = __float2int_rn(ws);
            const uint32_t ci = cell_index(d, node);
            if (!is_null_cell(ci)) {
                const uint32_t f = uint32_t(axis) * d.pool_cells + ci;
                atomicAdd(d.accum + f, mom);
                atomicAdd(d.accum + tf + f, wt);
            }
        }
    }
    const uint32_t ci = cell_index(d, p2g_cell(d, part.pos));
    if (!is_null_cell(ci)) atomicAdd(d.cell_count + ci, 1);
}

// Adds the non-zero entries of a tile (plane q of index l at tile[q * plane + l]) to global memory: per entry one
// cell lookup, then one global add per non-zero momentum, weight and count.
__device__ __forceinline__ void p2g_flush(const Dev& d, const P2GBox& b, const int* tile, int plane, int first, int stride) {
    const uint32_t tf = d.total_faces;
    // l / sy == __umulhi(l, my) and l / sz == __umulhi(l, mz) for l, sy, sz < 2^16 (sy >= 3)
    const uint32_t my = 0xFFFFFFFFu / uint32_t(b.sy) + 1u, mz = 0xFFFFFFFFu / uint32_t(b.sz) + 1u;
    for (int l = first; l < b.nodes; l += stride) {
        int v[7];
        int any = 0;
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            v[q] = tile[q * plane + l];
            any |= v[q];
        }
        if (any == 0) continue;
        const uint32_t lz = __umulhi(uint32_t(l), mz), r = uint32_t(l) - lz * uint32_t(b.sz);
        const uint32_t ly = __umulhi(r, my), lx = r - ly * uint32_t(b.sy);
        const int3 node = make_int3(b.origin.x + int(lx), b.origin.y + int(ly), b.origin.z + int(lz));
        if (!in_grid(d, node)) continue;
        const uint32_t ci = cell_index(d, node);
        if (is_null_cell(ci)) continue;
#pragma unroll
        for (int q = 0; q < 6; ++q)
            if (v[q] != 0) atomicAdd(d.accum + (q & 1) * tf + uint32_t(q >> 1) * d.pool_cells + ci, v[q]);
        if (v[6] != 0) atomicAdd(d.cell_count + ci, v[6]);
    }
}

// f(k) for k = 0 .. N - 1 until it returns false; unrolled where per-k registers are indexed by k.
template <bool UNROLL, int N, class F>
__device__ __forceinline__ void for_each_k(F f) {
    if constexpr (UNROLL) {
#pragma unroll
        for (int k = 0; k < N; ++k)
            if (!f(k)) break;
    } else {
        for (int k = 0; k < N; ++k)
            if (!f(k)) break;
    }
}

template <int P2G_PER_THREAD, bool WIDE = false>
__global__ void __launch_bounds__(P2G_THREADS, P2GTile<P2G_PER_THREAD, WIDE>::MINB) k_p2g(Dev d, Pass p, const slosh_particle_t* __restrict__ particles,
                                                                                 uint32_t n) {
    constexpr int CHUNK = P2G_THREADS * P2G_PER_THREAD;
    constexpr int NODES = P2GTile<P2G_PER_THREAD, WIDE>::NODES;
    constexpr int WARP_NODES = NODES / P2G_WARPS;
    extern __shared__ int p2g_smem[];  // [7][NODES]: momentum, weight of the 3 components, then counts
    __shared__ int s_box[6];
    const uint32_t first = blockIdx.x * uint32_t(CHUNK) + threadIdx.x * uint32_t(P2G_PER_THREAD);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int big = 0x7FFFFFFF;
    if (threadIdx.x < 3) { s_box[threadIdx.x] = big; s_box[3 + threadIdx.x] = -big; }
    __syncthreads();
    int3 wmn = make_int3(big, big, big), wmx = make_int3(-big, -big, -big);  // this warp's cell box
    // HOLD: the whole records are loaded here and kept in registers across the barrier, so their latency
    // overlaps the box reduction; otherwise only the positions, and the records are read again below.
    constexpr bool HOLD = P2G_PER_THREAD <= 2;
    constexpr int NH = HOLD ? P2G_PER_THREAD : 1;
    float4 ha[NH], hb[NH];
    uint4 hc[NH];
    for_each_k<HOLD, P2G_PER_THREAD>([&](int k) {
        const uint32_t i = first + uint32_t(k);
        if (i >= n) return false;
        float4 a;
        if constexpr (HOLD) {
            load_particle_raw(particles, i, ha[k], hb[k], hc[k]);
            a = ha[k];
        } else {
            a = __ldg(reinterpret_cast<const float4*>(particles + i));
        }
        if (is_dead_age(a.w)) return true;
        const int3 c = p2g_cell(d, make_float3(a.x, a.y, a.z));
        wmn = make_int3(min(wmn.x, c.x), min(wmn.y, c.y), min(wmn.z, c.z));
        wmx = make_int3(max(wmx.x, c.x), max(wmx.y, c.y), max(wmx.z, c.z));
        return true;
    });
    wmn.x = __reduce_min_sync(0xFFFFFFFFu, wmn.x); wmn.y = __reduce_min_sync(0xFFFFFFFFu, wmn.y); wmn.z = __reduce_min_sync(0xFFFFFFFFu, wmn.z);
    wmx.x = __reduce_max_sync(0xFFFFFFFFu, wmx.x); wmx.y = __reduce_max_sync(0xFFFFFFFFu, wmx.y); wmx.z = __reduce_max_sync(0xFFFFFFFFu, wmx.z);
    if (lane == 0 && wmn.x <= wmx.x) {
        atomicMin(s_box + 0, wmn.x); atomicMin(s_box + 1, wmn.y); atomicMin(s_box + 2, wmn.z);
        atomicMax(s_box + 3, wmx.x); atomicMax(s_box + 4, wmx.y); atomicMax(s_box + 5, wmx.z);
    }
    __syncthreads();
    if (s_box[0] == big) return;  // no live particle in this CTA (uniform)
    const bool apic = p.use_apic != 0;
    // The CTA's box in the whole tile (block-uniform), else this warp's box in its eighth (warp-uniform).
    P2GBox b;
    const bool cta = p2g_box(make_int3(s_box[0], s_box[1], s_box[2]), make_int3(s_box[3], s_box[4], s_box[5]), NODES, b);
    auto record = [&](int k, uint32_t i, float4& ra, float4& rb, uint4& rc) {
        if constexpr (HOLD) {
            ra = ha[k]; rb = hb[k]; rc = hc[k];
        } else {
            load_particle_raw(particles, i, ra, rb, rc);
        }
    };
    if (!cta && !p2g_box(wmn, wmx, WARP_NODES, b)) {
        for_each_k<HOLD, P2G_PER_THREAD>([&](int k) {
            const uint32_t i = first + uint32_t(k);
            if (i >= n) return false;
            float4 ra, rb;
            uint4 rc;
            record(k, i, ra, rb, rc);
            if (!is_dead_age(ra.w)) p2g_particle_global(d, apic, unpack_particle(ra, rb, rc));
            return true;
        });
        return;
    }
    int* tile = p2g_smem + (cta ? 0 : warp * WARP_NODES);  // this CTA's or warp's tile
    for (int t = cta ? int(threadIdx.x) : lane; t < b.nodes; t += cta ? P2G_THREADS : 32) {
#pragma unroll
        for (int q = 0; q < 7; ++q) tile[q * NODES + t] = 0;
    }
    if (cta) __syncthreads();
    else __syncwarp();
    const uint32_t tile_s = uint32_t(__cvta_generic_to_shared(tile));
    for_each_k<HOLD, P2G_PER_THREAD>([&](int k) {
        const uint32_t i = first + uint32_t(k);
        if (i >= n) return false;
        float4 ra, rb;
        uint4 rc;
        record(k, i, ra, rb, rc);
        if (!is_dead_age(ra.w)) p2g_particle_tile(d, apic, unpack_particle(ra, rb, rc), b, tile_s, NODES);
        return true;
    });
    if (cta) __syncthreads();
    else __syncwarp();
    p2g_flush(d, b, tile, NODES, cta ? int(threadIdx.x) : lane, cta ? P2G_THREADS : 32);
}

// ---- P2G as a per-brick gather (opt-in) -------------------------------------------------------------------
// The index: each live particle's rank in its cell from warp-aggregated adds into cell_count (which are P2G's
// particle counts themselves), an exclusive scan of the counts over the pool cells, and a scatter of the particle
// ids into pool-cell order. Particles in cells of unallocated bricks go to the overflow list instead.
__global__ void __launch_bounds__(256) k_gather_count(Dev d, const slosh_particle_t* __restrict__ particles, uint32_t n, P2GGather g) {
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    uint32_t ci = 0xFFFFFFFFu;  // no cell: out of range, dead, or in an unallocated brick
    if (i < n) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(particles + i));
        if (!is_dead_age(a.w)) {
            const uint32_t c = cell_index(d, p2g_cell(d, make_float3(a.x, a.y, a.z)));
            if (is_null_cell(c)) {
                const uint32_t k = atomicAdd(g.overflow, 1u);
                g.overflow[1u + k] = i;
            } else {
                ci = c;
            }
        }
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, ci);
    const uint32_t leader = uint32_t(__ffs(int(peers))) - 1u;
    uint32_t base = 0u;
    if (ci != 0xFFFFFFFFu && lane == leader) base = uint32_t(atomicAdd(d.cell_count + ci, __popc(peers)));
    base = __shfl_sync(0xFFFFFFFFu, base, int(leader));
    if (i < n) g.rank[i] = ci != 0xFFFFFFFFu ? base + uint32_t(__popc(peers & ((1u << lane) - 1u))) : 0xFFFFFFFFu;
}
__global__ void __launch_bounds__(256) k_gather_scatter(Dev d, const slosh_particle_t* __restrict__ particles, uint32_t n, P2GGather g) {
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = g.rank[i];
    if (r == 0xFFFFFFFFu) return;
    const float4 a = __ldg(reinterpret_cast<const float4*>(particles + i));
    const uint32_t ci = cell_index(d, p2g_cell(d, make_float3(a.x, a.y, a.z)));
    g.index[g.offsets[ci] + r] = i;
}

// The contributions of one particle to the nodes of brick bc only (node coordinates in [8 bc, 8 bc + 7] and inside
// the grid), added to a 6 x 512 tile: the momentum of component a at local node l is the word at shared address
// tile + 4 (2 a 512 + l), its weight the word at tile + 4 ((2 a + 1) 512 + l). The factors and roundings are
// p2g_particle_tile's, so each node receives the same integers as from the scatter (integer sums: any order).
__device__ __forceinline__ void p2g_particle_brick(const Dev& d, bool apic, const ParticleF& part, int3 bc, uint32_t tile) {
    const float inv_h = d.inv_h, h = d.h;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const float3 cp = apic ? (axis == 0 ? part.cx : (axis == 1 ? part.cy : part.cz)) : make_float3(0.0f, 0.0f, 0.0f);
        const float up = compf(part.vel, axis);
        const float ox = axis == 0 ? 0.0f : 0.5f, oy = axis == 1 ? 0.0f : 0.5f, oz = axis == 2 ? 0.0f : 0.5f;
        const float gx = part.pos.x * inv_h - ox, gy = part.pos.y * inv_h - oy, gz = part.pos.z * inv_h - oz;
        const int3 base = make_int3(int(floorf(gx)), int(floorf(gy)), int(floorf(gz)));
        const float fx = gx - float(base.x), fy = gy - float(base.y), fz = gz - float(base.z);
        const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
        float px[2], py[2], pz[2];
        bool inx[2], iny[2], inz[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            px[j] = cp.x * ((float(base.x + j) + ox) * h - part.pos.x);
            py[j] = cp.y * ((float(base.y + j) + oy) * h - part.pos.y);
            pz[j] = cp.z * ((float(base.z + j) + oz) * h - part.pos.z);
            inx[j] = ((base.x + j) >> 3) == bc.x && base.x + j < d.grid.x;
            iny[j] = ((base.y + j) >> 3) == bc.y && base.y + j < d.grid.y;
            inz[j] = ((base.z + j) >> 3) == bc.z && base.z + j < d.grid.z;
        }
        const float upx[2] = {up + px[0], up + px[1]};
        const uint32_t t = tile + 4u * uint32_t(2 * axis * BRICK_CELLS);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int oiy = q & 1, oiz = q >> 1;
            if (!(iny[oiy] && inz[oiz])) continue;
            const float wyzs = (wy[oiy] * wz[oiz]) * P2G_FIXED_SCALE;
            const float pyz = py[oiy] + pz[oiz];
#pragma unroll
            for (int oix = 0; oix < 2; ++oix) {
                if (!inx[oix]) continue;
                const float ws = wx[oix] * wyzs;
                const uint32_t l = uint32_t(((base.x + oix) & 7) + 8 * ((base.y + oiy) & 7) + 64 * ((base.z + oiz) & 7));
                red_shared_add_u32(t + 4u * l, uint32_t(__float2int_rn(ws * (upx[oix] + pyz))));
                red_shared_add_u32(t + 4u * (uint32_t(BRICK_CELLS) + l), uint32_t(__float2int_rn(ws)));
            }
        }
    }
}

// One CTA per active brick at a time (grid-stride): the particles of the 10 x 10 x 10 cells around the brick (its
// own 8^3 and the one-cell layer of its neighbours; a row of cells in one brick is one contiguous index range)
// add into a shared tile, which is then stored over the brick's nodes. No global atomics.
constexpr int P2GG_THREADS = 256;
__global__ void __launch_bounds__(P2GG_THREADS) k_p2g_gather(Dev d, Pass p, const slosh_particle_t* __restrict__ particles, P2GGather g) {
    __shared__ int tile[6 * BRICK_CELLS];
    const uint32_t tile_s = uint32_t(__cvta_generic_to_shared(tile));
    const bool apic = p.use_apic != 0;
    const uint32_t active = d.active_bricks[0];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
        for (uint32_t t = threadIdx.x; t < 6u * BRICK_CELLS; t += P2GG_THREADS) tile[t] = 0;
        __syncthreads();
        for (uint32_t row = warp; row < 100u; row += P2GG_THREADS / 32) {
            const int y = bc.y * 8 - 1 + int(row % 10u), z = bc.z * 8 - 1 + int(row / 10u);
            if (y < 0 || z < 0 || y >= d.grid.y || z >= d.grid.z) continue;
            for (int sg = 0; sg < 3; ++sg) {
                const int x0 = sg == 0 ? bc.x * 8 - 1 : (sg == 1 ? bc.x * 8 : bc.x * 8 + 8);
                const int x1 = sg == 1 ? min(bc.x * 8 + 7, d.grid.x - 1) : x0;
                if (x0 < 0 || x0 >= d.grid.x) continue;
                const uint32_t s2 = __ldg(d.brick_table + brick_index_of(d, make_int3(x0 >> 3, y >> 3, z >> 3)));
                if (s2 == 0u) continue;  // an unallocated brick: its particles are in the overflow list
                const uint32_t c0 = s2 * BRICK_CELLS + local_index_of(make_int3(x0, y, z));
                const uint32_t c1 = c0 + uint32_t(x1 - x0);
                const uint32_t start = g.offsets[c0], end = g.offsets[c1] + uint32_t(d.cell_count[c1]);
                for (uint32_t j = start + lane; j < end; j += 32u) {
                    float4 ra, rb;
                    uint4 rc;
                    load_particle_raw(particles, g.index[j], ra, rb, rc);
                    p2g_particle_brick(d, apic, unpack_particle(ra, rb, rc), bc, tile_s);
                }
            }
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < 6u * BRICK_CELLS; t += P2GG_THREADS) {
            const uint32_t q = t / uint32_t(BRICK_CELLS), l = t % uint32_t(BRICK_CELLS);
            d.accum[(q & 1u) * d.total_faces + (q >> 1) * d.pool_cells + slot * BRICK_CELLS + l] = tile[t];
        }
        __syncthreads();
    }
}
// Particles in cells of unallocated bricks (pool overflow): their contributions to allocated bricks by global adds.
__global__ void __launch_bounds__(256) k_p2g_overflow(Dev d, Pass p, const slosh_particle_t* __restrict__ particles, P2GGather g) {
    const uint32_t count = g.overflow[0];
    const bool apic = p.use_apic != 0;
    for (uint32_t k = blockIdx.x * 256u + threadIdx.x; k < count; k += gridDim.x * 256u) {
        float4 ra, rb;
        uint4 rc;
        load_particle_raw(particles, g.overflow[1u + k], ra, rb, rc);
        p2g_particle_global(d, apic, unpack_particle(ra, rb, rc));
    }
}

// ---- G2P + advection ---------------------------------------------------------------------------------
struct Stencil {
    int3 base;
    float fx, fy, fz;
};
__device__ __forceinline__ Stencil stencil_of(const Dev& d, float3 x, int axis) {
    const float ox = axis == 0 ? 0.0f : 0.5f, oy = axis == 1 ? 0.0f : 0.5f, oz = axis == 2 ? 0.0f : 0.5f;
    const float gx = x.x * d.inv_h - ox, gy = x.y * d.inv_h - oy, gz = x.z * d.inv_h - oz;
    Stencil s;
    s.base = make_int3(int(floorf(gx)), int(floorf(gy)), int(floorf(gz)));
    s.fx = gx - float(s.base.x);
    s.fy = gy - float(s.base.y);
    s.fz = gz - float(s.base.z);
    return s;
}
// Pool indices of the 8 (clamped) stencil nodes of one MAC component. The nodes span at most two
// bricks per axis; the brick table is read once for the base node's brick and again only for the
// neighbouring bricks the stencil actually crosses into.
__device__ __forceinline__ void stencil_indices(const Dev& d, const Stencil& s, int axis, uint32_t idx[8]) {
    const int x0 = clampi(s.base.x, 0, d.grid.x - 1), x1 = clampi(s.base.x + 1, 0, d.grid.x - 1);
    const int y0 = clampi(s.base.y, 0, d.grid.y - 1), y1 = clampi(s.base.y + 1, 0, d.grid.y - 1);
    const int z0 = clampi(s.base.z, 0, d.grid.z - 1), z1 = clampi(s.base.z + 1, 0, d.grid.z - 1);
    const bool cx = (x0 >> 3) != (x1 >> 3), cy = (y0 >> 3) != (y1 >> 3), cz = (z0 >> 3) != (z1 >> 3);
    const uint32_t b000 = brick_index_of(d, make_int3(x0 >> 3, y0 >> 3, z0 >> 3));
    const uint32_t sx = 1u, sy = uint32_t(d.brick_dim.x), sz = uint32_t(d.brick_dim.x * d.brick_dim.y);
    uint32_t slot[8];
    slot[0] = __ldg(d.brick_table + b000);
    slot[1] = cx ? __ldg(d.brick_table + b000 + sx) : slot[0];
    slot[2] = cy ? __ldg(d.brick_table + b000 + sy) : slot[0];
    slot[3] = cy ? (cx ? __ldg(d.brick_table + b000 + sy + sx) : slot[2]) : slot[1];
    slot[4] = cz ? __ldg(d.brick_table + b000 + sz) : slot[0];
    slot[5] = cz ? (cx ? __ldg(d.brick_table + b000 + sz + sx) : slot[4]) : slot[1];
    slot[6] = cz ? (cy ? __ldg(d.brick_table + b000 + sz + sy) : slot[4]) : slot[2];
    slot[7] = cz ? ((cx || cy) ? (cx && cy ? __ldg(d.brick_table + b000 + sz + sy + sx) : (cx ? slot[5] : slot[6])) : slot[4]) : slot[3];
    const uint32_t plane = uint32_t(axis) * d.pool_cells;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int x = (o & 1) ? x1 : x0, y = ((o >> 1) & 1) ? y1 : y0, z = ((o >> 2) & 1) ? z1 : z0;
        idx[o] = plane + slot[o] * BRICK_CELLS + uint32_t((x & 7) + 8 * ((y & 7) + 8 * (z & 7)));
    }
}

// Trilinear interpolation of the 8 stencil values u[o] (o = x + 2 y + 4 z) as lerps with fused
// multiply-adds, x then y then z, and (grad) the three partial derivatives from the same differences:
// mathematically the reference's sum_o w_o u_o and sum_o sign_o (w3 w3) inv_h u_o (Slosh.usf:1376-1443),
// in about a sixth of its operations. The oracle rounds in the same order.
__device__ __forceinline__ float lerp3(const float (&u)[8], float fx, float fy, float fz, float inv_h, bool grad, float3* g3) {
    const float d00 = u[1] - u[0], d10 = u[3] - u[2], d01 = u[5] - u[4], d11 = u[7] - u[6];
    const float a00 = __fmaf_rn(fx, d00, u[0]), a10 = __fmaf_rn(fx, d10, u[2]);
    const float a01 = __fmaf_rn(fx, d01, u[4]), a11 = __fmaf_rn(fx, d11, u[6]);
    const float e0 = a10 - a00, e1 = a11 - a01;
    const float b0 = __fmaf_rn(fy, e0, a00), b1 = __fmaf_rn(fy, e1, a01);
    const float g = b1 - b0;
    if (grad) {
        g3->z = g * inv_h;
        g3->y = __fmaf_rn(fz, e1 - e0, e0) * inv_h;
        const float c0 = __fmaf_rn(fy, d10 - d00, d00), c1 = __fmaf_rn(fy, d11 - d01, d01);
        g3->x = __fmaf_rn(fz, c1 - c0, c0) * inv_h;
    }
    return __fmaf_rn(fz, g, b0);
}

// GatherComponent (Slosh.usf:1376-1410).
__device__ __forceinline__ void gather_component(const Dev& d, const Pass& p, int axis, float3 xp, const float* __restrict__ vel,
                                                 float& unew, float& dsum, float& dw, float3& grad) {
    const Stencil s = stencil_of(d, xp, axis);
    uint32_t idx[8];
    stencil_indices(d, s, axis, idx);
    dsum = 0.0f; dw = 0.0f;
    grad = make_float3(0.0f, 0.0f, 0.0f);
    float u[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) u[o] = vel[idx[o]];
    if (p.use_apic == 0u) {
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const uint32_t f = idx[o];
            if ((d.face_flags[f] & FACE_HAS_WEIGHT) == 0u) continue;
            const int oix = o & 1, oiy = (o >> 1) & 1, oiz = (o >> 2) & 1;
            const float w3x = oix ? s.fx : 1.0f - s.fx, w3y = oiy ? s.fy : 1.0f - s.fy, w3z = oiz ? s.fz : 1.0f - s.fz;
            const float w = w3x * w3y * w3z;
            dsum = dsum + w * (u[o] - d.vel_old[f]);
            dw = dw + w;
        }
    }
    unew = lerp3(u, s.fx, s.fy, s.fz, d.inv_h, p.use_apic != 0u, &grad);
}
// SampleVelocityComponent (Slosh.usf:1417-1443).
__device__ __forceinline__ float sample_component(const Dev& d, int axis, float3 xp, float fallback, bool check,
                                                  const float* __restrict__ vel) {
    const uint32_t known = FACE_VALID | (0xFFFFFFFFu << FACE_EXTRAP_SHIFT);
    const Stencil s = stencil_of(d, xp, axis);
    uint32_t idx[8];
    stencil_indices(d, s, axis, idx);
    float u[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) u[o] = vel[idx[o]];
    if (check) {
#pragma unroll
        for (int o = 0; o < 8; ++o)
            if ((d.face_flags[idx[o]] & known) == 0u) u[o] = fallback;
    }
    return lerp3(u, s.fx, s.fy, s.fz, d.inv_h, false, nullptr);
}
// SampleDensityDisplacement (Slosh.usf:830-854).
__device__ __forceinline__ float3 sample_displacement(const Dev& d, float3 xp, const float* __restrict__ disp) {
    float out[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const Stencil s = stencil_of(d, xp, axis);
        uint32_t idx[8];
        stencil_indices(d, s, axis, idx);
        float u[8];
#pragma unroll
        for (int o = 0; o < 8; ++o) u[o] = disp[idx[o]];
        out[axis] = lerp3(u, s.fx, s.fy, s.fz, d.inv_h, false, nullptr);
    }
    const float3 v = make_float3(out[0], out[1], out[2]);
    const float len = len3(v);
    const float3 dd = len > 0.5f ? mul3s(v, 0.5f / len) : v;
    return mul3s(dd, d.h);
}

constexpr int G2P_THREADS = 256;
// The new particle record is written once and read again only by the next substep's passes, after the grid
// passes in between: cache-streaming (evict-first) stores keep it from displacing the face velocities the
// gathers reuse (0.993 -> 0.982 ms per 256^3 launch). Loading the record without an L1 allocation or evict-first
// in L2 was slower, here (0.996-0.998 ms) and in P2G (0.741-0.774 against 0.740 ms).
__device__ __forceinline__ void g2p_store(slosh_particle_t* out, uint32_t i, float3 pos, float age, float3 vel, const uint32_t (&c)[5]) {
    float4* v = reinterpret_cast<float4*>(out + i);
    __stcs(v, make_float4(pos.x, pos.y, pos.z, age));
    __stcs(v + 1, make_float4(vel.x, vel.y, vel.z, __uint_as_float(c[0])));
    __stcs(reinterpret_cast<uint4*>(v + 2), make_uint4(c[1], c[2], c[3], c[4]));
}

// AdvectParticle + G2PAdvectCS (Slosh.usf:1452-1678). Each thread gathers its stencils straight from the brick
// pool through the brick table; the particles are brick-sorted, so a warp's gathers hit the same few bricks in L1.
// Staging each CTA's particle box of face velocities in shared memory first (24 KB tile, 3-cell margin) measured
// slower (1.22 ms against 0.99 ms per 256^3 substep): the fill reads more nodes than the stencils touch.
template <int MINB>
__global__ void __launch_bounds__(G2P_THREADS, MINB) k_g2p(Dev d, Pass p, slosh_particle_t* __restrict__ particles, uint32_t n,
                                                     const float* __restrict__ vel, const float* __restrict__ disp,
                                                     uint32_t apply_density) {
    const uint32_t i = blockIdx.x * G2P_THREADS + threadIdx.x;
    uint32_t brick = NO_BRICK;
    uint32_t speed_bits = 0u;
    if (i < n) {
        float4 ra, rb;
        uint4 rc;
        load_particle_raw(particles, i, ra, rb, rc);
        ParticleF P = unpack_particle(ra, rb, rc);
        if (!is_dead_age(P.age)) {
            const float h = d.h, inv_h = d.inv_h, dt = p.dt;
            const float lo = h * 1.01f;
            const float3 hi = make_float3((float(d.grid.x) - 1.01f) * h, (float(d.grid.y) - 1.01f) * h, (float(d.grid.z) - 1.01f) * h);
            float3 pic, delta, dw, gx, gy, gz;
            const uint32_t zero_c = pack_half2(0.0f, 0.0f);
            uint32_t cw[5] = {zero_c, zero_c, zero_c, zero_c, zero_c};  // the packed APIC rows (zero for PIC/FLIP)
            gather_component(d, p, 0, P.pos, vel, pic.x, delta.x, dw.x, gx);
            gather_component(d, p, 1, P.pos, vel, pic.y, delta.y, dw.y, gy);
            gather_component(d, p, 2, P.pos, vel, pic.z, delta.z, dw.z, gz);
            float3 nv;
            if (p.use_apic) {
                nv = pic;
                // the new rows packed to halves at once: 5 words live to the store instead of 9 floats
                cw[0] = pack_half2(gx.x, gx.y);
                cw[1] = pack_half2(gx.z, gy.x);
                cw[2] = pack_half2(gy.y, gy.z);
                cw[3] = pack_half2(gz.x, gz.y);
                cw[4] = pack_half2(gz.z, 0.0f);
            } else {
                const float fdx = dw.x > 1e-4f ? delta.x / dw.x : pic.x - P.vel.x;
                const float fdy = dw.y > 1e-4f ? delta.y / dw.y : pic.y - P.vel.y;
                const float fdz = dw.z > 1e-4f ? delta.z / dw.z : pic.z - P.vel.z;
                const float3 target = make_float3(P.vel.x + fdx, P.vel.y + fdy, P.vel.z + fdz);
                nv = make_float3(pic.x + p.flip_ratio * (target.x - pic.x), pic.y + p.flip_ratio * (target.y - pic.y),
                                 pic.z + p.flip_ratio * (target.z - pic.z));
            }
            // RK2 midpoint with the Euler blend.
            const float3 v1 = pic;
            const float half_dt = 0.5f * dt;
            float3 mid = addf3(P.pos, scale3(half_dt, v1));
            mid = make_float3(clampf(mid.x, lo, hi.x), clampf(mid.y, lo, hi.y), clampf(mid.z, lo, hi.z));
            const float mid_cells = half_dt * len3(v1) * inv_h;
            float3 v2 = v1;
            if (mid_cells < 2.0f) {
                const bool check = mid_cells > 1.0f;
                const float3 sv = make_float3(sample_component(d, 0, mid, v1.x, check, vel), sample_component(d, 1, mid, v1.y, check, vel),
                                              sample_component(d, 2, mid, v1.z, check, vel));
                const float t = saturatef(mid_cells - 1.0f);
                v2 = make_float3(sv.x + t * (v1.x - sv.x), sv.y + t * (v1.y - sv.y), sv.z + t * (v1.z - sv.z));
            }
            float3 x = addf3(P.pos, scale3(dt, v2));
            if (apply_density) {
                const float3 cpos = make_float3(clampf(P.pos.x, lo, hi.x), clampf(P.pos.y, lo, hi.y), clampf(P.pos.z, lo, hi.z));
                x = addf3(x, sample_displacement(d, cpos, disp));
            }
            // Pool exhausted: ballistic.
            const int3 pcell = make_int3(clampi(int(floorf(P.pos.x * inv_h)), 0, d.grid.x - 1),
                                         clampi(int(floorf(P.pos.y * inv_h)), 0, d.grid.y - 1),
                                         clampi(int(floorf(P.pos.z * inv_h)), 0, d.grid.z - 1));
            if (is_null_cell(cell_index(d, pcell))) {
                const float3 g = make_float3(p.gravity[0], p.gravity[1], p.gravity[2]);
                nv = addf3(P.vel, mul3s(g, dt));
                x = addf3(P.pos, scale3(dt, nv));
#pragma unroll
                for (int k = 0; k < 5; ++k) cw[k] = zero_c;
            }
            // Force-field manipulators.
            for (uint32_t m = 0; m < p.num_manipulators; ++m) {
                const slosh_manipulator_t& f = d.manipulators[m];
                if (f.kind == MANIP_DRAIN) continue;
                const float w = manipulator_weight(f, x);
                if (w <= 0.0f) continue;
                const float3 r = sub3(x, ld3(f.center));
                const float3 ax = ld3(f.axis);
                if (f.kind == MANIP_DIRECTIONAL) {
                    nv = addf3(nv, mul3s(ax, f.strength * w * dt));
                } else if (f.kind == MANIP_RADIAL) {
                    const float rl = len3(r);
                    const float3 nn = rl > 1e-5f ? make_float3(r.x / rl, r.y / rl, r.z / rl) : make_float3(0.0f, 0.0f, 0.0f);
                    nv = addf3(nv, mul3s(nn, f.strength * w * dt));
                } else if (f.kind == MANIP_SWIRL) {
                    const float3 perp = sub3(r, scale3(dot3(r, ax), ax));
                    const float pl = len3(perp);
                    if (pl > 1e-5f) {
                        const float3 pn = make_float3(perp.x / pl, perp.y / pl, perp.z / pl);
                        const float3 tangent = cross3(ax, pn);
                        nv = addf3(nv, mul3s(sub3(tangent, mul3s(pn, f.param0)), f.strength * w * dt));
                    }
                } else if (f.kind == MANIP_DRAG) {
                    nv = mul3s(nv, exp_r(-f.strength * w * dt));
                }
            }
            // Colliders.
            const float radius = p.particle_radius, adh = p.adhesion_accel, adh_range = p.adhesion_range, friction = p.friction;
            for (uint32_t k = 0; k < p.num_colliders; ++k) {
                const slosh_collider_t& c = d.colliders[k];
                const float dist = collider_sdf(c, x);
                if (adh > 0.0f && dist < radius + adh_range) {
                    const float3 nn = collider_normal(c, x, 0.25f * h);
                    const float w = saturatef(1.0f - (dist - radius) / adh_range);
                    const float3 vs = collider_velocity_at(c, x);
                    const float vn = dot3(sub3(nv, vs), nn);
                    nv = sub3(nv, mul3s(nn, fminf(adh * w * dt, fmaxf(vn, 0.0f) + adh * w * dt * 0.25f)));
                }
                if (dist < radius) {
                    const float3 nn = collider_normal(c, x, 0.25f * h);
                    x = addf3(x, mul3s(nn, radius - dist));
                    const float3 vs = collider_velocity_at(c, x);
                    float3 rel = sub3(nv, vs);
                    const float vn = dot3(rel, nn);
                    if (vn < 0.0f) {
                        rel = sub3(rel, scale3(vn, nn));
                        rel = sub3(rel, scale3(friction, sub3(rel, scale3(dot3(rel, nn), nn))));
                    }
                    nv = addf3(vs, rel);
                }
            }
            // Domain walls.
            uint32_t wall = 0u;
            float xs[3] = {x.x, x.y, x.z}, vs[3] = {nv.x, nv.y, nv.z};
            const float his[3] = {hi.x, hi.y, hi.z};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (xs[a] < lo) { xs[a] = lo; vs[a] = fmaxf(vs[a], 0.0f); wall |= 1u << a; }
                else if (xs[a] > his[a]) { xs[a] = his[a]; vs[a] = fminf(vs[a], 0.0f); wall |= 1u << a; }
            }
            if (wall != 0u && friction > 0.0f) {
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    if ((wall & (1u << a)) == 0u) vs[a] = vs[a] * (1.0f - friction);
            }
            x = make_float3(xs[0], xs[1], xs[2]);
            nv = make_float3(vs[0], vs[1], vs[2]);
            const float speed = len3(nv);
            if (speed > p.max_speed) {
                atomicAdd(d.stats + 9, 1u);
                atomicAdd(d.stats + 10, __float2uint_rz(x.x * 100.0f));
                atomicAdd(d.stats + 11, __float2uint_rz(x.y * 100.0f));
                atomicAdd(d.stats + 12, __float2uint_rz(x.z * 100.0f));
                const int3 sc = make_int3(int(floorf(P.pos.x * inv_h)), int(floorf(P.pos.y * inv_h)), int(floorf(P.pos.z * inv_h)));
                if (type_of(get_cell_type(d, sc)) == CELL_SOLID) atomicAdd(d.stats + 13, 1u);
            }
            bool drained = false;
            for (uint32_t dr = 0; dr < p.num_manipulators && !drained; ++dr) {
                const slosh_manipulator_t& f = d.manipulators[dr];
                if (f.kind != MANIP_DRAIN || manipulator_sdf(f, x) > 0.0f) continue;
                const float chance = f.param0 > 0.0f ? 1.0f - exp_r(-f.param0 * dt) : 1.0f;
                if (chance >= 1.0f || hash_to_unit(pcg_hash(i * 2654435761u + p.frame_seed * 97u + dr)) < chance) {
                    store_dead(particles, i);
                    atomicAdd(d.stats + 15, 1u);
                    drained = true;
                }
            }
            if (!drained) {
                g2p_store(particles, i, x, P.age + dt, nv, cw);
                speed_bits = __float_as_uint(speed);
                const int3 ec = make_int3(clampi(int(floorf(x.x * inv_h)), 0, d.grid.x - 1), clampi(int(floorf(x.y * inv_h)), 0, d.grid.y - 1),
                                          clampi(int(floorf(x.z * inv_h)), 0, d.grid.z - 1));
                brick = brick_index_of(d, make_int3(ec.x >> 3, ec.y >> 3, ec.z >> 3));
            }
        }
    }
    // Touch flags: sorted particles mostly share bricks, so only the first lane of each run writes.
    const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, brick, 1);
    if (brick != NO_BRICK && ((threadIdx.x & 31) == 0 || prev != brick)) d.brick_touch[brick] = 1u;
    speed_bits = __reduce_max_sync(0xFFFFFFFFu, speed_bits);
    if ((threadIdx.x & 31) == 0 && speed_bits) atomicMax(d.stats + 0, speed_bits);
}

}  // namespace

int launch_emit_reserve(uint32_t* particle_count, uint32_t count, cudaStream_t s) {
    k_emit_reserve<<<1, 1, 0, s>>>(particle_count, count);
    return 1;
}
int launch_emit(const Dev& d, slosh_particle_t* particles, const uint32_t* pc, const slosh_emit_request_t& em, uint32_t count,
                uint32_t bound, uint32_t capacity, uint32_t seed, cudaStream_t s) {
    if (count == 0) return 0;
    k_emit<<<(count + 255u) / 256u, 256, 0, s>>>(d, particles, pc, em, count, bound, capacity, seed);
    return 1;
}
int launch_touch_particles(const Dev& d, const slosh_particle_t* particles, uint32_t n, cudaStream_t s) {
    if (n == 0) return 0;
    k_touch<<<(n + 255u) / 256u, 256, 0, s>>>(d, particles, n);
    return 1;
}
template <int PER, bool WIDE = false>
void launch_p2g_per(const Dev& d, const Pass& p, const slosh_particle_t* particles, uint32_t n, cudaStream_t s) {
    static bool configured = false;
    const int smem = P2GTile<PER, WIDE>::SMEM;
    if (!configured) {
        cudaFuncSetAttribute(k_p2g<PER, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        configured = true;
    }
    const uint32_t chunk = uint32_t(P2G_THREADS * PER);
    k_p2g<PER, WIDE><<<(n + chunk - 1u) / chunk, P2G_THREADS, smem, s>>>(d, p, particles, n);
}
int launch_p2g(const Dev& d, const Pass& p, const slosh_particle_t* particles, uint32_t n, bool unsorted, cudaStream_t s) {
    if (n == 0) return 0;
    static const int per = [] {
        const char* e = std::getenv("SLOSH_P2G_PER_THREAD");
        return e ? std::atoi(e) : P2G_PER_THREAD_DEFAULT;
    }();
    if (per == 2 && unsorted) launch_p2g_per<2, true>(d, p, particles, n, s);
    else if (per == 8) launch_p2g_per<8>(d, p, particles, n, s);
    else if (per == 4) launch_p2g_per<4>(d, p, particles, n, s);
    else if (per == 1) launch_p2g_per<1>(d, p, particles, n, s);
    else launch_p2g_per<2>(d, p, particles, n, s);
    return 1;
}
int launch_p2g_gather(const Dev& d, const Pass& p, const P2GGather& g, const slosh_particle_t* particles, uint32_t n,
                      cudaStream_t s) {
    if (n == 0) return 0;
    static const int sms = [] {
        int dev = 0, v = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v;
    }();
    cudaMemsetAsync(g.overflow, 0, 4, s);
    const uint32_t blocks = (n + 255u) / 256u;
    k_gather_count<<<blocks, 256, 0, s>>>(d, particles, n, g);
    const int scans = launch_exclusive_scan(reinterpret_cast<const uint32_t*>(d.cell_count), g.offsets, d.pool_cells, g.scan_tmp, s);
    k_gather_scatter<<<blocks, 256, 0, s>>>(d, particles, n, g);
    k_p2g_gather<<<sms * 8, P2GG_THREADS, 0, s>>>(d, p, particles, g);  // 8 CTAs of 12 KB per SM
    k_p2g_overflow<<<sms, 256, 0, s>>>(d, p, particles, g);
    return 4 + scans;
}
int launch_g2p(const Dev& d, const Pass& p, slosh_particle_t* particles, uint32_t n, const float* vel, const float* disp,
               bool apply_density, cudaStream_t s) {
    if (n == 0) return 0;
    // 4 CTAs per SM (64 registers): 5 (48 registers, spills) measured the same, 3 (no spills) 11 % and 2 42 % slower
    k_g2p<4><<<(n + G2P_THREADS - 1u) / G2P_THREADS, G2P_THREADS, 0, s>>>(d, p, particles, n, vel, disp, apply_density ? 1u : 0u);
    return 1;
}

}  // namespace slosh
