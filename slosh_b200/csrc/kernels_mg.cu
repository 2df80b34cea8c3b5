// Sparse-brick MGPCG pressure solve (sm_100a): McAdams-style multigrid-preconditioned CG with level 0
// in the brick pool and dense coarse levels.
//
// Reference: PLUG/Shaders/Private/SloshPressureMG.usf -- FINE_STENCIL (:142-157), MGBuildTypeCS
// (:256-278), PCGInitCS (:284-305), MGSmoothCS (:311-338), MGRestrictCS (:343-381), MGCoarseSolveCS
// (:386-413), MGProlongCS (:418-433), PCGApplyACS (:438-454), PCGFinalizeDotCS (:457-492),
// PCGUpdatePRCS (:495-524), PCGUpdateDCS (:527-543); driver SloshProxy.cpp:807-1020.
//
// Same arithmetic in the same order as the reference, different execution:
//   * dot products accumulate in FP64 through one fixed tree (a partial per active brick, then the
//     last CTA to finish reduces the partials in a fixed order): deterministic, no finalize launch;
//     alpha and beta are formed in FP64 and rounded to FP32;
//   * the iteration loop is controlled on the device: ctl[] holds the iteration count, its limit,
//     the stopping mode and a done flag; PCGUpdatePR decides whether another iteration runs and, when
//     the solve is a CUDA graph, sets the WHILE node's condition -- no host round trip per iteration;
//   * levels 1-3 are visited through the active bricks' footprints (a brick covers (8 >> l)^3 cells
//     of level l), not by scanning the dense level; every fluid coarse cell lies in such a footprint;
//   * the small coarse levels (<= 4096 cells) run as one single-CTA kernel (descent, coarse solve,
//     ascent with block barriers between passes).
#include <algorithm>
#include <cstdlib>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kernels.h"
#include "tc.cuh"

namespace slosh {

namespace {

// ---- storage precision of the coarse levels (precision_mode) --------------------------------------------
// Coarse-level x and b are computed in FP32; with FP16 or BF16 storage every store rounds to the format
// (round to nearest even) and the arrays hold 2-byte elements. Level 0 and the CG vectors stay FP32.
__device__ __forceinline__ float q_prec(float v, uint32_t prec) {
    if (prec == SLOSH_PRECISION_FP16_STORAGE) return __half2float(__float2half_rn(v));
    if (prec == SLOSH_PRECISION_BF16_STORAGE) return __bfloat162float(__float2bfloat16_rn(v));
    return v;
}
__device__ __forceinline__ float lv_ld(const float* a, uint32_t i, uint32_t prec) {
    if (prec == SLOSH_PRECISION_FP32) return a[i];
    const uint16_t h = reinterpret_cast<const uint16_t*>(a)[i];
    return prec == SLOSH_PRECISION_FP16_STORAGE ? __half2float(__ushort_as_half(h)) : __uint_as_float(uint32_t(h) << 16);
}
// The same load through L2 only (ld.global.cg): for values another CTA of the cluster wrote earlier in the
// same kernel, ordered by a cluster barrier.
__device__ __forceinline__ float lv_ldcg(const float* a, uint32_t i, uint32_t prec) {
    if (prec == SLOSH_PRECISION_FP32) return __ldcg(a + i);
    const uint16_t h = __ldcg(reinterpret_cast<const unsigned short*>(a) + i);
    return prec == SLOSH_PRECISION_FP16_STORAGE ? __half2float(__ushort_as_half(h)) : __uint_as_float(uint32_t(h) << 16);
}
template <bool CG>
__device__ __forceinline__ float lvx(const float* a, uint32_t i, uint32_t prec) {
    return CG ? lv_ldcg(a, i, prec) : lv_ld(a, i, prec);
}
__device__ __forceinline__ uint16_t to_storage16(float v, uint32_t prec) {
    return prec == SLOSH_PRECISION_FP16_STORAGE ? __half_as_ushort(__float2half_rn(v)) : __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
__device__ __forceinline__ void lv_st(float* a, uint32_t i, uint32_t prec, float v) {
    if (prec == SLOSH_PRECISION_FP32) a[i] = v;
    else reinterpret_cast<uint16_t*>(a)[i] = to_storage16(v, prec);
}

// Scale of the V-cycle's coarse levels with 16-bit storage: the restriction from level 0 multiplies by a power of
// two that brings the level-0 residual's norm (||r||^2 in scalars[5] when a V-cycle starts) to about 1, and the
// prolongation back to level 0 divides by it, so FP16's narrow exponent range holds the coarse values without
// flushing small ones; the V-cycle is linear and a power of two scales exactly. 1 with FP32 storage.
__device__ __forceinline__ float coarse_scale(const MGState& m) {
    if (m.lv[1].prec == SLOSH_PRECISION_FP32) return 1.0f;
    const double rr = m.scalars[5];
    int e = rr > 0.0 ? -ilogb(sqrt(rr)) : 0;
    e = max(-60, min(60, e));
    return ldexpf(1.0f, e);
}
// Coarse-level stencil word bits (k_level_words): bits 0-5 fluid neighbour, 6 fluid, 7 red, 8-13 non-solid neighbour.
constexpr uint32_t CW_FLUID = 1u << 6, CW_RED = 1u << 7, CW_NONSOLID_SHIFT = 8u;
// Level 0's over-relaxed sweep value x + w (x_GS - x) with w = mg_smoother_weight, and its red initialisation (one
// red half-sweep from zero) w x_GS; w == 1 leaves the reference's Gauss-Seidel value x_GS.
__device__ __forceinline__ float relax0(const MGState& m, float x_old, float gs) {
    return m.smooth_weight != 1.0f ? x_old + m.smooth_weight * (gs - x_old) : gs;
}
__device__ __forceinline__ float red_init0(const MGState& m, float gs) { return m.smooth_weight != 1.0f ? m.smooth_weight * gs : gs; }
__device__ __forceinline__ uint32_t lin3(int3 c, int3 dim) { return uint32_t(c.x + dim.x * (c.y + dim.y * c.z)); }
__device__ __forceinline__ int3 coord3(uint32_t i, int3 dim) {
    return make_int3(int(i % uint32_t(dim.x)), int((i / uint32_t(dim.x)) % uint32_t(dim.y)), int(i / uint32_t(dim.x * dim.y)));
}
__device__ __forceinline__ bool inside3(int3 c, int3 dim) {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < dim.x && c.y < dim.y && c.z < dim.z;
}
__device__ __forceinline__ bool is_red(int3 c) { return (uint32_t(c.x + c.y + c.z) & 1u) == 0u; }
// The iteration kernels carry no "solve finished" test: they are only ever issued while the solve runs
// (the graph's WHILE node runs its body while PCGInit / UpdatePR set the condition; the host loop reads
// the done flag before issuing each iteration), so a test would only put a dependent load in front of
// every kernel.

// Level-0 stencil (ghost-fluid diagonal DiagF + epsilon, sum of fluid neighbours of buf).
__device__ __forceinline__ void stencil0(const Dev& d, const float* buf, uint32_t i, int3 c, float& diag, float& sum) {
    sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        if (!in_grid(d, add3(c, nbr_off(n)))) continue;
        const uint32_t ni = nbr_index(d, i, c, n);
        if ((d.cell_type[ni] & CELL_TYPE_MASK) == CELL_FLUID) sum = sum + buf[ni];
    }
    diag = d.cell_diag[i] + DIAG_EPSILON;
}

// Shared-memory layout of the tail levels (byte offsets; every array padded to 4 cells, so each starts
// on 16 bytes): per level x, b, diag (f32), word (u16), colour list (u32; red then black). Level `tail`'s
// x and b come first. The same layout is used for the per-solve image in global memory.
struct TailOffsets {
    uint32_t x, b, diag, word, list;
};
__host__ __device__ __forceinline__ uint32_t tail_pad4(uint32_t cells) { return (cells + 3u) & ~3u; }
__host__ __device__ __forceinline__ TailOffsets tail_offsets(const MGState& m, int tail, int level, uint32_t* total) {
    uint32_t off = 0;
    TailOffsets o{};
    for (int l = tail; l < m.num_levels; ++l) {
        const uint32_t c4 = tail_pad4(m.lv[l].cells);
        TailOffsets t;
        t.x = off; off += c4 * 4u;
        t.b = off; off += c4 * 4u;
        t.diag = off; off += c4 * 4u;
        t.word = off; off += (c4 * 2u + 15u) & ~15u;
        t.list = off; off += c4 * 4u;
        if (l == level) o = t;
    }
    if (total) *total = off;
    return o;
}

// ---- canonical FP64 reduction ---------------------------------------------------------------------
struct DotSmem {
    double w8[GRID_THREADS / 32];
    double lanes[1024];
    double w32[32];
    uint32_t last;
};

// Final reduction over n brick partials: lanes t = 0..1023 sum entries t, t + 1024, ... in order, each
// group of 32 lanes folds with shfl_down 16..1, and the 32 group results are added in order.
__device__ double final_reduce(const double* partials, uint32_t n, DotSmem& sm) {
    // Thread x owns lanes x + 256 k (k = 0..3); lane t adds partials t, t + 1024, ... in that order.
    // The loads of four 1024-partial rounds are issued before any of them is added, so the pass costs
    // about one L2 round trip per 4096 partials instead of one per partial of a lane.
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t base = 0; base < n; base += 4096u) {
        double v[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t e = base + 1024u * uint32_t(r) + threadIdx.x + 256u * uint32_t(k);
                v[r][k] = e < n ? __ldcg(partials + e) : 0.0;
            }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (base + 1024u * uint32_t(r) + threadIdx.x + 256u * uint32_t(k) < n) acc[k] = acc[k] + v[r][k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) sm.lanes[threadIdx.x + 256u * uint32_t(k)] = acc[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int lw = warp + 8 * k;
        const double v = warp_fold(sm.lanes[lw * 32 + lane]);
        if (lane == 0) sm.w32[lw] = v;
    }
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0) {
        total = sm.w32[0];
        for (int w = 1; w < 32; ++w) total = total + sm.w32[w];
    }
    return total;
}

// Visits the cells of level l (1..3) that lie in the active bricks' footprints: fn(ci, c). Levels
// whose cells are coarser than a brick are scanned densely.
// Thread t0 of `stride` threads takes footprint cells t0, t0 + stride, ...
template <class Fn>
__device__ __forceinline__ void for_footprint_span(const Dev& d, const MGLevel& L, int l, uint32_t t0, uint32_t stride, Fn fn) {
    if (l > 3) {
        for (uint32_t i = t0; i < L.cells; i += stride) fn(i, coord3(i, L.dim));
        return;
    }
    const int side = 8 >> l;
    const uint32_t per = uint32_t(side * side * side);
    const uint32_t count = d.active_bricks[0];
    for (uint32_t t = t0;; t += stride) {
        const uint32_t e = t / per, lc = t % per;
        // The brick index is loaded before the bound is known (clamped into the list), so it overlaps
        // the load of the active count.
        const uint32_t brick = d.active_bricks[1u + min(e, d.num_bricks - 1u)];
        if (e >= count) break;
        const int3 bc = brick_coord_of(d, brick);
        const int3 c = make_int3(bc.x * side + int(lc % uint32_t(side)), bc.y * side + int((lc / uint32_t(side)) % uint32_t(side)),
                                 bc.z * side + int(lc / uint32_t(side * side)));
        if (inside3(c, L.dim)) fn(lin3(c, L.dim), c);
    }
}
// The footprint cells of one colour (parity 0: red, (x + y + z) even; 1: black) of level l = 1 or 2, whose brick
// footprints have an even side, so a cell's colour is that of its position inside the footprint: item j of a brick
// is (2 (j mod s/2) + ((y + z + parity) & 1), y, z) with y = (j / (s/2)) mod s, z = j / (s^2/2). A sweep then
// visits only the cells it updates: half the threads of the all-cell walk.
template <class Fn>
__device__ __forceinline__ void for_footprint_colour(const Dev& d, const MGLevel& L, int l, uint32_t parity, Fn fn) {
    const uint32_t side = uint32_t(8 >> l), half = side / 2u;
    const uint32_t per = side * side * half;
    const uint32_t count = d.active_bricks[0];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;; t += gridDim.x * blockDim.x) {
        const uint32_t e = t / per, j = t % per;
        const uint32_t brick = d.active_bricks[1u + min(e, d.num_bricks - 1u)];
        if (e >= count) break;
        const int3 bc = brick_coord_of(d, brick);
        const uint32_t y = (j / half) % side, z = j / (half * side);
        const uint32_t x = 2u * (j % half) + ((y + z + parity) & 1u);
        const int3 c = make_int3(bc.x * int(side) + int(x), bc.y * int(side) + int(y), bc.z * int(side) + int(z));
        if (inside3(c, L.dim)) fn(lin3(c, L.dim), c);
    }
}
template <class Fn>
__device__ __forceinline__ void for_footprint(const Dev& d, const MGLevel& L, int l, Fn fn) {
    for_footprint_span(d, L, l, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, fn);
}

// ---- level-0 stencil words ------------------------------------------------------------------------
// The cell types do not change during a solve, so PCGInit stores per level-0 cell one byte: bits 0-5
// = neighbour n (-x, +x, -y, +y, -z, +z) is fluid, bit 6 = the cell is fluid, bit 7 = red, and per
// active brick the slots of its 6 face neighbours. The level-0 passes then load only the word and
// issue all neighbour loads at once, instead of a type -> brick table -> value chain per neighbour.
constexpr uint32_t W_FLUID = 1u << 6, W_RED = 1u << 7;

__device__ __forceinline__ uint32_t l0_nbr(uint32_t i, uint32_t l, int n, const uint32_t* ns) {
    switch (n) {
        case 0: return (l & 7u) ? i - 1u : ns[0] * BRICK_CELLS + l + 7u;
        case 1: return ((l & 7u) != 7u) ? i + 1u : ns[1] * BRICK_CELLS + l - 7u;
        case 2: return (l & 56u) ? i - 8u : ns[2] * BRICK_CELLS + l + 56u;
        case 3: return ((l & 56u) != 56u) ? i + 8u : ns[3] * BRICK_CELLS + l - 56u;
        case 4: return (l & 448u) ? i - 64u : ns[4] * BRICK_CELLS + l + 448u;
        default: return ((l & 448u) != 448u) ? i + 64u : ns[5] * BRICK_CELLS + l - 448u;
    }
}

// ---- level-0 passes in half rows --------------------------------------------------------------------
// One warp per active brick (nbr_slots[8 e + 0..5] = face-neighbour slots, [8 e + 6] = own slot, [8 e + 7]
// = brick index, stored by PCGInit). In round k = 0..3 lane t takes the 4 consecutive cells x = 4h .. 4h+3
// of row y in plane z (h = t & 1, y = (t >> 1) & 7, z = 2k + (t >> 4)): one 16-byte load or store per
// array, the +-y and +-z neighbours as 16-byte loads of the adjacent rows (of the face-neighbour brick at
// the brick's faces; a missing neighbour is the all-zero null slot), the +-x neighbours inside the row from
// the lane's own quad or its partner lane t ^ 1, and one scalar load from the -x (h = 0) or +x (h = 1)
// neighbour brick. A brick's dot-product partial is the canonical per-brick tree: lane t adds its cells
// round by round, x ascending, starting from 0.0, and the lanes fold with shfl_down 16..1.
struct Geo {
    uint32_t i, l, h, y, z;  // pool and local index of the quad's first cell; half, row, plane
    uint32_t b;              // the brick (w4_pass only)
};
__device__ __forceinline__ Geo geo_of(uint32_t base, uint32_t lane, uint32_t k, uint32_t brick = 0u) {
    Geo g;
    g.b = brick;
    g.h = lane & 1u;
    g.y = (lane >> 1) & 7u;
    g.z = 2u * k + (lane >> 4);
    g.l = 4u * g.h + 8u * g.y + 64u * g.z;
    g.i = base + g.l;
    return g;
}
__device__ __forceinline__ float4 ld4(const float* q) { return *reinterpret_cast<const float4*>(q); }
__device__ __forceinline__ void st4(float* q, const float (&v)[4]) { *reinterpret_cast<float4*>(q) = make_float4(v[0], v[1], v[2], v[3]); }
__device__ __forceinline__ float comp(const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }
__device__ __forceinline__ uint32_t quad_words(const MGState& m, const Geo& g) { return *reinterpret_cast<const uint32_t*>(m.word + g.i); }
__device__ __forceinline__ uint32_t word_of(uint32_t w4, int j) { return (w4 >> (8 * j)) & 0xFFu; }

struct Q6 {  // a quad of one array and its face neighbours
    float4 c, ym, yp, zm, zp;
    float xb;  // h = 0: cell (7, y, z) of the -x brick; h = 1: cell (0, y, z) of the +x brick
};
__device__ __forceinline__ Q6 load_q6(const float* buf, const Geo& g, const uint32_t* ns) {
    Q6 q;
    q.c = ld4(buf + g.i);
    q.ym = ld4(buf + (g.y > 0u ? g.i - 8u : ns[2] * BRICK_CELLS + g.l + 56u));
    q.yp = ld4(buf + (g.y < 7u ? g.i + 8u : ns[3] * BRICK_CELLS + g.l - 56u));
    q.zm = ld4(buf + (g.z > 0u ? g.i - 64u : ns[4] * BRICK_CELLS + g.l + 448u));
    q.zp = ld4(buf + (g.z < 7u ? g.i + 64u : ns[5] * BRICK_CELLS + g.l - 448u));
    q.xb = buf[g.h == 0u ? ns[0] * BRICK_CELLS + g.l + 7u : ns[1] * BRICK_CELLS + g.l - 4u];
    return q;
}
// The partner lane's last (pw) and first (px) cell; every lane shuffles before any per-cell branch.
struct X2 {
    float pw, px;
};
__device__ __forceinline__ X2 partner(const Q6& q) {
    X2 x;
    x.pw = __shfl_xor_sync(0xFFFFFFFFu, q.c.w, 1);
    x.px = __shfl_xor_sync(0xFFFFFFFFu, q.c.x, 1);
    return x;
}
// Neighbour values of cell j of the quad, in the order -x, +x, -y, +y, -z, +z.
__device__ __forceinline__ void nbrs6(const Q6& q, const X2& x, uint32_t h, int j, float n[6]) {
    n[0] = j == 0 ? (h ? x.pw : q.xb) : comp(q.c, j - 1);
    n[1] = j == 3 ? (h ? q.xb : x.px) : comp(q.c, j + 1);
    n[2] = comp(q.ym, j);
    n[3] = comp(q.yp, j);
    n[4] = comp(q.zm, j);
    n[5] = comp(q.zp, j);
}

// load(g, ns) gathers a round's values; apply(g, vals, v0[4], v1[4]) computes and stores one round and
// yields the cells' dot terms. The loads of B rounds are issued before any of them is applied. With
// NDOT > 0 the last CTA reduces the brick partials (canonical tree) and calls store(t0, t1) in thread 0.
template <int NDOT, int B, class Load, class Apply, class Store>
__device__ __forceinline__ void w4_pass(const Dev& d, const MGState& m, uint32_t counter, Load load, Apply apply, Store store) {
    __shared__ DotSmem sm;
    const uint32_t active = d.active_bricks[0];
    const uint32_t cap = d.num_pool_bricks;
    const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
    for (uint32_t e = blockIdx.x * wpb + (threadIdx.x >> 5); e < active; e += gridDim.x * wpb) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        const uint32_t base = s1.z * BRICK_CELLS;
        double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
        for (uint32_t k0 = 0; k0 < 4u; k0 += uint32_t(B)) {
            decltype(load(Geo{}, ns)) vals[B];
#pragma unroll
            for (int b = 0; b < B; ++b) vals[b] = load(geo_of(base, lane, k0 + uint32_t(b), s1.w), ns);
#pragma unroll
            for (int b = 0; b < B; ++b) {
                double v0[4] = {0.0, 0.0, 0.0, 0.0}, v1[4] = {0.0, 0.0, 0.0, 0.0};
                apply(geo_of(base, lane, k0 + uint32_t(b), s1.w), vals[b], v0, v1);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc0 = acc0 + v0[j];
                    acc1 = acc1 + v1[j];
                }
            }
        }
        if (NDOT > 0) {
            const double t0 = warp_fold(acc0);
            if (lane == 0) m.partials[e] = t0;
        }
        if (NDOT > 1) {
            const double t1 = warp_fold(acc1);
            if (lane == 0) m.partials[cap + e] = t1;
        }
    }
    if (NDOT == 0) return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sm.last = (atomicAdd(m.counters + counter, 1u) == gridDim.x - 1u) ? 1u : 0u;
    __syncthreads();
    if (sm.last) {
        __threadfence();
        const double r0 = final_reduce(m.partials, active, sm);
        __syncthreads();
        double r1 = 0.0;
        if (NDOT > 1) r1 = final_reduce(m.partials + cap, active, sm);
        if (threadIdx.x == 0) {
            store(r0, r1);
            m.counters[counter] = 0u;
        }
    }
}

// The 256 black cells ((x + y + z) odd) of every active brick, one warp per brick, 8 cells per lane:
// round k takes plane z = k, row y = lane >> 2 and x = 2 (lane & 3) + ((y + z + 1) & 1), so no lane
// idles on a red cell. prep(brick, lane) runs once per brick before its cells (all lanes of the warp);
// the loads of a group of B cells are issued before any of them is applied.
__device__ __forceinline__ uint32_t black_local(uint32_t lane, uint32_t k) {
    const uint32_t y = lane >> 2;
    return 2u * (lane & 3u) + ((y + k + 1u) & 1u) + 8u * y + 64u * k;
}
template <int B, class Prep, class Load, class Apply>
__device__ __forceinline__ void w0_black(const Dev& d, const MGState& m, Prep prep, Load load, Apply apply) {
    const uint32_t active = d.active_bricks[0];
    const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
    for (uint32_t e = blockIdx.x * wpb + (threadIdx.x >> 5); e < active; e += gridDim.x * wpb) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        const uint32_t base = s1.z * BRICK_CELLS;
        prep(s1.w, lane);
        for (uint32_t k0 = 0; k0 < 8u; k0 += B) {
            decltype(load(0u, 0u, ns)) vals[B];
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const uint32_t l = black_local(lane, k0 + uint32_t(b));
                vals[b] = load(base + l, l, ns);
            }
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const uint32_t l = black_local(lane, k0 + uint32_t(b));
                apply(base + l, l, vals[b]);
            }
        }
    }
}

struct Nb6 {
    uint32_t w;
    float c0, c1, c2;
    float n[6];
};
__device__ __forceinline__ float nb_sum(const float* v, uint32_t w) {
    float sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n)
        if ((w >> n) & 1u) sum = sum + v[n];
    return sum;
}

// What a sweep or the restriction reads of a quad: z with its neighbours, r, the diagonal and the words.
struct SweepQ {
    Q6 z;
    float4 r, dg;
    uint32_t w;
    float pa, pb;  // PROLONGED: the prolongation terms of cells 0-1 and 2-3 (their level-1 parents)
};
// PROLONGED (the first red sweep after k_prolong_smooth0 with an over-relaxed smoother): the red cells' stored
// z lacks the prolongation, which the fused kernel adds only to the values it reads, so the sweep rebuilds each
// red cell's prolonged value z + x_parent / coarse scale (fluid parents) from level 1, as k_prolong_smooth0 does.
template <bool PROLONGED = false>
__device__ __forceinline__ SweepQ load_sweep(const Dev& d, const MGState& m, const Geo& g, const uint32_t* ns) {
    SweepQ v;
    v.z = load_q6(m.z, g, ns);
    v.r = ld4(m.r + g.i);
    v.dg = ld4(d.cell_diag + g.i);
    v.w = quad_words(m, g);
    v.pa = v.pb = 0.0f;
    if (PROLONGED) {
        const MGLevel C = m.lv[1];
        const float ivs = 1.0f / coarse_scale(m);  // a power of two: exact
        const int3 bc = brick_coord_of(d, g.b);
        float pv[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int3 c = make_int3(bc.x * 4 + 2 * int(g.h) + k, bc.y * 4 + int(g.y >> 1), bc.z * 4 + int(g.z >> 1));
            pv[k] = 0.0f;
            if (inside3(c, C.dim)) {
                const uint32_t ci = lin3(c, C.dim);
                const float x = lv_ld(C.x, ci, C.prec);
                pv[k] = (C.word[ci] & CW_FLUID) ? x * ivs : 0.0f;
            }
        }
        v.pa = pv[0];
        v.pb = pv[1];
    }
    return v;
}

__device__ __forceinline__ float ratio_f(double num, double den) { return fabs(den) > 1e-30 ? float(num / den) : 0.0f; }

// ---- solve setup: iteration state in ctl[] --------------------------------------------------------------
__global__ void k_solve_setup(MGState m, uint32_t limit, uint32_t tol_mode, double tol) {
    pdl_entry();
    m.ctl[0] = 0u;        // completed iterations
    m.ctl[1] = limit;     // iteration limit
    m.ctl[2] = tol_mode;  // 1: stop at ||r|| <= tol ||b||
    m.ctl[3] = 0u;        // done
    m.scalars[8] = tol;
}

// ---- MGBuildTypeCS: coarse cell = air if any child is air, else fluid if any child is fluid ---------------
__device__ __forceinline__ void build_type_cell(const Dev& d, const MGLevel& fine, const MGLevel& coarse, int fine_is_pool, uint32_t ci,
                                                int3 c) {
    bool any_air = false, any_fluid = false;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int3 f = make_int3(c.x * 2 + (o & 1), c.y * 2 + ((o >> 1) & 1), c.z * 2 + ((o >> 2) & 1));
        if (!inside3(f, fine.dim)) continue;
        const uint32_t t = (fine_is_pool ? d.cell_type[cell_index(d, f)] : fine.type[lin3(f, fine.dim)]) & CELL_TYPE_MASK;
        any_air = any_air || t == CELL_AIR;
        any_fluid = any_fluid || t == CELL_FLUID;
    }
    coarse.type[ci] = any_air ? CELL_AIR : (any_fluid ? CELL_FLUID : CELL_SOLID);
}
__global__ void k_build_type(Dev d, MGLevel fine, MGLevel coarse, int fine_is_pool) {
    pdl_entry();
    const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= coarse.cells) return;
    build_type_cell(d, fine, coarse, fine_is_pool, ci, coord3(ci, coarse.dim));
}
// Levels 1-3 over the active bricks' footprints only; the rest of the level was cleared to air (0) before, which is
// what the dense build gives cells over unallocated bricks (their fine cells are the null brick's air).
__global__ void k_build_type_fp(Dev d, MGLevel fine, MGLevel coarse, int lc) {
    pdl_entry();
    for_footprint(d, coarse, lc, [&](uint32_t ci, int3 c) { build_type_cell(d, fine, coarse, lc == 1 ? 1 : 0, ci, c); });
}

// Levels 1 to top (top <= 3) in one launch, one warp per active brick: a coarse type is air when any of its level-0
// descendants inside the grid is air, else fluid when any is fluid, else solid -- the rule above applied level by
// level gives the same (every cell inside a level has a child inside the level below), and the descendants of a
// brick's footprint cells at levels 1-3 are the brick's own 512 cells. Lane t holds cells l = t + 32 k (k = 0..15):
// x = t & 7, y = (t >> 3) + 4 (k & 1), z = k >> 1, so the children of one coarse cell are combined across lanes
// t ^ 1, t ^ 2, t ^ 4 (x), t ^ 8, t ^ 16 and k ^ 1 (y), k ^ 2, k ^ 4, k ^ 8 (z).
__device__ __forceinline__ uint32_t type_of_flags(uint32_t f) { return (f & 1u) ? CELL_AIR : ((f & 2u) ? CELL_FLUID : CELL_SOLID); }
__global__ void __launch_bounds__(256) k_build_types_fp13(Dev d, MGState m, int top) {
    pdl_entry();
    const uint32_t active = d.active_bricks[0];
    const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
    for (uint32_t e = blockIdx.x * wpb + (threadIdx.x >> 5); e < active; e += gridDim.x * wpb) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
        uint32_t g[16];  // bit 0: some descendant is air, bit 1: some is fluid
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const uint32_t l = lane + 32u * uint32_t(k);
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            const uint32_t t = in_grid(d, c) ? (d.cell_type[slot * BRICK_CELLS + l] & CELL_TYPE_MASK) : CELL_SOLID;
            g[k] = (t == CELL_AIR ? 1u : 0u) | (t == CELL_FLUID ? 2u : 0u);
        }
        const uint32_t x = lane & 7u, ylo = lane >> 3;
        // level 1: x pairs (t ^ 1), y pairs (t ^ 8), z pairs (k ^ 2)
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & 2) continue;
            uint32_t v = g[k] | g[k ^ 2];
            v |= __shfl_xor_sync(0xFFFFFFFFu, v, 1);
            v |= __shfl_xor_sync(0xFFFFFFFFu, v, 8);
            g[k] = v;
            const MGLevel& L = m.lv[1];
            const uint32_t y = ylo + 4u * uint32_t(k & 1), z = uint32_t(k) >> 1;
            const int3 c = make_int3(bc.x * 4 + int(x >> 1), bc.y * 4 + int(y >> 1), bc.z * 4 + int(z >> 1));
            if ((lane & 9u) == 0u && inside3(c, L.dim)) L.type[lin3(c, L.dim)] = type_of_flags(v);
        }
        if (top < 2) continue;
        // level 2: with the above, x quads (t ^ 2), y quads (t ^ 16), z quads (k ^ 4)
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k & 6) continue;
            uint32_t v = g[k] | g[k ^ 4];
            v |= __shfl_xor_sync(0xFFFFFFFFu, v, 2);
            v |= __shfl_xor_sync(0xFFFFFFFFu, v, 16);
            g[k] = v;
            const MGLevel& L = m.lv[2];
            const uint32_t y = ylo + 4u * uint32_t(k & 1), z = uint32_t(k) >> 1;
            const int3 c = make_int3(bc.x * 2 + int(x >> 2), bc.y * 2 + int(y >> 2), bc.z * 2 + int(z >> 2));
            if ((lane & 27u) == 0u && inside3(c, L.dim)) L.type[lin3(c, L.dim)] = type_of_flags(v);
        }
        if (top < 3) continue;
        // level 3: the whole brick
        uint32_t v = g[0] | g[1] | g[8] | g[9];
        v = __reduce_or_sync(0xFFFFFFFFu, v);
        const MGLevel& L = m.lv[3];
        if (lane == 0u && inside3(bc, L.dim)) L.type[lin3(bc, L.dim)] = type_of_flags(v);
    }
}
// The words of levels 1 to top (top <= 3) in one launch: each thread walks the three footprints in turn.
__global__ void k_level_words_fp13(Dev d, MGState m, int top);

// ---- coarse-level stencil words (once per solve, after the coarse types) -----------------------------------

__device__ __forceinline__ void level_word_cell(const MGLevel& L, uint32_t i, int3 c) {
    uint32_t w = (L.type[i] & CELL_TYPE_MASK) == CELL_FLUID ? CW_FLUID : 0u;
    if (is_red(c)) w |= CW_RED;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const int3 nb = add3(c, nbr_off(n));
        if (!inside3(nb, L.dim)) continue;
        const uint32_t t = L.type[lin3(nb, L.dim)] & CELL_TYPE_MASK;
        if (t == CELL_FLUID) w |= 1u << n;
        if (t != CELL_SOLID) w |= 1u << (CW_NONSOLID_SHIFT + n);
    }
    L.word[i] = uint16_t(w);
}
__global__ void k_level_words(MGLevel L) {
    pdl_entry();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.cells) return;
    level_word_cell(L, i, coord3(i, L.dim));
}
// Levels 1-3: only the footprint cells' words are read (by the footprint passes and their neighbours' sums).
__global__ void k_level_words_fp(Dev d, MGLevel L, int l) {
    pdl_entry();
    for_footprint(d, L, l, [&](uint32_t i, int3 c) { level_word_cell(L, i, c); });
}
__global__ void k_level_words_fp13(Dev d, MGState m, int top) {
    pdl_entry();
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (int l = 1; l <= top; ++l) {
        const MGLevel& L = m.lv[l];
        for_footprint_span(d, L, l, t0, stride, [&](uint32_t i, int3 c) { level_word_cell(L, i, c); });
    }
}
// DiagEpsilon plus one per non-solid neighbour, added in neighbour order like FINE_STENCIL.
__device__ __forceinline__ float word_diag(uint32_t w) {
    float d = DIAG_EPSILON;
#pragma unroll
    for (int n = 0; n < 6; ++n)
        if ((w >> (CW_NONSOLID_SHIFT + n)) & 1u) d = d + 1.0f;
    return d;
}
// Sum of x over the fluid neighbours of a dense global level, in neighbour order. All six values are
// loaded unconditionally (indices clamped into the level, so a missing neighbour reads some cell of
// the level) and then selected by the word, so the loads overlap the word's.
template <bool CG = false>
__device__ __forceinline__ float word_sum_g(const float* x, uint32_t prec, uint32_t w, uint32_t i, uint32_t dx, uint32_t dxy,
                                            uint32_t last) {
    const uint32_t off[6] = {i - 1u, i + 1u, i - dx, i + dx, i - dxy, i + dxy};
    float v[6];
#pragma unroll
    for (int n = 0; n < 6; ++n) v[n] = lvx<CG>(x, min(off[n], last), prec);
    float sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n)
        if ((w >> n) & 1u) sum = sum + v[n];
    return sum;
}
// Sum of x over the fluid neighbours (dense level), in neighbour order.
__device__ __forceinline__ float word_sum(const float* x, uint32_t w, uint32_t i, uint32_t dx, uint32_t dxy) {
    const uint32_t off[6] = {i - 1u, i + 1u, i - dx, i + dx, i - dxy, i + dxy};
    float v[6];
#pragma unroll
    for (int n = 0; n < 6; ++n) v[n] = ((w >> n) & 1u) ? x[off[n]] : 0.0f;
    float sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n)
        if ((w >> n) & 1u) sum = sum + v[n];
    return sum;
}

// ---- PCGInitCS (+ ||r0||^2 and ||b||^2, and the decision whether any iteration runs) ----------------------
// First stores the solve's stencil words and each active brick's neighbour and own slots; the residual
// pass itself reads the cell types directly (its neighbours' words may not be written yet).
__global__ void __launch_bounds__(GRID_THREADS) k_pcg_words(Dev d, MGState m) {
    pdl_entry();
    const uint32_t active = d.active_bricks[0];
    const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
    for (uint32_t e = blockIdx.x * wpb + (threadIdx.x >> 5); e < active; e += gridDim.x * wpb) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
        uint32_t mine = 0u;  // lanes 0-5: the slot of face neighbour `lane` (0 = outside the grid or unallocated)
        if (lane < 6) {
            const int3 nb = add3(bc, nbr_off(int(lane)));
            const bool in = nb.x >= 0 && nb.y >= 0 && nb.z >= 0 && nb.x < d.brick_dim.x && nb.y < d.brick_dim.y && nb.z < d.brick_dim.z;
            mine = in ? __ldg(d.brick_table + brick_index_of(d, nb)) : 0u;
            m.nbr_slots[8u * e + lane] = mine;
        } else if (lane == 6) {
            m.nbr_slots[8u * e + 6u] = slot;
        } else if (lane == 7) {
            m.nbr_slots[8u * e + 7u] = brick;
        }
        uint32_t ns[6];
#pragma unroll
        for (int n = 0; n < 6; ++n) ns[n] = __shfl_sync(0xFFFFFFFFu, mine, n);
        // the half-row quads of the level-0 passes: per round the types of the lane's 4 cells and of the adjacent
        // rows' 4 (16-byte loads; across a face through the face neighbour's slot, an unallocated brick being the
        // null slot of air cells), the +-x neighbours inside the row from the partner lane; the 4 words go out as
        // one 32-bit store
        const float* types = reinterpret_cast<const float*>(d.cell_type);  // loaded and shuffled as bits only
        const uint32_t base = slot * BRICK_CELLS;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            const Geo g = geo_of(base, lane, k);
            const Q6 q = load_q6(types, g, ns);
            const X2 x = partner(q);
            uint32_t packed = 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int3 c = make_int3(bc.x * 8 + int(4u * g.h) + j, bc.y * 8 + int(g.y), bc.z * 8 + int(g.z));
                uint32_t w = 0u;
                if (in_grid(d, c)) {
                    float n[6];
                    nbrs6(q, x, g.h, j, n);
                    if ((__float_as_uint(comp(q.c, j)) & CELL_TYPE_MASK) == CELL_FLUID) w |= W_FLUID;
                    if (is_red(c)) w |= W_RED;
#pragma unroll
                    for (int m6 = 0; m6 < 6; ++m6)
                        if (in_grid(d, add3(c, nbr_off(m6))) && (__float_as_uint(n[m6]) & CELL_TYPE_MASK) == CELL_FLUID) w |= 1u << m6;
                }
                packed |= w << (8 * j);
            }
            *reinterpret_cast<uint32_t*>(m.word + g.i) = packed;
        }
    }
}
__global__ void __launch_bounds__(GRID_THREADS) k_pcg_init(Dev d, MGState m, const float* __restrict__ p, const float* __restrict__ div,
                                                           unsigned long long handle) {
    pdl_entry();
    struct V {
        Q6 p;
        float4 dv, dg;
        uint32_t w;
    };
    w4_pass<2, 1>(d, m, 0,
        [&](const Geo& g, const uint32_t* ns) {
            V v;
            v.p = load_q6(p, g, ns);
            v.dv = ld4(div + g.i);
            v.dg = ld4(d.cell_diag + g.i);
            v.w = quad_words(m, g);
            return v;
        },
        [&](const Geo& g, const V& v, double* v0, double* v1) {
            const X2 x = partner(v.p);
            float r[4], z[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                r[j] = 0.0f;
                z[j] = 0.0f;
                if (!(w & W_FLUID)) continue;
                const float diag = comp(v.dg, j) + DIAG_EPSILON;
                float n[6];
                nbrs6(v.p, x, g.h, j, n);
                const float b = -comp(v.dv, j);
                const float ri = b - (diag * comp(v.p.c, j) - nb_sum(n, w));
                r[j] = ri;
                z[j] = (w & W_RED) ? red_init0(m, ri / diag) : 0.0f;
                v0[j] = double(ri * ri);
                v1[j] = double(b * b);
            }
            st4(m.r + g.i, r);
            st4(m.z + g.i, z);
        },
        [&](double rr, double bb) {
            m.scalars[5] = rr;
            m.scalars[4] = bb;
            const double rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
            const bool run = m.ctl[1] > 0u && !(m.ctl[2] != 0u && rel <= m.scalars[8]);
            if (!run) m.ctl[3] = 1u;
            if (handle) cudaGraphSetConditional(handle, run ? 1u : 0u);
        });
}

// ---- MGSmoothCS on level 0 (z as x, r as b); with dot the r.z reduction shifts rho -----------------------
// What a black sweep reads of a cell: word, r, diagonal and the six neighbours' z (c1 unused).
__device__ __forceinline__ Nb6 load_black(const Dev& d, const MGState& m, uint32_t i, uint32_t l, const uint32_t* ns) {
    Nb6 v;
    v.w = m.word[i];
    v.c0 = m.r[i];
    v.c1 = m.smooth_weight != 1.0f ? m.z[i] : 0.0f;  // the cell's own value, for the over-relaxed update
    v.c2 = d.cell_diag[i];
#pragma unroll
    for (int n = 0; n < 6; ++n) v.n[n] = m.z[l0_nbr(i, l, n, ns)];
    return v;
}

// Red sweep; with DOT also rho = r . z over all cells (red: the new value, black: the current z), which
// shifts rho. Cells the sweep does not update are stored back unchanged (each cell belongs to one warp's
// brick).
template <bool DOT, bool PROLONGED = false>
__global__ void __launch_bounds__(GRID_THREADS, 3) k_smooth0(Dev d, MGState m) {
    pdl_entry();
    w4_pass<DOT ? 1 : 0, 1>(d, m, 1,
        [&](const Geo& g, const uint32_t* ns) { return load_sweep<PROLONGED>(d, m, g, ns); },
        [&](const Geo& g, const SweepQ& v, double* v0, double*) {
            const X2 x = partner(v.z);
            float out[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                const float zj = comp(v.z.c, j), rj = comp(v.r, j);
                out[j] = zj;
                if (!(w & W_FLUID)) continue;
                if (w & W_RED) {
                    float n[6];
                    nbrs6(v.z, x, g.h, j, n);
                    const float val = (rj + nb_sum(n, w)) / (comp(v.dg, j) + DIAG_EPSILON);
                    out[j] = relax0(m, PROLONGED ? zj + (j < 2 ? v.pa : v.pb) : zj, val);
                    v0[j] = double(rj * out[j]);
                } else {
                    v0[j] = double(rj * zj);
                }
            }
            st4(m.z + g.i, out);
        },
        [&](double rho, double) { m.scalars[3] = m.scalars[0]; m.scalars[0] = rho; });
}

// Black sweep (no dot product).
__global__ void __launch_bounds__(GRID_THREADS) k_smooth0_black(Dev d, MGState m) {
    pdl_entry();
    w0_black<4>(d, m, [](uint32_t, uint32_t) {},
        [&](uint32_t i, uint32_t l, const uint32_t* ns) { return load_black(d, m, i, l, ns); },
        [&](uint32_t i, uint32_t, const Nb6& v) {
            if (!(v.w & W_FLUID)) return;
            m.z[i] = relax0(m, v.c1, (v.c0 + nb_sum(v.n, v.w)) / (v.c2 + DIAG_EPSILON));
        });
}

// ---- MGProlongCS (level 1 -> 0) fused with the following black sweep ------------------------------
// After the prolongation only the black sweep reads the prolonged values (of its red neighbours) and
// it overwrites the black cells; the red sweep that follows overwrites the red cells. So the black
// sweep reads z_n + x_c(parent of n) directly and nothing else needs to be written. Each warp first
// stages the level-1 correction of its brick's 4^3 parents and their face neighbours (a 6^3 block,
// x_c where the parent is fluid and 0 elsewhere) in shared memory. Adding +0 instead of skipping the
// addition changes at most the sign of a zero z_n, which the neighbour sum (started at +0) absorbs.
__global__ void __launch_bounds__(GRID_THREADS) k_prolong_smooth0(Dev d, MGState m) {
    pdl_entry();
    constexpr int WARPS = GRID_THREADS / 32;
    __shared__ float s_cx[WARPS][216];
    const MGLevel C = m.lv[1];
    const float ivs = 1.0f / coarse_scale(m);  // a power of two: exact
    float* cx = s_cx[threadIdx.x >> 5];
    w0_black<4>(d, m,
        [&](uint32_t brick, uint32_t lane) {
            const int3 bc = brick_coord_of(d, brick);
            __syncwarp();
            float v[7];
#pragma unroll
            for (int r = 0; r < 7; ++r) {
                const uint32_t j = lane + 32u * uint32_t(r);
                const int3 c = make_int3(bc.x * 4 - 1 + int(j % 6u), bc.y * 4 - 1 + int((j / 6u) % 6u), bc.z * 4 - 1 + int(j / 36u));
                v[r] = 0.0f;
                if (j < 216u && inside3(c, C.dim)) {
                    const uint32_t ci = lin3(c, C.dim);
                    const float x = lv_ld(C.x, ci, C.prec);
                    v[r] = (C.word[ci] & CW_FLUID) ? x * ivs : 0.0f;
                }
            }
#pragma unroll
            for (int r = 0; r < 7; ++r) {
                const uint32_t j = lane + 32u * uint32_t(r);
                if (j < 216u) cx[j] = v[r];
            }
            __syncwarp();
        },
        [&](uint32_t i, uint32_t l, const uint32_t* ns) { return load_black(d, m, i, l, ns); },
        [&](uint32_t i, uint32_t l, const Nb6& v) {
            if (!(v.w & W_FLUID)) return;
            const int x = int(l & 7u), y = int((l >> 3) & 7u), z = int(l >> 6);
            const int p = ((x >> 1) + 1) + 6 * ((y >> 1) + 1) + 36 * ((z >> 1) + 1);
            const int px = (x & 1) ? 1 : 0, py = (y & 1) ? 6 : 0, pz = (z & 1) ? 36 : 0;
            const int po[6] = {p - 1 + px, p + px, p - 6 + py, p + py, p - 36 + pz, p + pz};
            float sum = 0.0f;
#pragma unroll
            for (int n = 0; n < 6; ++n)
                if ((v.w >> n) & 1u) sum = sum + (v.n[n] + cx[po[n]]);
            m.z[i] = relax0(m, v.c1 + cx[p], (v.c0 + sum) / (v.c2 + DIAG_EPSILON));
        });
}

// Levels 1..3 through the active-brick footprints, with the per-solve stencil words; each pass is a
// per-cell body and a grid-wide kernel over the level's footprint.
// Sweep of one colour (want = CW_RED: red cells, 0: black cells) at cell i of level L.
template <bool CG = false>
__device__ __forceinline__ void smooth_fp_cell(const MGLevel& L, uint32_t i, uint32_t want) {
    const uint32_t dx = uint32_t(L.dim.x), dxy = uint32_t(L.dim.x * L.dim.y);
    const uint32_t w = L.word[i];
    const float b = lvx<CG>(L.b, i, L.prec);
    const float sum = word_sum_g<CG>(L.x, L.prec, w, i, dx, dxy, L.cells - 1u);
    if (!(w & CW_FLUID) || (w & CW_RED) != want) return;
    lv_st(L.x, i, L.prec, (b + sum) / word_diag(w));
}
// Restriction F -> C at coarse cell ci: b_c = scale x (sum of the fluid children's residuals), scale = 1/4 in
// the reference (times mg_correction_scale).
template <bool CG = false>
__device__ __forceinline__ void restrict_fp_cell(const MGLevel& F, const MGLevel& C, uint32_t ci, int3 c, float scale) {
    const uint32_t fdx = uint32_t(F.dim.x), fdxy = uint32_t(F.dim.x * F.dim.y);
    const uint32_t flast = F.cells - 1u;
    // Every child's word, b, x and neighbours are loaded before any of them is tested.
    const uint32_t cw = C.word[ci];
    float res[8];
    uint32_t fl = 0u;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int3 f = make_int3(c.x * 2 + (o & 1), c.y * 2 + ((o >> 1) & 1), c.z * 2 + ((o >> 2) & 1));
        const bool in = inside3(f, F.dim);
        const uint32_t fi = in ? lin3(f, F.dim) : 0u;
        const uint32_t w = F.word[fi];
        const float r = lvx<CG>(F.b, fi, F.prec) - (word_diag(w) * lvx<CG>(F.x, fi, F.prec) - word_sum_g<CG>(F.x, F.prec, w, fi, fdx, fdxy, flast));
        res[o] = 0.0f;
        if (in && (w & CW_FLUID)) {
            fl |= 1u << o;
            res[o] = r;
        }
    }
    if (!(cw & CW_FLUID)) { lv_st(C.b, ci, C.prec, 0.0f); lv_st(C.x, ci, C.prec, 0.0f); return; }
    float sum = 0.0f;
#pragma unroll
    for (int o = 0; o < 8; ++o)
        if ((fl >> o) & 1u) sum = sum + res[o];
    const float bb = scale * sum;
    lv_st(C.b, ci, C.prec, bb);
    lv_st(C.x, ci, C.prec, (cw & CW_RED) ? bb / word_diag(cw) : 0.0f);
}
// Prolongation C -> F fused with the black sweep of F (see k_prolong_smooth0) at fine cell i.
template <bool CG = false>
__device__ __forceinline__ void prolong_smooth_fp_cell(const MGLevel& F, const MGLevel& C, uint32_t i, int3 c) {
    const uint32_t dx = uint32_t(F.dim.x), dxy = uint32_t(F.dim.x * F.dim.y);
    const uint32_t last = F.cells - 1u, clast = C.cells - 1u;
    // The neighbours' x and their parents' words and x are loaded before the word is tested
    // (indices clamped into the levels; values of non-fluid neighbours are not used).
    const uint32_t w = F.word[i];
    const float b = lvx<CG>(F.b, i, F.prec);
    const uint32_t off[6] = {i - 1u, i + 1u, i - dx, i + dx, i - dxy, i + dxy};
    float v[6];
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const int3 nb = add3(c, nbr_off(n));
        const uint32_t pi = min(lin3(make_int3(nb.x / 2, nb.y / 2, nb.z / 2), C.dim), clast);
        const float xn = lvx<CG>(F.x, min(off[n], last), F.prec);
        const uint32_t pw = C.word[pi];
        const float px = lvx<CG>(C.x, pi, C.prec);
        v[n] = (pw & CW_FLUID) ? q_prec(xn + px, F.prec) : xn;  // the prolonged value as it would be stored
    }
    if (!(w & CW_FLUID) || (w & CW_RED)) return;
    float sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n)
        if ((w >> n) & 1u) sum = sum + v[n];
    lv_st(F.x, i, F.prec, (b + sum) / word_diag(w));
}

__global__ void k_smooth_fp(Dev d, MGState m, int l, uint32_t parity) {
    pdl_entry();
    const MGLevel L = m.lv[l];
    const uint32_t want = parity == 0u ? CW_RED : 0u;
    if (l <= 2) for_footprint_colour(d, L, l, parity, [&](uint32_t i, int3) { smooth_fp_cell(L, i, want); });
    else for_footprint(d, L, l, [&](uint32_t i, int3) { smooth_fp_cell(L, i, want); });
}
// Restriction l -> l + 1 over level l + 1's footprint.
__global__ void k_restrict_fp(Dev d, MGState m, int l) {
    pdl_entry();
    const MGLevel F = m.lv[l], C = m.lv[l + 1];
    for_footprint(d, C, l + 1, [&](uint32_t ci, int3 c) { restrict_fp_cell(F, C, ci, c, m.restrict_scale); });
}
// Prolongation l + 1 -> l fused with the black sweep of level l.
__global__ void k_prolong_smooth_fp(Dev d, MGState m, int l) {
    pdl_entry();
    const MGLevel F = m.lv[l], C = m.lv[l + 1];
    if (l <= 2) for_footprint_colour(d, F, l, 1u, [&](uint32_t i, int3 c) { prolong_smooth_fp_cell(F, C, i, c); });
    else for_footprint(d, F, l, [&](uint32_t i, int3 c) { prolong_smooth_fp_cell(F, C, i, c); });
}

// ---- MGRestrictCS level 0 -> 1 over the 4^3 level-1 cells of every active brick (SparseCoarse) -----------
// One warp per brick: the lanes form the fine residuals of the brick's 512 cells in warp-private shared
// memory, then sum each of the 64 coarse cells' fluid children in child order (x fastest), as the
// per-coarse-cell loop does.
__global__ void __launch_bounds__(GRID_THREADS) k_restrict0(Dev d, MGState m) {
    pdl_entry();
    constexpr int WARPS = GRID_THREADS / 32;
    __shared__ float s_res[WARPS][BRICK_CELLS];
    __shared__ uint8_t s_fluid[WARPS][BRICK_CELLS];
    const MGLevel C = m.lv[1];
    const float vs = coarse_scale(m);
    const uint32_t active = d.active_bricks[0];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    for (uint32_t e = blockIdx.x * wpb + warp; e < active; e += gridDim.x * wpb) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        const uint32_t base = s1.z * BRICK_CELLS;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            const Geo g = geo_of(base, lane, k);
            const SweepQ v = load_sweep(d, m, g, ns);
            const X2 x = partner(v.z);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                float n[6];
                nbrs6(v.z, x, g.h, j, n);
                const float diag = comp(v.dg, j) + DIAG_EPSILON;
                s_fluid[warp][g.l + uint32_t(j)] = (w & W_FLUID) ? 1 : 0;
                if (w & W_FLUID) s_res[warp][g.l + uint32_t(j)] = comp(v.r, j) - (diag * comp(v.z.c, j) - nb_sum(n, w));
            }
        }
        __syncwarp();
        const int3 bc = brick_coord_of(d, s1.w);
#pragma unroll
        for (uint32_t h = 0; h < 2u; ++h) {
            const uint32_t lc = lane + 32u * h;
            const int3 cl = make_int3(int(lc & 3u), int((lc >> 2) & 3u), int(lc >> 4));
            const int3 c = make_int3(bc.x * 4 + cl.x, bc.y * 4 + cl.y, bc.z * 4 + cl.z);
            if (!inside3(c, C.dim)) continue;
            const uint32_t ci = lin3(c, C.dim);
            const uint32_t cw = C.word[ci];
            if (!(cw & CW_FLUID)) {
                lv_st(C.b, ci, C.prec, 0.0f);
                lv_st(C.x, ci, C.prec, 0.0f);
                continue;
            }
            float sum = 0.0f;
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                const uint32_t fl = uint32_t((2 * cl.x + (o & 1)) + 8 * ((2 * cl.y + ((o >> 1) & 1)) + 8 * (2 * cl.z + ((o >> 2) & 1))));
                if (s_fluid[warp][fl]) sum = sum + s_res[warp][fl];
            }
            const float bb = (m.restrict_scale * sum) * vs;
            lv_st(C.b, ci, C.prec, bb);
            lv_st(C.x, ci, C.prec, (cw & CW_RED) ? bb / word_diag(cw) : 0.0f);
        }
        __syncwarp();
    }
}

__device__ __forceinline__ float* dir_buf(const MGState& m, uint32_t parity) { return parity ? m.dvec2 : m.dvec; }
__device__ __forceinline__ const float* dir_buf_c(const MGState& m, uint32_t parity) { return parity ? m.dvec2 : m.dvec; }

// ---- level-0 passes from a shared-memory stage of the brick (bulk async copies) ---------------------------
// One warp per active brick, as above, but before computing the warp copies everything its pass reads into
// a per-warp stage in shared memory, so a brick costs one round trip to L2 instead of one per round of
// dependent loads:
//   * per "face" array (one read with neighbours): the brick's 512 cells, then its six neighbour faces of 64
//     cells each at 512 + 64 n (n = -x, +x, -y, +y, -z, +z; index y + 8 z, x + 8 z, x + 8 y in the face);
//   * per "body" array: the brick's 512 cells; and the 512 stencil bytes.
// Bodies (2 KB, 512 B) and the +-z faces (one 256-byte plane each) are 1-D bulk copies (cp.async.bulk, into this
// CTA's own shared memory) that complete on the warp's mbarrier; the +-x and +-y faces are strided in the neighbour
// brick and are read by plain loads issued alongside. A missing neighbour is the all-zero null slot 0.
// The stage of a warp is reused brick after brick; its mbarrier phase alternates.
constexpr int ST_WARPS = 4;  // warps (bricks in flight) per CTA of a staged pass
constexpr uint32_t ST_FACE = 896u;  // floats of a staged face array: body + 6 x 64
template <int NF, int NB>
struct __align__(16) WarpStage {
    float f[NF > 0 ? NF : 1][NF > 0 ? ST_FACE : 4u];
    float b[NB > 0 ? NB : 1][BRICK_CELLS];
    uint8_t word[BRICK_CELLS];
    uint64_t bar;
    uint64_t pad;
};
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(tc::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
                 : "memory");
}
// Issues the copies of one brick into S (all lanes of the warp); stage_wait then waits for them.
template <int NF, int NB>
__device__ __forceinline__ void stage_issue(WarpStage<NF, NB>& S, const float* const* fa, const float* const* ba, const uint8_t* word,
                                            uint32_t slot, const uint32_t* ns, uint32_t lane) {
    constexpr uint32_t bytes = uint32_t(NF) * 2560u + uint32_t(NB) * 2048u + 512u;
    constexpr int NC = NF * 3 + NB + 1;
    // the stage's previous contents were read by generic loads: order them before the async-proxy writes
    __syncwarp();
    tc::fence_async_shared();
    if (lane == 0) tc::mbar_arrive_expect_tx(&S.bar, bytes);
    __syncwarp();
    for (int c = int(lane); c < NC; c += 32) {
        if constexpr (NF > 0) {
            if (c < NF * 3) {
                const int f = c / 3, q = c - 3 * f;
                const float* a = fa[f];
                float* dst = &S.f[0][0] + size_t(f) * ST_FACE;
                if (q == 0) bulk_load(dst, a + size_t(slot) * BRICK_CELLS, 2048u, &S.bar);
                else if (q == 1) bulk_load(dst + 768, a + size_t(ns[4]) * BRICK_CELLS + 448, 256u, &S.bar);
                else bulk_load(dst + 832, a + size_t(ns[5]) * BRICK_CELLS, 256u, &S.bar);
                continue;
            }
        }
        if (c < NF * 3 + NB) {
            const int b = c - NF * 3;
            bulk_load(S.b[b], ba[b] + size_t(slot) * BRICK_CELLS, 2048u, &S.bar);
        } else {
            bulk_load(S.word, word + size_t(slot) * BRICK_CELLS, 512u, &S.bar);
        }
    }
    // +-x faces: cells (7, y, z) of the -x brick and (0, y, z) of the +x brick (j = y + 8 z); +-y faces:
    // cells (x, 7, z) of the -y brick and (x, 0, z) of the +y brick (j = x + 8 z). Plain loads, all issued
    // before any is stored.
    if constexpr (NF > 0) {
        float xv[NF > 0 ? NF : 1][8];
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const uint32_t j = lane + 32u * uint32_t(k);
                const uint32_t lx = 8u * j;                      // local index of (0, y, z), j = y + 8 z
                const uint32_t ly = (j & 7u) + 64u * (j >> 3);   // local index of (x, 0, z), j = x + 8 z
                xv[f][4 * k] = fa[f][size_t(ns[0]) * BRICK_CELLS + lx + 7u];
                xv[f][4 * k + 1] = fa[f][size_t(ns[1]) * BRICK_CELLS + lx];
                xv[f][4 * k + 2] = fa[f][size_t(ns[2]) * BRICK_CELLS + ly + 56u];
                xv[f][4 * k + 3] = fa[f][size_t(ns[3]) * BRICK_CELLS + ly];
            }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const uint32_t j = lane + 32u * uint32_t(k);
                S.f[f][512u + j] = xv[f][4 * k];
                S.f[f][576u + j] = xv[f][4 * k + 1];
                S.f[f][640u + j] = xv[f][4 * k + 2];
                S.f[f][704u + j] = xv[f][4 * k + 3];
            }
    }
}
// Waits for the stage's copies (phase `parity` of its mbarrier); false if the bounded wait gave up, which
// records the error in *error (ctl[5]).
template <int NF, int NB>
__device__ __forceinline__ bool stage_wait(WarpStage<NF, NB>& S, uint32_t parity, uint32_t* error) {
    const bool ok = tc::mbar_wait(&S.bar, parity, error, 1u);
    __syncwarp();
    return ok;
}
template <int NF, int NB>
__device__ __forceinline__ bool stage_brick(WarpStage<NF, NB>& S, const float* const* fa, const float* const* ba, const uint8_t* word,
                                            uint32_t slot, const uint32_t* ns, uint32_t lane, uint32_t parity, uint32_t* error) {
    stage_issue<NF, NB>(S, fa, ba, word, slot, ns, lane);
    return stage_wait<NF, NB>(S, parity, error);
}
// Neighbour n of local cell l of a staged face array.
__device__ __forceinline__ float snbr(const float* F, uint32_t l, int n) {
    const uint32_t x = l & 7u, y = (l >> 3) & 7u, z = l >> 6;
    switch (n) {
        case 0: return x > 0u ? F[l - 1u] : F[512u + y + 8u * z];
        case 1: return x < 7u ? F[l + 1u] : F[576u + y + 8u * z];
        case 2: return y > 0u ? F[l - 8u] : F[640u + x + 8u * z];
        case 3: return y < 7u ? F[l + 8u] : F[704u + x + 8u * z];
        case 4: return z > 0u ? F[l - 64u] : F[768u + x + 8u * y];
        default: return z < 7u ? F[l + 64u] : F[832u + x + 8u * y];
    }
}
__device__ __forceinline__ float4 sld4(const float* F, uint32_t l) { return *reinterpret_cast<const float4*>(F + l); }
// A quad of a staged face array with its neighbours, as load_q6 reads it from global memory.
__device__ __forceinline__ Q6 sq6(const float* F, const Geo& g) {
    Q6 q;
    q.c = sld4(F, g.l);
    q.ym = sld4(F, g.y > 0u ? g.l - 8u : 640u + 4u * g.h + 8u * g.z);
    q.yp = sld4(F, g.y < 7u ? g.l + 8u : 704u + 4u * g.h + 8u * g.z);
    q.zm = sld4(F, g.z > 0u ? g.l - 64u : 768u + 4u * g.h + 8u * g.y);
    q.zp = sld4(F, g.z < 7u ? g.l + 64u : 832u + 4u * g.h + 8u * g.y);
    q.xb = F[(g.h == 0u ? 512u : 576u) + g.y + 8u * g.z];
    return q;
}
__device__ __forceinline__ uint32_t sword4(const uint8_t* W, const Geo& g) { return *reinterpret_cast<const uint32_t*>(W + g.l); }

// Final FP64 reduction over the brick partials for a CTA of T threads: the canonical tree of final_reduce
// (lane t = 0..1023 adds partials t, t + 1024, ... in order; groups of 32 lanes fold with shfl_down; the
// 32 group sums are added in order), with each thread owning lanes x + T k.
template <int T>
__device__ double final_reduce_t(const double* partials, uint32_t n, double* lanes, double* w32) {
    constexpr int K = 1024 / T;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t base = 0; base < n; base += 1024u) {
        double v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t e = base + threadIdx.x + uint32_t(T * k);
            v[k] = e < n ? __ldcg(partials + e) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (base + threadIdx.x + uint32_t(T * k) < n) acc[k] = acc[k] + v[k];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) lanes[threadIdx.x + uint32_t(T * k)] = acc[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int lw = warp + (T / 32) * k;
        const double v = warp_fold(lanes[lw * 32 + lane]);
        if (lane == 0) w32[lw] = v;
    }
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0) {
        total = w32[0];
        for (int w = 1; w < 32; ++w) total = total + w32[w];
    }
    return total;
}

// Staged pass over the active bricks: per brick the stage is filled, then rounds k = 0..3 of the half-row
// layout call apply(S, g, v0, v1) (dot terms as in w4_pass); with NDOT > 0 the last CTA reduces the brick
// partials and calls store(t0, t1) in thread 0. fa/ba name the face and body arrays.
template <int NF, int NB, int NDOT, class Apply, class Store>
__device__ __forceinline__ void st_pass(const Dev& d, const MGState& m, uint32_t counter, const float* const* fa, const float* const* ba,
                                        Apply apply, Store store) {
    extern __shared__ __align__(16) unsigned char st_smem[];
    using Stg = WarpStage<NF, NB>;
    __shared__ uint32_t s_last;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    Stg& S = reinterpret_cast<Stg*>(st_smem)[warp];
    if (lane == 0) {
        tc::mbar_init(&S.bar, 1u);
        tc::fence_mbar_init();
    }
    __syncwarp();
    const uint32_t active = d.active_bricks[0];
    const uint32_t cap = d.num_pool_bricks;
    uint32_t parity = 0u;
    for (uint32_t e = blockIdx.x * ST_WARPS + warp; e < active; e += gridDim.x * ST_WARPS) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        const uint32_t base = s1.z * BRICK_CELLS;
        if (!stage_brick<NF, NB>(S, fa, ba, m.word, s1.z, ns, lane, parity, m.ctl + 5)) break;
        parity ^= 1u;
        double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            const Geo g = geo_of(base, lane, k);
            double v0[4] = {0.0, 0.0, 0.0, 0.0}, v1[4] = {0.0, 0.0, 0.0, 0.0};
            apply(S, g, v0, v1);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc0 = acc0 + v0[j];
                acc1 = acc1 + v1[j];
            }
        }
        if (NDOT > 0) {
            const double t0 = warp_fold(acc0);
            if (lane == 0) m.partials[e] = t0;
        }
        if (NDOT > 1) {
            const double t1 = warp_fold(acc1);
            if (lane == 0) m.partials[cap + e] = t1;
        }
    }
    if (NDOT == 0) return;
    __syncwarp();
    if (lane == 0) tc::mbar_inval(&S.bar);  // the stage memory is reused by the final reduction below
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(m.counters + counter, 1u) == gridDim.x - 1u) ? 1u : 0u;
    __syncthreads();
    if (s_last) {
        __threadfence();
        // the stages are free now: the reduction's lanes live in their shared memory
        double* lanes = reinterpret_cast<double*>(st_smem);
        double* w32 = lanes + 1024;
        const double r0 = final_reduce_t<ST_WARPS * 32>(m.partials, active, lanes, w32);
        __syncthreads();
        double r1 = 0.0;
        if (NDOT > 1) r1 = final_reduce_t<ST_WARPS * 32>(m.partials + cap, active, lanes, w32);
        if (threadIdx.x == 0) {
            store(r0, r1);
            m.counters[counter] = 0u;
        }
    }
}
// Staged pass in the black-cell layout of w0_black: prep(S, brick, lane) once per brick, then each lane's 8
// black cells through apply(S, i, l).
template <int NF, int NB, class Prep, class Apply>
__device__ __forceinline__ void st_black(const Dev& d, const MGState& m, const float* const* fa, const float* const* ba, Prep prep,
                                         Apply apply) {
    extern __shared__ __align__(16) unsigned char st_smem[];
    using Stg = WarpStage<NF, NB>;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    Stg& S = reinterpret_cast<Stg*>(st_smem)[warp];
    if (lane == 0) {
        tc::mbar_init(&S.bar, 1u);
        tc::fence_mbar_init();
    }
    __syncwarp();
    const uint32_t active = d.active_bricks[0];
    uint32_t parity = 0u;
    for (uint32_t e = blockIdx.x * ST_WARPS + warp; e < active; e += gridDim.x * ST_WARPS) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        const uint32_t base = s1.z * BRICK_CELLS;
        stage_issue<NF, NB>(S, fa, ba, m.word, s1.z, ns, lane);
        prep(S, s1.w, lane);  // its loads overlap the copies
        if (!stage_wait<NF, NB>(S, parity, m.ctl + 5)) break;
        parity ^= 1u;
#pragma unroll
        for (uint32_t k = 0; k < 8u; ++k) {
            const uint32_t l = black_local(lane, k);
            apply(S, base + l, l);
        }
    }
}
template <int NF, int NB>
constexpr size_t st_smem_bytes() {
    const size_t stage = sizeof(WarpStage<NF, NB>) * ST_WARPS;
    const size_t reduce = (1024 + 32) * sizeof(double);
    return stage > reduce ? stage : reduce;
}

// k_smooth0 from a stage: z (face), r and the diagonal (bodies).
template <bool DOT>
__global__ void __launch_bounds__(ST_WARPS * 32) k_smooth0_st(Dev d, MGState m) {
    pdl_entry();
    const float* fa[1] = {m.z};
    const float* ba[2] = {m.r, d.cell_diag};
    st_pass<1, 2, DOT ? 1 : 0>(d, m, 1, fa, ba,
        [&](WarpStage<1, 2>& S, const Geo& g, double* v0, double*) {
            const Q6 z = sq6(S.f[0], g);
            const float4 r = sld4(S.b[0], g.l), dg = sld4(S.b[1], g.l);
            const uint32_t w4 = sword4(S.word, g);
            const X2 x = partner(z);
            float out[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(w4, j);
                const float zj = comp(z.c, j), rj = comp(r, j);
                out[j] = zj;
                if (!(w & W_FLUID)) continue;
                if (w & W_RED) {
                    float n[6];
                    nbrs6(z, x, g.h, j, n);
                    const float val = (rj + nb_sum(n, w)) / (comp(dg, j) + DIAG_EPSILON);
                    out[j] = val;
                    v0[j] = double(rj * val);
                } else {
                    v0[j] = double(rj * zj);
                }
            }
            st4(m.z + g.i, out);
        },
        [&](double rho, double) { m.scalars[3] = m.scalars[0]; m.scalars[0] = rho; });
}
// Black sweep from a stage.
__global__ void __launch_bounds__(ST_WARPS * 32) k_smooth0_black_st(Dev d, MGState m) {
    pdl_entry();
    const float* fa[1] = {m.z};
    const float* ba[2] = {m.r, d.cell_diag};
    st_black<1, 2>(d, m, fa, ba, [](WarpStage<1, 2>&, uint32_t, uint32_t) {},
        [&](WarpStage<1, 2>& S, uint32_t i, uint32_t l) {
            const uint32_t w = S.word[l];
            if (!(w & W_FLUID)) return;
            float n[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) n[k] = snbr(S.f[0], l, k);
            m.z[i] = (S.b[0][l] + nb_sum(n, w)) / (S.b[1][l] + DIAG_EPSILON);
        });
}
// k_prolong_smooth0 from a stage (the level-1 6^3 block is staged by plain loads as before).
__global__ void __launch_bounds__(ST_WARPS * 32) k_prolong_smooth0_st(Dev d, MGState m) {
    pdl_entry();
    __shared__ float s_cx[ST_WARPS][216];
    const MGLevel C = m.lv[1];
    const float ivs = 1.0f / coarse_scale(m);  // a power of two: exact
    float* cx = s_cx[threadIdx.x >> 5];
    const float* fa[1] = {m.z};
    const float* ba[2] = {m.r, d.cell_diag};
    st_black<1, 2>(d, m, fa, ba,
        [&](WarpStage<1, 2>&, uint32_t brick, uint32_t lane) {
            const int3 bc = brick_coord_of(d, brick);
            __syncwarp();
            float v[7];
#pragma unroll
            for (int r = 0; r < 7; ++r) {
                const uint32_t j = lane + 32u * uint32_t(r);
                const int3 c = make_int3(bc.x * 4 - 1 + int(j % 6u), bc.y * 4 - 1 + int((j / 6u) % 6u), bc.z * 4 - 1 + int(j / 36u));
                v[r] = 0.0f;
                if (j < 216u && inside3(c, C.dim)) {
                    const uint32_t ci = lin3(c, C.dim);
                    const float x = lv_ld(C.x, ci, C.prec);
                    v[r] = (C.word[ci] & CW_FLUID) ? x * ivs : 0.0f;
                }
            }
#pragma unroll
            for (int r = 0; r < 7; ++r) {
                const uint32_t j = lane + 32u * uint32_t(r);
                if (j < 216u) cx[j] = v[r];
            }
        },
        [&](WarpStage<1, 2>& S, uint32_t i, uint32_t l) {
            const uint32_t w = S.word[l];
            if (!(w & W_FLUID)) return;
            const int x = int(l & 7u), y = int((l >> 3) & 7u), z = int(l >> 6);
            const int p = ((x >> 1) + 1) + 6 * ((y >> 1) + 1) + 36 * ((z >> 1) + 1);
            const int px = (x & 1) ? 1 : 0, py = (y & 1) ? 6 : 0, pz = (z & 1) ? 36 : 0;
            const int po[6] = {p - 1 + px, p + px, p - 6 + py, p + py, p - 36 + pz, p + pz};
            float sum = 0.0f;
#pragma unroll
            for (int n = 0; n < 6; ++n)
                if ((w >> n) & 1u) sum = sum + (snbr(S.f[0], l, n) + cx[po[n]]);
            m.z[i] = (S.b[0][l] + sum) / (S.b[1][l] + DIAG_EPSILON);
        });
}
// k_restrict0 from a stage: the brick's fine residuals into the warp's s_res, then the 64 coarse cells.
__global__ void __launch_bounds__(ST_WARPS * 32) k_restrict0_st(Dev d, MGState m) {
    pdl_entry();
    __shared__ float s_res[ST_WARPS][BRICK_CELLS];
    const MGLevel C = m.lv[1];
    const uint32_t warp = threadIdx.x >> 5;
    const float* fa[1] = {m.z};
    const float* ba[2] = {m.r, d.cell_diag};
    const float scale = m.restrict_scale;
    const float vs = coarse_scale(m);
    extern __shared__ __align__(16) unsigned char st_smem[];
    using Stg = WarpStage<1, 2>;
    const uint32_t lane = threadIdx.x & 31u;
    Stg& S = reinterpret_cast<Stg*>(st_smem)[warp];
    if (lane == 0) {
        tc::mbar_init(&S.bar, 1u);
        tc::fence_mbar_init();
    }
    __syncwarp();
    const uint32_t active = d.active_bricks[0];
    uint32_t parity = 0u;
    for (uint32_t e = blockIdx.x * ST_WARPS + warp; e < active; e += gridDim.x * ST_WARPS) {
        const uint4 s0 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e);
        const uint4 s1 = *reinterpret_cast<const uint4*>(m.nbr_slots + 8u * e + 4u);
        const uint32_t ns[6] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
        if (!stage_brick<1, 2>(S, fa, ba, m.word, s1.z, ns, lane, parity, m.ctl + 5)) break;
        parity ^= 1u;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            const Geo g = geo_of(0u, lane, k);
            const Q6 z = sq6(S.f[0], g);
            const float4 r = sld4(S.b[0], g.l), dg = sld4(S.b[1], g.l);
            const uint32_t w4 = sword4(S.word, g);
            const X2 x = partner(z);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(w4, j);
                float n[6];
                nbrs6(z, x, g.h, j, n);
                const float diag = comp(dg, j) + DIAG_EPSILON;
                if (w & W_FLUID) s_res[warp][g.l + uint32_t(j)] = comp(r, j) - (diag * comp(z.c, j) - nb_sum(n, w));
            }
        }
        __syncwarp();
        const int3 bc = brick_coord_of(d, s1.w);
#pragma unroll
        for (uint32_t h = 0; h < 2u; ++h) {
            const uint32_t lc = lane + 32u * h;
            const int3 cl = make_int3(int(lc & 3u), int((lc >> 2) & 3u), int(lc >> 4));
            const int3 c = make_int3(bc.x * 4 + cl.x, bc.y * 4 + cl.y, bc.z * 4 + cl.z);
            if (!inside3(c, C.dim)) continue;
            const uint32_t ci = lin3(c, C.dim);
            const uint32_t cw = C.word[ci];
            if (!(cw & CW_FLUID)) {
                lv_st(C.b, ci, C.prec, 0.0f);
                lv_st(C.x, ci, C.prec, 0.0f);
                continue;
            }
            float sum = 0.0f;
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                const uint32_t fl = uint32_t((2 * cl.x + (o & 1)) + 8 * ((2 * cl.y + ((o >> 1) & 1)) + 8 * (2 * cl.z + ((o >> 2) & 1))));
                if (S.word[fl] & W_FLUID) sum = sum + s_res[warp][fl];
            }
            const float bb = (scale * sum) * vs;
            lv_st(C.b, ci, C.prec, bb);
            lv_st(C.x, ci, C.prec, (cw & CW_RED) ? bb / word_diag(cw) : 0.0f);
        }
    }
}
// k_apply_a from a stage: z and the previous direction (faces), the diagonal (body).
__global__ void __launch_bounds__(ST_WARPS * 32) k_apply_a_st(Dev d, MGState m) {
    pdl_entry();
    const uint32_t it = m.ctl[0];
    const bool first = it == 0u;
    const float beta = first ? 0.0f : ratio_f(m.flexible ? m.scalars[0] - m.scalars[9] : m.scalars[0], m.scalars[3]);
    const float* dold = dir_buf_c(m, it & 1u);
    float* dnew = dir_buf(m, (it + 1u) & 1u);
    const float* fa[2] = {m.z, dold};
    const float* ba[1] = {d.cell_diag};
    st_pass<2, 1, 1>(d, m, 2, fa, ba,
        [&](WarpStage<2, 1>& S, const Geo& g, double* v0, double*) {
            const Q6 vz = sq6(S.f[0], g), vd = sq6(S.f[1], g);
            const float4 dg = sld4(S.b[0], g.l);
            const uint32_t w4 = sword4(S.word, g);
            const X2 xz = partner(vz), xd = partner(vd);
            float dn[4], q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(w4, j);
                dn[j] = 0.0f;
                q[j] = 0.0f;
                if (!(w & W_FLUID)) continue;
                const float dj = first ? comp(vz.c, j) : comp(vz.c, j) + beta * comp(vd.c, j);
                float nz[6], nd[6];
                nbrs6(vz, xz, g.h, j, nz);
                nbrs6(vd, xd, g.h, j, nd);
                float sum = 0.0f;
#pragma unroll
                for (int n = 0; n < 6; ++n)
                    if ((w >> n) & 1u) sum = sum + (first ? nz[n] : nz[n] + beta * nd[n]);
                const float qi = (comp(dg, j) + DIAG_EPSILON) * dj - sum;
                dn[j] = dj;
                q[j] = qi;
                v0[j] = double(dj * qi);
            }
            st4(dnew + g.i, dn);
            st4(m.q + g.i, q);
        },
        [&](double dq, double) { m.scalars[2] = dq; });
}

// k_update_pr from a stage: p, the current direction, r, q, the diagonal (and with FLEX the finished
// V-cycle's z) as bodies.
template <bool FLEX>
__global__ void __launch_bounds__(ST_WARPS * 32) k_update_pr_st(Dev d, MGState m, float* __restrict__ p, unsigned long long handle) {
    pdl_entry();
    constexpr int NB = FLEX ? 6 : 5;
    const float alpha = ratio_f(m.scalars[0], m.scalars[2]);
    const float* dcur = dir_buf_c(m, (m.ctl[0] + 1u) & 1u);
    const float* ba[6] = {p, dcur, m.r, m.q, d.cell_diag, m.z};
    st_pass<0, NB, FLEX ? 2 : 1>(d, m, 3, nullptr, ba,
        [&](WarpStage<0, NB>& S, const Geo& g, double* v0, double* v1) {
            const float4 vp = sld4(S.b[0], g.l), vd = sld4(S.b[1], g.l), vr = sld4(S.b[2], g.l), vq = sld4(S.b[3], g.l);
            const float4 dg = sld4(S.b[4], g.l);
            const float4 vz = FLEX ? sld4(S.b[NB - 1], g.l) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const uint32_t w4 = sword4(S.word, g);
            float po[4], ro[4], zo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(w4, j);
                po[j] = comp(vp, j);
                ro[j] = comp(vr, j);
                zo[j] = 0.0f;
                if (!(w & W_FLUID)) continue;
                po[j] = comp(vp, j) + alpha * comp(vd, j);
                const float ri = comp(vr, j) - alpha * comp(vq, j);
                ro[j] = ri;
                zo[j] = (w & W_RED) ? red_init0(m, ri / (comp(dg, j) + DIAG_EPSILON)) : 0.0f;
                v0[j] = double(ri * ri);
                if (FLEX) v1[j] = double(ri * comp(vz, j));
            }
            st4(p + g.i, po);
            st4(m.r + g.i, ro);
            st4(m.z + g.i, zo);
        },
        [&](double rr, double rz) {
            m.scalars[5] = rr;
            if (FLEX) m.scalars[9] = rz;
            const uint32_t it = m.ctl[0] + 1u;
            m.ctl[0] = it;
            const double bb = m.scalars[4];
            const double rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
            const bool converged = m.ctl[2] != 0u && rel <= m.scalars[8];
            const bool more = it < m.ctl[1] && !converged;
            if (!more) m.ctl[3] = 1u;
            if (!more && m.ctl[2] != 0u && !converged) m.ctl[4] = 1u;  // stopped at the limit: sticky for the frame
            if (handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
        });
}

// ---- the small coarse levels in one CTA: levels tail..nl-1 of the V-cycle --------------------------------
// Once per solve, k_tail_lists stores each tail level's fluid cells by colour. Each V-cycle,
// k_vcycle_tail copies the tail levels into shared memory (word, diagonal, x, b per cell; the colour
// lists), runs the descent, the coarse solve and the ascent there -- every sweep visits only the fluid
// cells of its colour -- and writes level tail's x back. On entry level `tail` holds b and the
// red-initialised x from the restriction that produced it.
__global__ void __launch_bounds__(1024) k_tail_lists(MGState m, int tail) {
    pdl_entry();
    __shared__ uint32_t s_warp[33];
    uint32_t off = 0;
    for (int l = tail; l < m.num_levels; ++l) {
        const MGLevel L = m.lv[l];
        for (uint32_t colour = 0; colour < 2u; ++colour) {
            const uint32_t want = colour == 0u ? CW_RED : 0u;
            uint32_t base = 0;
            for (uint32_t start = 0; start < L.cells; start += blockDim.x) {
                const uint32_t i = start + threadIdx.x;
                const uint32_t w = i < L.cells ? uint32_t(L.word[i]) : 0u;
                const uint32_t flag = (i < L.cells && (w & CW_FLUID) && (w & CW_RED) == want) ? 1u : 0u;
                // block-wide exclusive scan of flag
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, flag);
                if (lane == 0) s_warp[warp] = __popc(bal);
                __syncthreads();
                if (warp == 0) {
                    const uint32_t v = s_warp[lane];
                    uint32_t x = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                        if (lane >= o) x += y;
                    }
                    s_warp[lane] = x - v;
                    if (lane == 31) s_warp[32] = x;
                }
                __syncthreads();
                if (flag) m.tail_list[off + base + s_warp[warp] + __popc(bal & ((1u << lane) - 1u))] = i;
                base += s_warp[32];
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                m.tail_meta[4 * l + 2 * colour] = off;
                m.tail_meta[4 * l + 2 * colour + 1] = base;
            }
            off += base;
        }
    }
    // The static part of the tail's shared-memory image for this solve: diagonals, words, colour lists.
    __syncthreads();
    for (int l = tail; l < m.num_levels; ++l) {
        const MGLevel L = m.lv[l];
        const TailOffsets o = tail_offsets(m, tail, l, nullptr);
        float* diag = reinterpret_cast<float*>(m.tail_image + o.diag);
        uint16_t* word = reinterpret_cast<uint16_t*>(m.tail_image + o.word);
        uint32_t* list = reinterpret_cast<uint32_t*>(m.tail_image + o.list);
        for (uint32_t i = threadIdx.x; i < L.cells; i += blockDim.x) {
            const uint32_t w = L.word[i];
            word[i] = uint16_t(w);
            diag[i] = word_diag(w);
        }
        const uint32_t first = m.tail_meta[4 * l], n = m.tail_meta[4 * l + 1] + m.tail_meta[4 * l + 3];
        for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) list[j] = m.tail_list[first + j];
    }
}

struct SLevel {
    int3 dim;
    uint32_t cells, dx, dxy;
    uint16_t* word;
    float* diag;
    float* x;
    float* b;
    const uint32_t* list;  // red cells then black cells
    uint32_t nred, nblack;
    uint32_t prec;         // storage precision: stores round to it (the values stay FP32 in shared memory)
};
__device__ __forceinline__ void s_sweep(const SLevel L, uint32_t colour) {
    const uint32_t n = colour == 0u ? L.nred : L.nblack;
    const uint32_t* list = L.list + (colour == 0u ? 0u : L.nred);
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const uint32_t i = list[j];
        const uint32_t w = L.word[i];
        L.x[i] = q_prec((L.b[i] + word_sum(L.x, w, i, L.dx, L.dxy)) / L.diag[i], L.prec);
    }
    __syncthreads();
}
// The coarsest level's red-black iterations on the first 4 warps, synchronised by a 128-thread named
// barrier (the level has at most 512 cells, so 128 threads visit each colour in a few rounds).
__device__ __forceinline__ void s_coarse_solve(const SLevel L, int iterations) {
    if (threadIdx.x < 128u) {
        for (int it = 0; it < iterations; ++it) {
#pragma unroll
            for (uint32_t colour = 0; colour < 2u; ++colour) {
                const uint32_t n = colour == 0u ? L.nred : L.nblack;
                const uint32_t* list = L.list + (colour == 0u ? 0u : L.nred);
                for (uint32_t j = threadIdx.x; j < n; j += 128u) {
                    const uint32_t i = list[j];
                    const uint32_t w = L.word[i];
                    L.x[i] = q_prec((L.b[i] + word_sum(L.x, w, i, L.dx, L.dxy)) / L.diag[i], L.prec);
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
            }
        }
    }
    __syncthreads();
}
// The tail's V-cycle on one CTA of 1024 threads (s_tail: mg_tail_smem bytes of shared memory). CG: level tail's x
// and b were written earlier in the same kernel by other CTAs of the cluster, so they are read through L2.
template <bool CG>
__device__ __forceinline__ void vcycle_tail_body(const MGState& m, int tail, int iterations, unsigned char* s_tail) {
    const int nl = m.num_levels;
    SLevel S[SLOSH_MAX_MG_LEVELS];
    uint32_t total = 0;
    for (int l = tail; l < nl; ++l) {
        const MGLevel G = m.lv[l];
        const TailOffsets o = tail_offsets(m, tail, l, &total);
        SLevel& L = S[l];
        L.dim = G.dim;
        L.cells = G.cells;
        L.dx = uint32_t(G.dim.x);
        L.dxy = uint32_t(G.dim.x * G.dim.y);
        L.x = reinterpret_cast<float*>(s_tail + o.x);
        L.b = reinterpret_cast<float*>(s_tail + o.b);
        L.diag = reinterpret_cast<float*>(s_tail + o.diag);
        L.word = reinterpret_cast<uint16_t*>(s_tail + o.word);
        L.list = reinterpret_cast<const uint32_t*>(s_tail + o.list);
        L.nred = m.tail_meta[4 * l + 1];
        L.nblack = m.tail_meta[4 * l + 3];
        L.prec = G.prec;
    }
    // One round trip: level tail's x and b from the level arrays, everything static (diagonals, words,
    // colour lists of all tail levels) from the image k_tail_lists built for this solve.
    {
        const uint32_t c16 = tail_pad4(m.lv[tail].cells) / 4u;  // 16-byte chunks of one level-tail array
        const uint32_t n16 = total / 16u;
        const uint4* gx = reinterpret_cast<const uint4*>(m.lv[tail].x);
        const uint4* gb = reinterpret_cast<const uint4*>(m.lv[tail].b);
        const uint4* img = reinterpret_cast<const uint4*>(m.tail_image);
        uint4* dst = reinterpret_cast<uint4*>(s_tail);
        for (uint32_t k0 = 0; k0 < n16; k0 += 8u * 1024u) {
            uint4 v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint32_t k = k0 + uint32_t(r) * 1024u + threadIdx.x;
                if (k < n16) {
                    if (k < 2u * c16 && m.lv[tail].prec != SLOSH_PRECISION_FP32) {
                        // 2-byte storage: four elements per 16-byte chunk of shared memory
                        const float* src = k < c16 ? m.lv[tail].x : m.lv[tail].b;
                        const uint32_t e = 4u * (k < c16 ? k : k - c16);
                        const uint32_t pr = m.lv[tail].prec;
                        v[r] = make_uint4(__float_as_uint(lvx<CG>(src, e, pr)), __float_as_uint(lvx<CG>(src, e + 1u, pr)),
                                          __float_as_uint(lvx<CG>(src, e + 2u, pr)), __float_as_uint(lvx<CG>(src, e + 3u, pr)));
                    } else if (k < 2u * c16) {
                        const uint4* g = k < c16 ? gx + k : gb + (k - c16);
                        v[r] = CG ? __ldcg(g) : *g;
                    } else {
                        v[r] = img[k];
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint32_t k = k0 + uint32_t(r) * 1024u + threadIdx.x;
                if (k < n16) dst[k] = v[r];
            }
        }
    }
    __syncthreads();
    // pre-smoothing of a level: its black half (the red half is the restriction's initialisation), then
    // m.sweeps - 1 more red-black pairs
    auto pre_smooth = [&](const SLevel& L) {
        s_sweep(L, 1u);
        for (int k = 1; k < m.sweeps; ++k) {
            s_sweep(L, 0u);
            s_sweep(L, 1u);
        }
    };
    if (tail < nl - 1) pre_smooth(S[tail]);
    for (int l = tail; l < nl - 1; ++l) {
        const SLevel F = S[l];
        const SLevel C = S[l + 1];
        for (uint32_t j = threadIdx.x; j < C.nred + C.nblack; j += blockDim.x) {
            const uint32_t ci = C.list[j];
            const int3 c = coord3(ci, C.dim);
            float res[8];
            uint32_t fl = 0u;
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                res[o] = 0.0f;
                const int3 f = make_int3(c.x * 2 + (o & 1), c.y * 2 + ((o >> 1) & 1), c.z * 2 + ((o >> 2) & 1));
                if (!inside3(f, F.dim)) continue;
                const uint32_t fi = lin3(f, F.dim);
                const uint32_t w = F.word[fi];
                if (!(w & CW_FLUID)) continue;
                fl |= 1u << o;
                res[o] = F.b[fi] - (F.diag[fi] * F.x[fi] - word_sum(F.x, w, fi, F.dx, F.dxy));
            }
            float sum = 0.0f;
#pragma unroll
            for (int o = 0; o < 8; ++o)
                if ((fl >> o) & 1u) sum = sum + res[o];
            const float bb = m.restrict_scale * sum;
            C.b[ci] = q_prec(bb, C.prec);
            C.x[ci] = q_prec((C.word[ci] & CW_RED) ? bb / C.diag[ci] : 0.0f, C.prec);
        }
        __syncthreads();
        if (l + 1 < nl - 1) pre_smooth(C);
    }
    s_coarse_solve(S[nl - 1], iterations);
    for (int l = nl - 2; l >= tail; --l) {
        const SLevel F = S[l];
        const SLevel C = S[l + 1];
        for (uint32_t j = threadIdx.x; j < F.nred + F.nblack; j += blockDim.x) {
            const uint32_t i = F.list[j];
            const int3 c = coord3(i, F.dim);
            const uint32_t pi = lin3(make_int3(c.x / 2, c.y / 2, c.z / 2), C.dim);
            if (C.word[pi] & CW_FLUID) F.x[i] = q_prec(F.x[i] + C.x[pi], F.prec);
        }
        __syncthreads();
        for (int k = 0; k < m.sweeps; ++k) {
            s_sweep(F, 1u);
            s_sweep(F, 0u);
        }
    }
    {
        const uint32_t c16 = tail_pad4(m.lv[tail].cells) / 4u;
        const uint4* src = reinterpret_cast<const uint4*>(s_tail);
        const uint32_t pr = m.lv[tail].prec;
        if (pr == SLOSH_PRECISION_FP32) {
            uint4* gx = reinterpret_cast<uint4*>(m.lv[tail].x);
            for (uint32_t k = threadIdx.x; k < c16; k += blockDim.x) gx[k] = src[k];
        } else {
            const float* sx = reinterpret_cast<const float*>(s_tail);
            for (uint32_t e = threadIdx.x; e < 4u * c16; e += blockDim.x) lv_st(m.lv[tail].x, e, pr, sx[e]);
        }
    }
}
__global__ void __launch_bounds__(1024) k_vcycle_tail(MGState m, int tail, int iterations) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char s_tail[];
    vcycle_tail_body<false>(m, tail, iterations, s_tail);
}

// ---- the middle levels in one thread-block cluster ------------------------------------------------------
// Levels c0..tail-1 of the V-cycle are small (at 256^3 level 2 has 8 and level 3 one cell per active brick),
// so as separate grid-wide passes each costs a launch and a chain of dependent loads, not bandwidth. One
// cluster of MID_CLUSTER CTAs (one per SM) runs them instead, from the restriction c0 - 1 -> c0 to the
// post-smoothing of level c0, each pass over the level's footprint split across the cluster's threads and
// followed by a cluster barrier (release / acquire); values written by other CTAs are read through L2. Between
// the descent and the ascent CTA 0 runs the tail's V-cycle in its shared memory. The passes are the per-cell
// bodies of k_restrict_fp, k_smooth_fp and k_prolong_smooth_fp, so the results are those of the separate
// launches. Measured slower on B200 and therefore opt-in (SLOSH_MG_CLUSTER=2 or 3): a 256^3 substep's pressure
// solve takes 3.66 ms with the cluster from level 2 and 3.07 ms from level 3, against 2.76 ms with the separate
// launches -- on 16 SMs each pass's chain of dependent L2 loads takes longer than a launch across all 148.
constexpr int MID_CLUSTER = 16;
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__global__ void __launch_bounds__(1024) k_vcycle_mid(Dev d, MGState m, int c0, int tail, int iterations) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char s_tail[];
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    const uint32_t t0 = rank * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;  // the grid is one cluster
    const int sweeps = max(m.sweeps, 1);
    auto sweep = [&](int l, uint32_t parity) {
        const MGLevel L = m.lv[l];
        const uint32_t want = parity == 0u ? CW_RED : 0u;
        for_footprint_span(d, L, l, t0, stride, [&](uint32_t i, int3) { smooth_fp_cell<true>(L, i, want); });
        cluster_barrier();
    };
    for (int l = c0 - 1; l < tail; ++l) {
        const MGLevel F = m.lv[l], C = m.lv[l + 1];
        for_footprint_span(d, C, l + 1, t0, stride, [&](uint32_t ci, int3 c) { restrict_fp_cell<true>(F, C, ci, c, m.restrict_scale); });
        cluster_barrier();
        if (l + 1 < tail) {
            sweep(l + 1, 1u);
            for (int k = 1; k < sweeps; ++k) {
                sweep(l + 1, 0u);
                sweep(l + 1, 1u);
            }
        }
    }
    if (rank == 0u) vcycle_tail_body<true>(m, tail, iterations, s_tail);
    cluster_barrier();
    for (int l = tail - 1; l >= c0; --l) {
        const MGLevel F = m.lv[l], C = m.lv[l + 1];
        for_footprint_span(d, F, l, t0, stride, [&](uint32_t i, int3 c) { prolong_smooth_fp_cell<true>(F, C, i, c); });
        cluster_barrier();
        for (int k = 1; k < sweeps; ++k) {
            sweep(l, 0u);
            sweep(l, 1u);
        }
        sweep(l, 0u);
    }
}

// ---- the coarse solve directly on level 0 (grids of <= 512 cells have a single level) --------------------
__global__ void __launch_bounds__(1024) k_coarse_solve0(Dev d, MGState m, int iterations) {
    pdl_entry();
    const MGLevel L = m.lv[0];
    for (int it = 0; it < iterations; ++it) {
        for (uint32_t colour = 0; colour < 2u; ++colour) {
            for (uint32_t li = threadIdx.x; li < L.cells; li += blockDim.x) {
                const int3 c = coord3(li, L.dim);
                if ((is_red(c) ? 0u : 1u) != colour) continue;
                const uint32_t i = cell_index(d, c);
                if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) continue;
                float diag, sum;
                stencil0(d, m.z, i, c, diag, sum);
                m.z[i] = (m.r[i] + sum) / diag;
            }
            __syncthreads();
        }
    }
}

// ---- PCGUpdateDCS fused into PCGApplyACS: d = z + beta d, q = A d, d.q ------------------------------------
// d is double-buffered by iteration parity (ctl[0] is the number of finished iterations): the pass reads
// the previous direction from one buffer and writes the new one to the other, and forms each fluid
// neighbour's new direction z_n + beta d_n itself (bit-identical to what that neighbour writes).

__global__ void __launch_bounds__(GRID_THREADS, 3) k_apply_a(Dev d, MGState m) {
    pdl_entry();
    const uint32_t it = m.ctl[0];
    const bool first = it == 0u;
    // flexible PCG: beta = (rho_k - r_k.z_{k-1}) / rho_{k-1}, the numerator formed in FP64
    const float beta = first ? 0.0f : ratio_f(m.flexible ? m.scalars[0] - m.scalars[9] : m.scalars[0], m.scalars[3]);
    const float* dold = dir_buf(m, it & 1u);
    float* dnew = dir_buf(m, (it + 1u) & 1u);
    struct V {
        Q6 z, dd;
        float4 dg;
        uint32_t w;
    };
    w4_pass<1, 1>(d, m, 2,
        [&](const Geo& g, const uint32_t* ns) {
            V v;
            v.z = load_q6(m.z, g, ns);
            v.dd = load_q6(dold, g, ns);
            v.dg = ld4(d.cell_diag + g.i);
            v.w = quad_words(m, g);
            return v;
        },
        [&](const Geo& g, const V& v, double* v0, double*) {
            const X2 xz = partner(v.z), xd = partner(v.dd);
            float dn[4], q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                dn[j] = 0.0f;
                q[j] = 0.0f;
                if (!(w & W_FLUID)) continue;
                const float dj = first ? comp(v.z.c, j) : comp(v.z.c, j) + beta * comp(v.dd.c, j);
                float nz[6], nd[6];
                nbrs6(v.z, xz, g.h, j, nz);
                nbrs6(v.dd, xd, g.h, j, nd);
                float sum = 0.0f;
#pragma unroll
                for (int n = 0; n < 6; ++n)
                    if ((w >> n) & 1u) sum = sum + (first ? nz[n] : nz[n] + beta * nd[n]);
                const float qi = (comp(v.dg, j) + DIAG_EPSILON) * dj - sum;
                dn[j] = dj;
                q[j] = qi;
                v0[j] = double(dj * qi);
            }
            st4(dnew + g.i, dn);
            st4(m.q + g.i, q);
        },
        [&](double dq, double) { m.scalars[2] = dq; });
}

// ---- PCGUpdatePRCS: p += alpha d, r -= alpha q, red pre-smooth; ||r||^2 and the loop decision -------------
// FLEX (flexible PCG) also reduces r_{k+1}.z_k with the z of the finished V-cycle, before it is overwritten.
template <bool FLEX>
__global__ void __launch_bounds__(GRID_THREADS, 3) k_update_pr(Dev d, MGState m, float* __restrict__ p, unsigned long long handle) {
    pdl_entry();
    const float alpha = ratio_f(m.scalars[0], m.scalars[2]);
    const float* dcur = dir_buf(m, (m.ctl[0] + 1u) & 1u);
    struct V {
        float4 p, d, r, q, dg, z;
        uint32_t w;
    };
    w4_pass<FLEX ? 2 : 1, 2>(d, m, 3,
        [&](const Geo& g, const uint32_t*) {
            V v;
            v.p = ld4(p + g.i);
            v.d = ld4(dcur + g.i);
            v.r = ld4(m.r + g.i);
            v.q = ld4(m.q + g.i);
            v.dg = ld4(d.cell_diag + g.i);
            v.z = FLEX ? ld4(m.z + g.i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            v.w = quad_words(m, g);
            return v;
        },
        [&](const Geo& g, const V& v, double* v0, double* v1) {
            float po[4], ro[4], zo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                po[j] = comp(v.p, j);
                ro[j] = comp(v.r, j);
                zo[j] = 0.0f;
                if (!(w & W_FLUID)) continue;
                po[j] = comp(v.p, j) + alpha * comp(v.d, j);
                const float ri = comp(v.r, j) - alpha * comp(v.q, j);
                ro[j] = ri;
                zo[j] = (w & W_RED) ? red_init0(m, ri / (comp(v.dg, j) + DIAG_EPSILON)) : 0.0f;
                v0[j] = double(ri * ri);
                if (FLEX) v1[j] = double(ri * comp(v.z, j));
            }
            st4(p + g.i, po);
            st4(m.r + g.i, ro);
            st4(m.z + g.i, zo);
        },
        [&](double rr, double rz) {
            m.scalars[5] = rr;
            if (FLEX) m.scalars[9] = rz;
            const uint32_t it = m.ctl[0] + 1u;
            m.ctl[0] = it;
            const double bb = m.scalars[4];
            const double rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
            const bool converged = m.ctl[2] != 0u && rel <= m.scalars[8];
            const bool more = it < m.ctl[1] && !converged;
            if (!more) m.ctl[3] = 1u;
            if (!more && m.ctl[2] != 0u && !converged) m.ctl[4] = 1u;  // stopped at the limit: sticky for the frame
            if (handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
        });
}

// ---- ||b - A p||^2 (FP64 evaluation) and ||b||^2 of a finished solve (diagnostic) -------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_true_residual(Dev d, MGState m, const float* __restrict__ p,
                                                                const float* __restrict__ div) {
    pdl_entry();
    struct V {
        Q6 p;
        float4 dv, dg;
        uint32_t w;
    };
    w4_pass<2, 1>(d, m, 4,
        [&](const Geo& g, const uint32_t* ns) {
            V v;
            v.p = load_q6(p, g, ns);
            v.dv = ld4(div + g.i);
            v.dg = ld4(d.cell_diag + g.i);
            v.w = quad_words(m, g);
            return v;
        },
        [&](const Geo& g, const V& v, double* v0, double* v1) {
            const X2 x = partner(v.p);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t w = word_of(v.w, j);
                if (!(w & W_FLUID)) continue;
                const float diag = comp(v.dg, j) + DIAG_EPSILON;
                float n[6];
                nbrs6(v.p, x, g.h, j, n);
                const float b = -comp(v.dv, j);
                // evaluated in FP64 from the stored solution, so it measures the solution rather than the
                // cancellation of an FP32 evaluation of A p
                double nsum = 0.0;
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    if ((w >> k) & 1u) nsum = nsum + double(n[k]);
                const double r = double(b) - (double(diag) * double(comp(v.p.c, j)) - nsum);
                v0[j] = r * r;
                v1[j] = double(b * b);
            }
        },
        [&](double num, double den) { m.scalars[6] = num; m.scalars[7] = den; });
}

inline int blocks_for(uint32_t n, int threads) { return int((n + uint32_t(threads) - 1u) / uint32_t(threads)); }

// Level-0 passes straight from global memory (default) or from shared-memory stages filled by bulk copies
// (SLOSH_MG_STAGED=1). Both give identical results; the staged form measured slower on B200 (a 256^3 substep's
// pressure solve 2.94 against 2.75 ms: fewer long-scoreboard stalls, but fewer resident warps and more
// instructions), so it is kept as the measured alternative.
bool mg_staged() {
    static const int v = [] {
        const char* e = std::getenv("SLOSH_MG_STAGED");
        return (e && e[0] == '1') ? 1 : 0;
    }();
    return v != 0;
}
// Grid of a staged pass: every CTA resident at once (one wave), at most one warp per pool brick.
template <class K>
int st_grid(K kernel, size_t smem, const Dev& d, const Shape& sh) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, ST_WARPS * 32, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int cap = int((d.num_pool_bricks + uint32_t(ST_WARPS) - 1u) / uint32_t(ST_WARPS));
    return std::max(1, std::min(cap, per_sm * sh.num_sms));
}
#define ST_LAUNCH_ARGS(kernel, NF, NB, d, sh, s, ...)                                              \
    do {                                                                                            \
        constexpr size_t smem_ = st_smem_bytes<NF, NB>();                                           \
        static int grid_ = 0;                                                                       \
        if (!grid_) {                                                                               \
            if (smem_ > 48u * 1024u) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_)); \
            grid_ = st_grid(kernel, smem_, d, sh);                                                  \
        }                                                                                           \
        kernel<<<std::min(grid_, st_grid_cap(d)), ST_WARPS * 32, smem_, s>>>(__VA_ARGS__);          \
    } while (0)
#define ST_LAUNCH(kernel, NF, NB, d, m, sh, s) ST_LAUNCH_ARGS(kernel, NF, NB, d, sh, s, d, m)
inline int st_grid_cap(const Dev& d) { return std::max(1, int((d.num_pool_bricks + uint32_t(ST_WARPS) - 1u) / uint32_t(ST_WARPS))); }

}  // namespace

// Programmatic dependent launch of the solve's kernels (launch_k): on unless SLOSH_PDL=0.
bool pdl_enabled() {
    static const int v = [] {
        const char* e = std::getenv("SLOSH_PDL");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return v != 0;
}

int mg_tail_level(const MGState& m) {
    int t = m.num_levels - 1;
    while (t - 1 >= 1 && m.lv[t - 1].cells <= 4096u) --t;
    return t;
}

// First level of the cluster segment (k_vcycle_mid) for this hierarchy, 0 when the separate passes run (the
// default): SLOSH_MG_CLUSTER=2 or =3 starts it at that level, when the tail is at or below it and the GPU can
// place a cluster of MID_CLUSTER CTAs with the tail's shared memory.
int mid_level(const MGState& m, int tail) {
    static const int from = [] {
        const char* e = std::getenv("SLOSH_MG_CLUSTER");
        return e ? std::atoi(e) : 0;
    }();
    if (from < 2 || tail < from) return 0;
    static int ok = -1;
    static size_t checked_smem = 0;
    const size_t smem = mg_tail_smem(m);
    if (ok < 0 || smem > checked_smem) {
        ok = 0;
        if (cudaFuncSetAttribute(k_vcycle_mid, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
            cudaFuncSetAttribute(k_vcycle_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(MID_CLUSTER);
            cfg.blockDim = dim3(1024);
            cfg.dynamicSmemBytes = smem;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = MID_CLUSTER;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, k_vcycle_mid, &cfg) == cudaSuccess && clusters > 0) ok = 1;
        }
        cudaGetLastError();
        checked_smem = smem;
    }
    return ok ? from : 0;
}

int launch_mg_setup(const MGState& m, uint32_t limit, bool tol_mode, double tol, cudaStream_t s) {
    static size_t configured = 0;
    const size_t smem = mg_tail_smem(m);
    if (smem > 48u * 1024u && smem > configured) {
        cudaFuncSetAttribute(k_vcycle_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        configured = smem;
    }
    mid_level(m, mg_tail_level(m));
    launch_k(k_solve_setup, 1, 1, 0, s, m, limit, tol_mode ? 1u : 0u, tol);
    return 1;
}
// Grid of a footprint walk over level l (1-3): one thread per footprint cell of the pool's capacity, capped at the
// brick passes' width (a grid-stride loop).
static int fp_grid(const Dev& d, const Shape& sh, int l) {
    const uint64_t side = uint64_t(8 >> l);
    const uint64_t cells = uint64_t(d.num_pool_bricks - 1u) * side * side * side;
    return int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(sh.brick_ctas), (cells + 255u) / 256u)));
}
int launch_mg_build_type(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s) {
    const MGLevel& C = m.lv[l + 1];
    if (l + 1 <= 3) {
        cudaMemsetAsync(C.type, 0, size_t(C.cells) * sizeof(uint32_t), s);
        launch_k(k_build_type_fp, fp_grid(d, sh, l + 1), 256, 0, s, d, m.lv[l], C, l + 1);
        return 1;
    }
    launch_k(k_build_type, blocks_for(C.cells, 256), 256, 0, s, d, m.lv[l], C, l == 0 ? 1 : 0);
    return 1;
}
// The coarse types and stencil words of every level: levels 1-3 (those walked through the active bricks'
// footprints) by one launch each for the types and the words, the dense levels below them level by level.
int launch_mg_coarse_setup(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s) {
    const int nl = m.num_levels;
    if (nl < 2) return 0;
    const int top = std::min(3, nl - 1);
    int n = 0;
    for (int l = 1; l <= top; ++l) cudaMemsetAsync(m.lv[l].type, 0, size_t(m.lv[l].cells) * sizeof(uint32_t), s);
    launch_k(k_build_types_fp13, sh.mg_ctas, 256, 0, s, d, m, top);
    ++n;
    for (int l = top; l < nl - 1; ++l) n += launch_mg_build_type(d, m, l, sh, s);
    launch_k(k_level_words_fp13, fp_grid(d, sh, 1), 256, 0, s, d, m, top);
    ++n;
    for (int l = top + 1; l < nl; ++l) n += launch_mg_words(d, m, l, sh, s);
    return n;
}
int launch_pcg_init(const Dev& d, const MGState& m, const float* p, const float* div, unsigned long long handle, const Shape& sh,
                    cudaStream_t s, bool words) {
    if (words) launch_k(k_pcg_words, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
    launch_k(k_pcg_init, sh.mg_ctas, GRID_THREADS, 0, s, d, m, p, div, handle);
    return words ? 2 : 1;
}

size_t mg_tail_smem(const MGState& m) {
    uint32_t total = 0;
    tail_offsets(m, mg_tail_level(m), -1, &total);
    return total;
}
int launch_mg_words(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s) {
    if (l <= 3) launch_k(k_level_words_fp, fp_grid(d, sh, l), 256, 0, s, d, m.lv[l], l);
    else launch_k(k_level_words, blocks_for(m.lv[l].cells, 256), 256, 0, s, m.lv[l]);
    return 1;
}
int launch_mg_tail_lists(const MGState& m, cudaStream_t s) {
    if (m.num_levels < 2) return 0;
    launch_k(k_tail_lists, 1, 1024, 0, s, m, mg_tail_level(m));
    return 1;
}

// One V-cycle (SloshProxy.cpp:904-959), leaving rho = r.z in scalars[0] (previous rho in scalars[3]).
int launch_vcycle(const Dev& d, const MGState& m, int coarse_iterations, const Shape& sh, cudaStream_t s) {
    const int nl = m.num_levels;
    const bool relaxed = m.smooth_weight != 1.0f;  // over-relaxed level 0: the global-memory passes only
    const bool staged = mg_staged() && !relaxed;
    // prolonged: the first red sweep after k_prolong_smooth0, which with the over-relaxed smoother rebuilds the red
    // cells' prolonged values (the Gauss-Seidel value does not depend on them)
    auto smooth0_red = [&](bool dot, bool prolonged = false) {
        if (staged) {
            if (dot) ST_LAUNCH(k_smooth0_st<true>, 1, 2, d, m, sh, s);
            else ST_LAUNCH(k_smooth0_st<false>, 1, 2, d, m, sh, s);
        } else if (prolonged && relaxed) {
            if (dot) launch_k(k_smooth0<true, true>, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
            else launch_k(k_smooth0<false, true>, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
        } else {
            if (dot) launch_k(k_smooth0<true>, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
            else launch_k(k_smooth0<false>, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
        }
    };
    auto smooth0_black = [&]() {
        if (staged) ST_LAUNCH(k_smooth0_black_st, 1, 2, d, m, sh, s);
        else launch_k(k_smooth0_black, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
    };
    if (nl == 1) {
        launch_k(k_coarse_solve0, 1, 1024, 0, s, d, m, coarse_iterations);
        smooth0_red(true);
        return 2;
    }
    const int tail = mg_tail_level(m);
    // Footprint grids sized to the most cells a level can have in the pool's bricks.
    auto fp_blocks = [&](int l) {
        const uint32_t side = l <= 3 ? uint32_t(8 >> l) : 1u;
        const uint64_t cells = l <= 3 ? uint64_t(d.num_pool_bricks - 1u) * side * side * side : uint64_t(m.lv[l].cells);
        return int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(sh.brick_ctas), (cells + 255u) / 256u)));
    };
    // the one-colour passes (k_smooth_fp, k_prolong_smooth_fp) of levels 1 and 2 visit half the footprint
    auto fp_blocks_sweep = [&](int l) {
        if (l > 2) return fp_blocks(l);
        const uint32_t side = uint32_t(8 >> l);
        const uint64_t cells = uint64_t(d.num_pool_bricks - 1u) * side * side * side / 2u;
        return int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(sh.brick_ctas), (cells + 255u) / 256u)));
    };
    // Pre-smoothing: the black half of the first pair (the red half is the red initialisation written by
    // UpdatePR or the restriction), then sweeps - 1 red-black pairs. Post-smoothing: sweeps black-red pairs,
    // the first black half fused with the prolongation, the last red half of level 0 with rho = r.z.
    const int sweeps = std::max(m.sweeps, 1);
    int n = 0;
    smooth0_black();
    ++n;
    for (int k = 1; k < sweeps; ++k) {
        smooth0_red(false);
        smooth0_black();
        n += 2;
    }
    const int mid = mid_level(m, tail);  // levels mid..tail-1 and the tail in one cluster (0: separate passes)
    const int down_end = mid > 0 ? mid - 1 : tail;
    for (int l = 0; l < down_end; ++l) {
        if (l == 0) {
            if (staged) ST_LAUNCH(k_restrict0_st, 1, 2, d, m, sh, s);
            else launch_k(k_restrict0, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
        } else {
            launch_k(k_restrict_fp, fp_blocks(l + 1), 256, 0, s, d, m, l);
        }
        ++n;
        if (l + 1 < tail) {  // the tail kernel does its own pre-smoothing
            launch_k(k_smooth_fp, fp_blocks_sweep(l + 1), 256, 0, s, d, m, l + 1, 1u);
            ++n;
            for (int k = 1; k < sweeps; ++k) {
                launch_k(k_smooth_fp, fp_blocks_sweep(l + 1), 256, 0, s, d, m, l + 1, 0u);
                launch_k(k_smooth_fp, fp_blocks_sweep(l + 1), 256, 0, s, d, m, l + 1, 1u);
                n += 2;
            }
        }
    }
    if (mid > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(MID_CLUSTER);
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = mg_tail_smem(m);
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = MID_CLUSTER;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_vcycle_mid, d, m, mid, tail, coarse_iterations);
    } else {
        launch_k(k_vcycle_tail, 1, 1024, mg_tail_smem(m), s, m, tail, coarse_iterations);
    }
    ++n;
    for (int l = (mid > 0 ? mid - 1 : tail - 1); l >= 0; --l) {
        if (l == 0) {
            if (staged) ST_LAUNCH(k_prolong_smooth0_st, 1, 2, d, m, sh, s);
            else launch_k(k_prolong_smooth0, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
            for (int k = 1; k < sweeps; ++k) {
                smooth0_red(false, k == 1);
                smooth0_black();
                n += 2;
            }
            smooth0_red(true, sweeps == 1);
        } else {
            launch_k(k_prolong_smooth_fp, fp_blocks_sweep(l), 256, 0, s, d, m, l);
            for (int k = 1; k < sweeps; ++k) {
                launch_k(k_smooth_fp, fp_blocks_sweep(l), 256, 0, s, d, m, l, 0u);
                launch_k(k_smooth_fp, fp_blocks_sweep(l), 256, 0, s, d, m, l, 1u);
                n += 2;
            }
            launch_k(k_smooth_fp, fp_blocks_sweep(l), 256, 0, s, d, m, l, 0u);
        }
        n += 2;
    }
    return n;
}
int launch_pcg_apply_a(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s) {
    if (mg_staged()) ST_LAUNCH(k_apply_a_st, 2, 1, d, m, sh, s);
    else launch_k(k_apply_a, sh.mg_ctas, GRID_THREADS, 0, s, d, m);
    return 1;
}
int launch_pcg_update_pr(const Dev& d, const MGState& m, float* p, unsigned long long handle, const Shape& sh, cudaStream_t s) {
    if (mg_staged()) {
        if (m.flexible) ST_LAUNCH_ARGS(k_update_pr_st<true>, 0, 6, d, sh, s, d, m, p, handle);
        else ST_LAUNCH_ARGS(k_update_pr_st<false>, 0, 5, d, sh, s, d, m, p, handle);
    } else if (m.flexible) {
        launch_k(k_update_pr<true>, sh.mg_ctas, GRID_THREADS, 0, s, d, m, p, handle);
    } else {
        launch_k(k_update_pr<false>, sh.mg_ctas, GRID_THREADS, 0, s, d, m, p, handle);
    }
    return 1;
}
int launch_pcg_update_d(const Dev&, const MGState&, const Shape&, cudaStream_t) { return 0; }  // fused into ApplyA
int launch_true_residual(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s) {
    launch_k(k_true_residual, sh.mg_ctas, GRID_THREADS, 0, s, d, m, p, div);
    return 1;
}

}  // namespace slosh
