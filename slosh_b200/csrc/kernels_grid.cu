// Brick-pool allocator and per-cell grid passes of the Slosh substep (sm_100a).
//
// Reference kernels (PLUG/Shaders/Private/Slosh.usf): BrickFreeCS / BrickAllocCS / PoolArgsCS
// (:1719-1817), ClearNewSlotsCS (:1819-1831), BuildSolidCS (:365-395) fused into MarkCellsCS
// (:569-598), NormalizeFace (:604-651), ViscosityJacobiFace (:657-686), DivergenceCS (:692-741),
// DensityProjectionRhsCS (:775-805), DensityDisplacementFace (:808-828), PressureRBGSCS (:860-892),
// ProjectFace (:995-1052), ResidualCS (:1222-1257), ExtrapolateFace (:1263-1310).
//
// Every brick pass is a grid-stride loop of 256-thread CTAs over the active-brick list; thread t of a
// CTA owns cells t and t + 256 of the current brick, so each warp touches 32 consecutive cells of a
// 512-cell slot (fully coalesced 128-byte lines). The pass is HBM-bound; the launch shape is fixed
// (a multiple of the SM count) and the active count is read on the device, so no host round trip
// and a capturable stream.
#include "kernels.h"

namespace slosh {

namespace {

// Slots of the six face-neighbour bricks (-x, +x, -y, +y, -z, +z; 0 = the null slot when the neighbour
// brick lies outside the grid) of the brick this CTA visits in for_active_cells, loaded once per brick, so
// that a neighbour across the brick's faces costs no brick-table read.
__device__ __forceinline__ uint32_t* cta_nbr_slots() {
    __shared__ uint32_t s_slots[6];
    return s_slots;
}
// Neighbour n of cell (c, index) of the current brick: a fixed offset inside the brick, otherwise the
// same local cell with the axis coordinate wrapped in the neighbour brick's slot. Valid inside
// for_active_cells only; equal to nbr_index (common.cuh) there.
__device__ __forceinline__ uint32_t nbr_index_cta(uint32_t index, int3 c, int n) {
    const int a = n >> 1;
    const int l = comp(c, a) & 7;
    const bool plus = (n & 1) != 0;
    const uint32_t stride = a == 0 ? 1u : (a == 1 ? 8u : 64u);
    if (plus ? l < 7 : l > 0) return plus ? index + stride : index - stride;
    const uint32_t local = index & (BRICK_CELLS - 1u);
    return cta_nbr_slots()[n] * BRICK_CELLS + (plus ? local - 7u * stride : local + 7u * stride);
}
// Neighbour n of cell (c, index): from the CTA's neighbour slots (for_active_cells<true>) or through
// the brick table (for_active_cells<false>).
template <bool kSlots = true>
__device__ __forceinline__ uint32_t nbr_at(const Dev& d, uint32_t index, int3 c, int n) {
    return kSlots ? nbr_index_cta(index, c, n) : nbr_index(d, index, c, n);
}
// In-grid neighbour n of cell (c, index); out-of-grid neighbours resolve into the null brick.
template <bool kSlots = true>
__device__ __forceinline__ uint32_t nidx(const Dev& d, uint32_t index, int3 c, int n) {
    const int3 nb = add3(c, nbr_off(n));
    if (!in_grid(d, nb)) return local_index_of(nb);
    return nbr_at<kSlots>(d, index, c, n);
}
template <bool kSlots = true>
__device__ __forceinline__ uint32_t ntype(const Dev& d, uint32_t index, int3 c, int n) {
    const int3 nb = add3(c, nbr_off(n));
    if (!in_grid(d, nb)) return CELL_SOLID;
    return d.cell_type[nbr_at<kSlots>(d, index, c, n)];
}

// CellDensity (Slosh.usf:211-224).
__device__ float cell_density(const Dev& d, const Pass& p, int3 c) {
    if (!in_grid(d, c)) return 0.0f;
    float ws = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        ws = ws + (d.face_weight[face_index(d, a, c)] + d.face_weight[face_index(d, a, add3(c, axis_off(a)))]);
    return ws / (6.0f * p.target_ppc);
}
// AirFaceWeight (Slosh.usf:227-230).
__device__ __forceinline__ float air_face_weight(const Dev& d, const Pass& p, float rho_fluid, int3 air) {
    return p.ghost_fluid != 0u ? 1.0f / ghost_theta(rho_fluid, cell_density(d, p, air)) : 1.0f;
}
// CellDensityInterior (Slosh.usf:753-773) and whether a cell touches air, from one round of loads: the six
// neighbours' types (outside the grid: solid) and the weights of the cell's six faces (-x, +x, -y, +y, -z, +z), all
// issued before any is tested; the sums keep CellDensityInterior's order.
struct DensityNbrs {
    uint32_t nt[6];
    float w[6];
};
template <bool kSlots = true>
__device__ __forceinline__ DensityNbrs load_density_nbrs(const Dev& d, uint32_t index, int3 c) {
    DensityNbrs q;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const uint32_t ni = nidx<kSlots>(d, index, c, n);
        q.nt[n] = in_grid(d, add3(c, nbr_off(n))) ? d.cell_type[ni] : CELL_SOLID;
        const uint32_t a = uint32_t(n >> 1);
        q.w[n] = d.face_weight[a * d.pool_cells + ((n & 1) ? ni : index)];
    }
    return q;
}
__device__ __forceinline__ float density_interior_of(const Pass& p, const DensityNbrs& q) {
    float ws = 0.0f, faces = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        if (type_of(q.nt[n]) != CELL_SOLID) {
            ws = ws + q.w[n];
            faces = faces + 1.0f;
        }
    }
    return faces > 0.0f ? ws / (faces * p.target_ppc) : 1.0f;
}
__device__ __forceinline__ bool touches_air_of(const DensityNbrs& q) {
    bool t = false;
#pragma unroll
    for (int n = 0; n < 6; ++n) t = t || type_of(q.nt[n]) == CELL_AIR;
    return t;
}

// Visits the in-grid cells of the active bricks: fn(index, c); one brick per CTA iteration. With kSlots
// the brick's six face-neighbour slots are first loaded into shared memory (between two barriers), so
// nbr_index_cta resolves neighbours across the brick's faces without brick-table reads; then fn must not
// contain CTA barriers and every thread must call it. Passes with little work per brick (one colour of
// a sweep, no neighbours at all) take kSlots = false: no barriers, neighbours through the brick table.
template <bool kSlots, class Fn>
__device__ __forceinline__ void for_active_cells(const Dev& d, Fn fn) {
    const uint32_t active = d.active_bricks[0];
    uint32_t* ns = cta_nbr_slots();
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const int3 bc = brick_coord_of(d, brick);
        if (kSlots) {
            __syncthreads();  // the previous brick's cells are done with the neighbour slots
            if (threadIdx.x < 6u) {
                const int3 nb = add3(bc, nbr_off(int(threadIdx.x)));
                const bool in = nb.x >= 0 && nb.y >= 0 && nb.z >= 0 && nb.x < d.brick_dim.x && nb.y < d.brick_dim.y && nb.z < d.brick_dim.z;
                ns[threadIdx.x] = in ? __ldg(d.brick_table + brick_index_of(d, nb)) : 0u;
            }
        }
        const uint32_t slot = __ldg(d.brick_table + brick);
        if (kSlots) __syncthreads();
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t l = threadIdx.x + uint32_t(k) * 256u;
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            if (in_grid(d, c)) fn(slot * BRICK_CELLS + l, c);
        }
    }
}

// Block-wide exclusive scan of one value per thread (1024 threads). Returns the exclusive prefix;
// *total receives the sum.
__device__ uint32_t block_scan_1024(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = s_warp[lane];
        uint32_t ws = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, ws, off);
            if (lane >= off) ws += y;
        }
        s_warp[lane] = ws - w;  // exclusive prefix of warp totals
        if (lane == 31) s_warp[32] = ws;
    }
    __syncthreads();
    const uint32_t excl = s_warp[warp] + x - v;
    *total = s_warp[32];
    __syncthreads();
    return excl;
}

// ---- brick pool: BrickFreeCS + BrickAllocCS + PoolArgsCS -------------------------------------------------
// The reference pushes and pops the free stack with atomics, so slot assignment depends on thread timing. Here
// the same stack discipline runs in ascending brick order through scans: freed slots are pushed in brick order,
// the j-th brick needing storage pops entry (free count - j), and the active and new-slot lists come out in brick
// order. This is the serial (canonical) result. Four launches, one thread per brick in CTAs of 1,024 bricks:
//   k_pool_flags  wanted (touched within one brick: BrickAllocCS's 3x3x3 dilation) and held flags per brick, and
//                 each CTA's counts of bricks that free, need and keep a slot;
//   k_pool_plan   one CTA: the CTAs' exclusive offsets of the three counts, the stack's new top, the lists'
//                 lengths and the statistics;
//   k_pool_free   freed slots pushed at their offsets;
//   k_pool_alloc  slots popped in brick order (the pushes are complete), the active list, touch flags consumed.
// pool_scratch: [c] frees, [n + c] needs, [2n + c] keeps of CTA c (n CTAs), then the three offsets the same way,
// then the stack's old and new top.
constexpr uint32_t POOL_CTA = 1024u;
__device__ __forceinline__ uint32_t pool_ctas(uint32_t nb) { return (nb + POOL_CTA - 1u) / POOL_CTA; }

__global__ void __launch_bounds__(POOL_CTA) k_pool_flags(Dev d) {
    __shared__ uint32_t s_warp[33];
    const uint32_t b = blockIdx.x * POOL_CTA + threadIdx.x;
    const uint32_t nc = pool_ctas(d.num_bricks);
    uint32_t f = 0u;
    if (b < d.num_bricks) {
        const int3 c = brick_coord_of(d, b);
        const int bx = d.brick_dim.x, by = d.brick_dim.y, bz = d.brick_dim.z;
        uint32_t touched = 0u;
        for (int z = max(c.z - 1, 0); z <= min(c.z + 1, bz - 1); ++z)
            for (int y = max(c.y - 1, 0); y <= min(c.y + 1, by - 1); ++y)
                for (int x = max(c.x - 1, 0); x <= min(c.x + 1, bx - 1); ++x) touched |= d.brick_touch[uint32_t(x + bx * (y + by * z))];
        f = (touched != 0u ? 1u : 0u) | (d.brick_table_w[b] != 0u ? 2u : 0u);
        d.brick_want[b] = f;
    }
    uint32_t total;
    block_scan_1024(f == 2u ? 1u : 0u, s_warp, &total);  // held, not wanted: frees
    if (threadIdx.x == 0) d.pool_scratch[blockIdx.x] = total;
    block_scan_1024(f == 1u ? 1u : 0u, s_warp, &total);  // wanted, not held: needs
    if (threadIdx.x == 0) d.pool_scratch[nc + blockIdx.x] = total;
    block_scan_1024(f == 3u ? 1u : 0u, s_warp, &total);  // wanted and held: keeps
    if (threadIdx.x == 0) d.pool_scratch[2u * nc + blockIdx.x] = total;
}

// Exclusive scan of n per-CTA counts in place (1,024 threads, each over a contiguous run); returns the sum.
__device__ uint32_t pool_scan_runs(uint32_t* v, uint32_t* out, uint32_t n, uint32_t* s_warp) {
    const uint32_t per = (n + blockDim.x - 1u) / blockDim.x;
    const uint32_t c0 = min(threadIdx.x * per, n), c1 = min(c0 + per, n);
    uint32_t sum = 0u;
    for (uint32_t c = c0; c < c1; ++c) sum += v[c];
    uint32_t total;
    uint32_t run = block_scan_1024(sum, s_warp, &total);
    for (uint32_t c = c0; c < c1; ++c) {
        const uint32_t t = v[c];
        out[c] = run;
        run += t;
    }
    __syncthreads();
    return total;
}
__global__ void __launch_bounds__(1024) k_pool_plan(Dev d) {
    __shared__ uint32_t s_warp[33];
    const uint32_t nc = pool_ctas(d.num_bricks);
    uint32_t* cnt = d.pool_scratch;
    uint32_t* off = d.pool_scratch + 3u * nc;
    const int f0 = int(d.free_slots[0]);
    const uint32_t total_free = pool_scan_runs(cnt, off, nc, s_warp);
    const uint32_t total_need = pool_scan_runs(cnt + nc, off + nc, nc, s_warp);
    const int f = f0 + int(total_free);
    // a CTA's active bricks: those keeping their slot and those of its needs whose pop finds a slot (rank < f)
    for (uint32_t c = threadIdx.x; c < nc; c += blockDim.x) {
        const int got = min(max(f - int(off[nc + c]), 0), int(cnt[nc + c]));
        cnt[2u * nc + c] += uint32_t(got);
    }
    __syncthreads();
    const uint32_t total_act = pool_scan_runs(cnt + 2u * nc, off + 2u * nc, nc, s_warp);
    if (threadIdx.x == 0) {
        d.pool_scratch[6u * nc] = uint32_t(f0);
        d.pool_scratch[6u * nc + 1u] = uint32_t(f);
        const uint32_t ok = uint32_t(min(int(total_need), max(f, 0)));
        d.new_slots[0] = ok;
        d.free_slots[0] = uint32_t(max(f - int(total_need), 0));
        d.active_bricks[0] = total_act;
        d.stats[8] += total_need - ok;
        d.stats[7] = max(d.stats[7], total_act);
    }
}
__global__ void __launch_bounds__(POOL_CTA) k_pool_free(Dev d) {
    __shared__ uint32_t s_warp[33];
    const uint32_t b = blockIdx.x * POOL_CTA + threadIdx.x;
    const uint32_t nc = pool_ctas(d.num_bricks);
    const uint32_t f = b < d.num_bricks ? d.brick_want[b] : 0u;
    uint32_t total;
    const uint32_t k = block_scan_1024(f == 2u ? 1u : 0u, s_warp, &total) + d.pool_scratch[3u * nc + blockIdx.x];
    if (f == 2u) {
        const uint32_t f0 = d.pool_scratch[6u * nc];
        const uint32_t slot = d.brick_table_w[b];
        d.free_slots[1u + f0 + k] = slot;
        d.slot_brick[slot] = NO_BRICK;
        d.brick_table_w[b] = 0u;
    }
}
__global__ void __launch_bounds__(POOL_CTA) k_pool_alloc(Dev d) {
    __shared__ uint32_t s_warp[33];
    const uint32_t b = blockIdx.x * POOL_CTA + threadIdx.x;
    const uint32_t nc = pool_ctas(d.num_bricks);
    const uint32_t f = b < d.num_bricks ? d.brick_want[b] : 0u;
    uint32_t total;
    const uint32_t j = block_scan_1024(f == 1u ? 1u : 0u, s_warp, &total) + d.pool_scratch[4u * nc + blockIdx.x];
    bool act = f == 3u;
    if (f == 1u) {
        const int count = int(d.pool_scratch[6u * nc + 1u]) - int(j);
        if (count > 0) {
            const uint32_t slot = d.free_slots[count];
            d.brick_table_w[b] = slot;
            d.slot_brick[slot] = b;
            d.new_slots[1u + j] = slot;
            act = true;
        }
    }
    const uint32_t a = block_scan_1024(act ? 1u : 0u, s_warp, &total) + d.pool_scratch[5u * nc + blockIdx.x];
    if (act) d.active_bricks[1u + a] = b;
    if (b < d.num_bricks) d.brick_touch[b] = 0u;
}

__global__ void k_clear_new_slots(Dev d) {  // ClearNewSlotsCS
    const uint32_t n = d.new_slots[0];
    for (uint32_t e = blockIdx.x; e < n; e += gridDim.x) {
        const uint32_t base = d.new_slots[1u + e] * BRICK_CELLS;
        for (uint32_t l = threadIdx.x; l < BRICK_CELLS; l += blockDim.x) {
            d.pressure[base + l] = 0.0f;
            d.cell_count[base + l] = 0;
            d.density_q[base + l] = 0.0f;
        }
    }
}

// ---- BuildSolidCS fused into MarkCellsCS -------------------------------------------------------------
// BuildSolid runs before P2G in the reference but P2G never reads CellType, so classifying solids here,
// just before the count-based fluid marking, gives the same types in one pass over the cells.
__global__ void __launch_bounds__(GRID_THREADS) k_mark_cells(Dev d, Pass p) {
    uint32_t fluid = 0;
    for_active_cells<false>(d, [&](uint32_t index, int3 c) {
        const int count = d.cell_count[index];  // loaded before the collider tests, like the pressure
        const float pressure = d.pressure[index];
        uint32_t packed = CELL_AIR;
        if (c.x == 0 || c.y == 0 || c.z == 0 || c.x == d.grid.x - 1 || c.y == d.grid.y - 1 || c.z == d.grid.z - 1) {
            packed = CELL_SOLID;
        } else {
            const float3 x = make_float3((float(c.x) + 0.5f) * d.h, (float(c.y) + 0.5f) * d.h, (float(c.z) + 0.5f) * d.h);
            float best = 0.0f;
            for (uint32_t k = 0; k < p.num_colliders; ++k) {
                const float s = collider_sdf(d.colliders[k], x);
                if (s < best) { best = s; packed = CELL_SOLID | ((k + 1u) << CELL_COLLIDER_SHIFT); }
            }
        }
        if (type_of(packed) != CELL_SOLID) {
            packed = count > 0 ? CELL_FLUID : CELL_AIR;
            if (float(count) >= 0.5f * p.target_ppc) packed |= CELL_DENSE_FLAG;
        }
        d.cell_type[index] = packed;
        if (type_of(packed) == CELL_FLUID) {
            d.pressure[index] = pressure * p.warm_start_scale;
            ++fluid;
        } else {
            d.pressure[index] = 0.0f;
        }
    });
    fluid = __reduce_add_sync(0xFFFFFFFFu, fluid);
    if ((threadIdx.x & 31) == 0 && fluid) atomicAdd(d.stats + 1, fluid);
}

// ---- NormalizeFace ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_normalize(Dev d, Pass p, float* __restrict__ vel) {
    const uint32_t tf = d.total_faces;
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        // the cell's and the three lower neighbours' types and the three faces' sums, before any store
        const uint32_t b = d.cell_type[index];
        int moms[3], wts[3];
        uint32_t tas[3];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            moms[axis] = d.accum[f];
            wts[axis] = d.accum[tf + f];
            tas[axis] = d.cell_type[nidx(d, index, c, 2 * axis)];
        }
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            const int mom = moms[axis], wt = wts[axis];
            if (mom != 0 || wt != 0) { d.accum[f] = 0; d.accum[tf + f] = 0; }
            float u = wt > 0 ? float(mom) / float(wt) : 0.0f;
            d.face_weight[f] = float(wt) * P2G_FIXED_INV;
            uint32_t flags = wt > 0 ? FACE_HAS_WEIGHT : 0u;
            if (p.use_apic == 0u) d.vel_old[f] = u;
            const uint32_t a = in_grid(d, add3(c, nbr_off(2 * axis))) ? tas[axis] : CELL_SOLID;
            if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                const uint32_t solid = type_of(b) == CELL_SOLID ? b : a;
                const uint32_t id = collider_of(solid);
                if (id == 0u) {
                    u = 0.0f;
                } else {
                    const float3 x = make_float3((float(c.x) + (axis == 0 ? 0.0f : 0.5f)) * d.h,
                                                 (float(c.y) + (axis == 1 ? 0.0f : 0.5f)) * d.h,
                                                 (float(c.z) + (axis == 2 ? 0.0f : 0.5f)) * d.h);
                    const float3 v = collider_velocity_at(d.colliders[id - 1u], x);
                    const float3 e = make_float3(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f);
                    u = dot3(v, e);
                }
                if (!(type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID)) flags |= FACE_VALID | FACE_SOLID;
            } else if (type_of(a) == CELL_FLUID || type_of(b) == CELL_FLUID) {
                u = u + p.gravity[axis] * p.dt;
                flags |= FACE_VALID;
            } else {
                u = 0.0f;
            }
            vel[f] = u;
            d.face_flags[f] = flags;
        }
    });
}

// ---- ViscosityJacobiFace -----------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_viscosity(Dev d, Pass p, const float* __restrict__ ustar,
                                                            const float* __restrict__ src, float* __restrict__ dst) {
    const float alpha = p.viscosity_alpha;
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            const uint32_t flags = d.face_flags[f];
            const float center = src[f];
            if ((flags & FACE_VALID) == 0u || (flags & FACE_SOLID) != 0u) { dst[f] = center; continue; }
            float sum = 0.0f;
            for (int n = 0; n < 6; ++n) {
                float value = center;
                if (in_grid(d, add3(c, nbr_off(n)))) {
                    const uint32_t ni = uint32_t(axis) * d.pool_cells + nbr_index_cta(index, c, n);
                    if ((d.face_flags[ni] & FACE_VALID) != 0u) value = src[ni];
                }
                sum = sum + value;
            }
            dst[f] = (ustar[f] + alpha * sum) / (1.0f + 6.0f * alpha);
        }
    });
}

// ---- DivergenceCS --------------------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_divergence(Dev d, Pass p, const float* __restrict__ vel) {
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        // one round of loads: the cell's type, its six faces' velocities and weights and its neighbours' types
        // (a neighbour outside the grid reads the null brick and counts as solid); only cells beside air load
        // more (the air cells' densities)
        const uint32_t type = d.cell_type[index];
        uint32_t nbr[6], nts[6];
        float vlo[3], vhi[3], wlo[3], whi[3];
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            nbr[n] = nidx(d, index, c, n);
            nts[n] = d.cell_type[nbr[n]];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            vlo[a] = vel[uint32_t(a) * d.pool_cells + index];
            vhi[a] = vel[uint32_t(a) * d.pool_cells + nbr[2 * a + 1]];
            wlo[a] = d.face_weight[uint32_t(a) * d.pool_cells + index];
            whi[a] = d.face_weight[uint32_t(a) * d.pool_cells + nbr[2 * a + 1]];
        }
        d.cell_count[index] = 0;
        if (type_of(type) != CELL_FLUID) {
            d.divergence[index] = 0.0f;
            d.cell_diag[index] = 0.0f;
            return;
        }
        float div = 0.0f;
        float ws = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) div = div + (vhi[a] - vlo[a]);
#pragma unroll
        for (int a = 0; a < 3; ++a) ws = ws + (wlo[a] + whi[a]);
        const float rho = ws / (6.0f * p.target_ppc);
        const float excess = fmaxf(rho - (1.0f + p.density_deadband), 0.0f);
        const float target = fminf(p.density_correction * excess, 0.5f) * d.h / p.dt;
        d.divergence[index] = div - target;
        float diag = 0.0f;
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const int3 nc = add3(c, nbr_off(n));
            const uint32_t nt = in_grid(d, nc) ? type_of(nts[n]) : CELL_SOLID;
            diag = diag + (nt == CELL_FLUID ? 1.0f : (nt == CELL_AIR ? air_face_weight(d, p, rho, nc) : 0.0f));
        }
        d.cell_diag[index] = diag;
    });
}

// ---- PressureRBGSCS: one SOR colour sweep ----------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_rbgs(Dev d, float* __restrict__ pres, const float* __restrict__ rhs,
                                                       uint32_t parity, float omega) {
    for_active_cells<false>(d, [&](uint32_t index, int3 c) {
        if (type_of(d.cell_type[index]) != CELL_FLUID) return;
        if ((uint32_t(c.x + c.y + c.z) & 1u) != parity) return;
        float sum = 0.0f;
        const float diag = d.cell_diag[index];
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const int3 nb = add3(c, nbr_off(n));
            if (!in_grid(d, nb)) continue;
            const uint32_t ni = nbr_at<false>(d, index, c, n);
            if (type_of(d.cell_type[ni]) == CELL_FLUID) sum = sum + pres[ni];
        }
        if (diag > 0.0f) {
            const float gs = (sum - rhs[index]) / diag;
            const float old = pres[index];
            pres[index] = old + omega * (gs - old);
        }
    });
}

// ---- ProjectFace (its two-way coupling terms are accumulated by k_coupling_faces after the pass) ---------
// Every value a face may need (the neighbour's type and pressure, the cell's pressure, the face's velocity
// and flags) is loaded before the types are tested, so a cell costs one round of loads; a neighbour outside
// the grid reads the null brick and counts as solid. Only faces between fluid and air load more (the
// densities of the ghost-fluid weight).
__global__ void __launch_bounds__(GRID_THREADS) k_project(Dev d, Pass p, float* __restrict__ vel) {
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        const uint32_t b = d.cell_type[index];
        const float pc = d.pressure[index];
        uint32_t ta[3], fl[3];
        float pn[3], vf[3];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            const uint32_t ni = nidx(d, index, c, 2 * axis);
            ta[axis] = d.cell_type[ni];
            pn[axis] = d.pressure[ni];
            fl[axis] = d.face_flags[f];
            vf[axis] = vel[f];
        }
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            const int3 ca = add3(c, nbr_off(2 * axis));
            const uint32_t a = in_grid(d, ca) ? ta[axis] : CELL_SOLID;
            uint32_t flags = fl[axis] & FACE_HAS_WEIGHT;
            if (type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID) {
            } else if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                flags |= FACE_VALID | FACE_SOLID;
            } else if (type_of(a) == CELL_FLUID || type_of(b) == CELL_FLUID) {
                float pa, pb;
                if (type_of(a) == CELL_FLUID && type_of(b) == CELL_FLUID) {
                    pa = pn[axis];
                    pb = pc;
                } else if (type_of(a) == CELL_FLUID) {
                    pa = pn[axis];
                    pb = pa - pa * air_face_weight(d, p, cell_density(d, p, ca), c);
                } else {
                    pb = pc;
                    pa = pb - pb * air_face_weight(d, p, cell_density(d, p, c), ca);
                }
                vel[f] = vf[axis] - (pb - pa);
                flags |= FACE_VALID;
            }
            d.face_flags[f] = flags;
        }
    });
}

// ---- two-way collider coupling (Slosh.usf:897-993, 1062-1216, 1316-1370) ---------------------------------
// Per-collider integer accumulators in 1/1024 fixed point, so the totals do not depend on the order of the
// atomic additions. Slots: 0-2 force, 3-5 torque, 6 wetted faces, 7 submerged cells, 8-10 fluid velocity
// sum, 11 solid cells, 12-14 submerged centroid offset sum.
__device__ __forceinline__ bool two_way(const Dev& d, uint32_t k) { return (d.colliders[k].flags & COLLIDER_FLAG_TWO_WAY) != 0u; }
__device__ __forceinline__ void coupling_add(const Dev& d, uint32_t k, int slot, float v) {
    atomicAdd(d.coupling + k * SLOSH_COUPLING_STRIDE + uint32_t(slot), __float2int_rn(v * COUPLING_SCALE));
}
__device__ __forceinline__ void coupling_count(const Dev& d, uint32_t k, int slot) {
    atomicAdd(d.coupling + k * SLOSH_COUPLING_STRIDE + uint32_t(slot), 1);
}
__device__ __forceinline__ float3 face_position(const Dev& d, int axis, int3 f) {  // Slosh.usf:204-208
    return make_float3((float(f.x) + (axis == 0 ? 0.0f : 0.5f)) * d.h, (float(f.y) + (axis == 1 ? 0.0f : 0.5f)) * d.h,
                       (float(f.z) + (axis == 2 ? 0.0f : 0.5f)) * d.h);
}
// CellCenterVelocity, Slosh.usf:897-906.
__device__ __forceinline__ float3 cell_center_velocity(const Dev& d, const float* vel, int3 c) {
    float out[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = 0.5f * (vel[face_index(d, a, c)] + vel[face_index(d, a, add3(c, nbr_off(2 * a + 1)))]);
    return make_float3(out[0], out[1], out[2]);
}
// AccumulatePressureForce, Slosh.usf:913-925.
__device__ void accumulate_pressure_force(const Dev& d, const Pass& p, uint32_t k, float3 face_pos, float3 into, float p_hat) {
    const float pa = p_hat * p.pressure_to_pascal;
    const float3 force = scale3((pa * d.h) * d.h, into);
    const float3 torque = cross3(sub3(face_pos, ld3(d.colliders[k].center)), force);
    coupling_add(d, k, 0, force.x); coupling_add(d, k, 1, force.y); coupling_add(d, k, 2, force.z);
    coupling_add(d, k, 3, torque.x); coupling_add(d, k, 4, torque.y); coupling_add(d, k, 5, torque.z);
}
// AccumulateCoupling, Slosh.usf:929-946.
__device__ void accumulate_coupling(const Dev& d, const Pass& p, const float* vel, uint32_t k, int3 fluid_cell, float3 face_pos,
                                    float3 into, float p_hat) {
    if (!two_way(d, k)) return;
    if (p.smooth_coupling == 0u) accumulate_pressure_force(d, p, k, face_pos, into, p_hat);
    const float3 fv = cell_center_velocity(d, vel, fluid_cell);
    coupling_count(d, k, 6);
    coupling_add(d, k, 8, fv.x); coupling_add(d, k, 9, fv.y); coupling_add(d, k, 10, fv.z);
}
// EstimateSeepagePressure, Slosh.usf:952-977.
__device__ bool seepage_pressure(const Dev& d, int3 body, uint32_t id, float& p_hat) {
    const int3 dirs[4] = {make_int3(1, 0, 0), make_int3(-1, 0, 0), make_int3(0, 1, 0), make_int3(0, -1, 0)};
    float sum = 0.0f, count = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int3 q = body;
        for (int step = 0; step < 16; ++step) {
            q = add3(q, dirs[k]);
            const uint32_t t = get_cell_type(d, q);
            if (type_of(t) != CELL_SOLID || collider_of(t) != id) {
                if (type_of(t) == CELL_FLUID) {
                    sum = sum + d.pressure[cell_index(d, q)];
                    count = count + 1.0f;
                }
                break;
            }
        }
    }
    p_hat = count > 0.0f ? sum / count : 0.0f;
    return count > 0.0f;
}
// AccumulateContact, Slosh.usf:979-992.
__device__ void accumulate_contact(const Dev& d, const Pass& p, uint32_t solid_packed, int3 body, float3 face_pos, float3 into) {
    const uint32_t id = collider_of(solid_packed);
    if (id == 0u || !two_way(d, id - 1u)) return;
    float ph;
    if (seepage_pressure(d, body, id, ph)) accumulate_pressure_force(d, p, id - 1u, face_pos, into, ph);
}
// The coupling terms of ProjectFace (Slosh.usf:1004-1029), on the projected field after the projection
// pass (the reference samples the wetted-face velocity while the same pass writes it).
__global__ void __launch_bounds__(GRID_THREADS) k_coupling_faces(Dev d, Pass p, const float* __restrict__ vel) {
    for_active_cells<false>(d, [&](uint32_t index, int3 c) {
        const uint32_t b = d.cell_type[index];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const int3 ca = add3(c, nbr_off(2 * axis));
            const uint32_t a = get_cell_type(d, ca);
            const float3 e = make_float3(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f);
            const float3 ne = make_float3(axis == 0 ? -1.0f : 0.0f, axis == 1 ? -1.0f : 0.0f, axis == 2 ? -1.0f : 0.0f);
            if (type_of(a) == CELL_SOLID && type_of(b) == CELL_SOLID) {
                if (collider_of(a) != collider_of(b)) {
                    const float3 fp = face_position(d, axis, c);
                    accumulate_contact(d, p, b, c, fp, e);
                    accumulate_contact(d, p, a, ca, fp, ne);
                }
            } else if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                if (type_of(a) == CELL_FLUID && collider_of(b) != 0u)
                    accumulate_coupling(d, p, vel, collider_of(b) - 1u, ca, face_position(d, axis, c), e, d.pressure[cell_index(d, ca)]);
                else if (type_of(b) == CELL_FLUID && collider_of(a) != 0u)
                    accumulate_coupling(d, p, vel, collider_of(a) - 1u, c, face_position(d, axis, c), ne, d.pressure[index]);
            }
        }
    });
}
// FluidPressureGradient, Slosh.usf:1086-1101.
__device__ float3 fluid_pressure_gradient(const Dev& d, int3 c, float pc) {
    float g[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int3 cp = add3(c, nbr_off(2 * a + 1)), cm = add3(c, nbr_off(2 * a));
        const bool bp = type_of(get_cell_type(d, cp)) == CELL_FLUID, bm = type_of(get_cell_type(d, cm)) == CELL_FLUID;
        const float pp = bp ? d.pressure[cell_index(d, cp)] : 0.0f;
        const float pm = bm ? d.pressure[cell_index(d, cm)] : 0.0f;
        g[a] = bp && bm ? (pp - pm) * 0.5f : (bp ? pp - pc : (bm ? pc - pm : 0.0f));
    }
    return make_float3(g[0] * d.inv_h, g[1] * d.inv_h, g[2] * d.inv_h);
}
// BodySurfacePressure, Slosh.usf:1105-1125.
__device__ bool body_surface_pressure(const Dev& d, int3 c, float& p_hat) {
    float sum = 0.0f, count = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const int3 dd = nbr_off(n);
        const int3 nb = add3(c, dd);
        if (type_of(get_cell_type(d, nb)) == CELL_FLUID) {
            const float pn = d.pressure[cell_index(d, nb)];
            const int3 nb2 = add3(nb, dd);
            const float slope = type_of(get_cell_type(d, nb2)) == CELL_FLUID ? d.pressure[cell_index(d, nb2)] - pn : 0.0f;
            sum = sum + (pn - 0.5f * slope);
            count = count + 1.0f;
        }
    }
    p_hat = count > 0.0f ? sum / count : 0.0f;
    return count > 0.0f;
}
// CouplingForceCS, Slosh.usf:1127-1216.
__global__ void __launch_bounds__(GRID_THREADS) k_coupling_force(Dev d, Pass p) {
    for_active_cells<false>(d, [&](uint32_t index, int3 c) {
        const uint32_t packed = d.cell_type[index];
        const uint32_t type = type_of(packed);
        if (type == CELL_AIR) return;
        const float h = d.h;
        const float3 x = make_float3((float(c.x) + 0.5f) * h, (float(c.y) + 0.5f) * h, (float(c.z) + 0.5f) * h);
        float p_hat = 0.0f;
        float3 g = make_float3(0.0f, 0.0f, 0.0f);
        bool have = false;
        if (type == CELL_FLUID) {
            p_hat = d.pressure[index];
            g = fluid_pressure_gradient(d, c, p_hat);
            have = true;
        } else if (collider_of(packed) != 0u) {
            have = body_surface_pressure(d, c, p_hat);
        }
        if (!have) return;
        for (uint32_t k = 0; k < p.num_colliders; ++k) {
            const slosh_collider_t& col = d.colliders[k];
            if ((col.flags & COLLIDER_FLAG_TWO_WAY) == 0u || fabsf(collider_sdf(col, x)) > h) continue;
            if (type == CELL_SOLID && collider_of(packed) != k + 1u) continue;
            float sp = p_hat;
            if (type == CELL_FLUID) {
                const float phi = collider_sdf(col, x);
                sp = sp + dot3(g, scale3(-phi, collider_normal(col, x, 0.25f * h)));
            }
            const float scale = (((-sp) * p.pressure_to_pascal) * h) * h;
            float3 force = make_float3(0.0f, 0.0f, 0.0f), torque = make_float3(0.0f, 0.0f, 0.0f);
            const float3 center = ld3(col.center);
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const int3 dd = nbr_off(n);
                const float3 normal = make_float3(float(dd.x), float(dd.y), float(dd.z));
                const float3 fp = addf3(x, scale3(0.5f * h, normal));
                if (type == CELL_SOLID) {
                    const uint32_t nbp = get_cell_type(d, add3(c, dd));
                    if (type_of(nbp) == CELL_SOLID && collider_of(nbp) != k + 1u) continue;
                }
                const float w = saturatef(0.5f + collider_sdf(col, fp) * d.inv_h);
                const float3 df = scale3(scale * w, normal);
                force = addf3(force, df);
                torque = addf3(torque, cross3(sub3(fp, center), df));
            }
            coupling_add(d, k, 0, force.x); coupling_add(d, k, 1, force.y); coupling_add(d, k, 2, force.z);
            coupling_add(d, k, 3, torque.x); coupling_add(d, k, 4, torque.y); coupling_add(d, k, 5, torque.z);
        }
    });
}
// SubmergedCS, Slosh.usf:1316-1370.
__global__ void __launch_bounds__(GRID_THREADS) k_submerged(Dev d) {
    for_active_cells<false>(d, [&](uint32_t index, int3 c) {
        const uint32_t packed = d.cell_type[index];
        const uint32_t id = collider_of(packed);
        if (type_of(packed) != CELL_SOLID || id == 0u) return;
        coupling_count(d, id - 1u, 11);
        const int3 dirs[4] = {make_int3(1, 0, 0), make_int3(-1, 0, 0), make_int3(0, 1, 0), make_int3(0, -1, 0)};
        bool sub = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int3 q = c;
            for (int step = 0; step < 12; ++step) {
                q = add3(q, dirs[k]);
                const uint32_t t = get_cell_type(d, q);
                if (type_of(t) != CELL_SOLID || collider_of(t) != id) {
                    bool liquid = type_of(t) == CELL_FLUID && (t & CELL_DENSE_FLAG) != 0u;
#pragma unroll
                    for (int below = 1; below <= 3; ++below)
                        liquid = liquid && type_of(get_cell_type(d, make_int3(q.x, q.y, q.z - below))) != CELL_AIR;
                    sub = sub || liquid;
                    break;
                }
            }
        }
        if (sub) {
            const float h = d.h;
            const float3 off = sub3(make_float3((float(c.x) + 0.5f) * h, (float(c.y) + 0.5f) * h, (float(c.z) + 0.5f) * h),
                                    ld3(d.colliders[id - 1u].center));
            coupling_count(d, id - 1u, 7);
            coupling_add(d, id - 1u, 12, off.x); coupling_add(d, id - 1u, 13, off.y); coupling_add(d, id - 1u, 14, off.z);
        }
    });
}

// ---- ResidualCS ------------------------------------------------------------------------------------------
// The statistics are integers (the maximum rate's bits, fixed-point sums modulo 2^32, counts), so each thread
// accumulates its cells, each warp reduces them, and one lane adds the warp's totals: the same values as one
// atomic per cell, without every fluid cell contending for the same five words.
__global__ void __launch_bounds__(GRID_THREADS) k_residual(Dev d, Pass p, const float* __restrict__ vel) {
    uint32_t max_bits = 0u, rate_sum = 0u, cells = 0u, dens_sum = 0u, interior = 0u;
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        if (type_of(d.cell_type[index]) != CELL_FLUID) return;
        // one round of loads: the faces' velocities, the neighbours' types and the face weights
        float vlo[3], vhi[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            vhi[a] = vel[uint32_t(a) * d.pool_cells + nidx(d, index, c, 2 * a + 1)];
            vlo[a] = vel[uint32_t(a) * d.pool_cells + index];
        }
        const DensityNbrs q = load_density_nbrs(d, index, c);
        float div = 0.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) div = div + (vhi[a] - vlo[a]);
        const float rate = fabsf(div) * d.inv_h;
        max_bits = max(max_bits, __float_as_uint(rate));
        rate_sum += __float2uint_rz(fminf(rate, 1.0e5f) * 1000.0f);
        ++cells;
        if (!touches_air_of(q)) {
            const float dens = clampf(density_interior_of(p, q), 0.0f, 4.0f);
            dens_sum += uint32_t(__float2int_rn((dens - 1.0f) * 10000.0f));
            ++interior;
        }
    });
    max_bits = __reduce_max_sync(0xFFFFFFFFu, max_bits);
    rate_sum = __reduce_add_sync(0xFFFFFFFFu, rate_sum);
    cells = __reduce_add_sync(0xFFFFFFFFu, cells);
    dens_sum = __reduce_add_sync(0xFFFFFFFFu, dens_sum);
    interior = __reduce_add_sync(0xFFFFFFFFu, interior);
    if ((threadIdx.x & 31u) == 0u && cells > 0u) {
        atomicMax(d.stats + 2, max_bits);
        atomicAdd(d.stats + 3, rate_sum);
        atomicAdd(d.stats + 4, cells);
        if (interior > 0u) {
            atomicAdd(d.stats + 5, dens_sum);
            atomicAdd(d.stats + 6, interior);
        }
    }
}

// ---- DensityProjectionRhsCS -------------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_density_rhs(Dev d, Pass p) {
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        d.density_q[index] = 0.0f;
        if (type_of(d.cell_type[index]) != CELL_FLUID) { d.density_rhs[index] = 0.0f; return; }
        const DensityNbrs q = load_density_nbrs(d, index, c);
        float dev = density_interior_of(p, q) - 1.0f;
        if (touches_air_of(q)) dev = fmaxf(dev, 0.0f);
        d.density_rhs[index] = -p.density_relaxation * clampf(dev, -0.5f, 0.5f);
    });
}

// ---- DensityDisplacementFace -----------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_density_displacement(Dev d, float* __restrict__ dst) {
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        const uint32_t b = d.cell_type[index];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            const uint32_t a = ntype(d, index, c, 2 * axis);
            float value;
            if (type_of(a) == CELL_SOLID || type_of(b) == CELL_SOLID) {
                value = 0.0f;
            } else {
                const float qa = type_of(a) == CELL_FLUID ? d.density_q[nbr_index_cta(index, c, 2 * axis)] : 0.0f;
                const float qb = type_of(b) == CELL_FLUID ? d.density_q[index] : 0.0f;
                value = -(qb - qa);
            }
            dst[f] = value;
        }
    });
}

// ---- ExtrapolateFace -------------------------------------------------------------------------------------------
// In place: a layer writes only faces unknown so far (the average of their known neighbours, with the layer's bit,
// or zero), and every reader uses only faces known from earlier layers, which no layer writes, so the result equals
// the reference's pass from one buffer into another. A face's own new bit is written while neighbours read its
// flags; readers only test bits set by earlier layers, so the result does not depend on the interleaving. Known
// faces cost one flag load (the two-buffer form copies their values).
__global__ void __launch_bounds__(GRID_THREADS) k_extrapolate(Dev d, float* vel, uint32_t iteration) {
    uint32_t known = FACE_VALID;
    for (uint32_t it = 0; it < iteration; ++it) known |= 1u << (FACE_EXTRAP_SHIFT + it);
    const uint32_t new_bit = 1u << (FACE_EXTRAP_SHIFT + iteration);
    for_active_cells<true>(d, [&](uint32_t index, int3 c) {
        uint32_t fls[3];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) fls[axis] = d.face_flags[uint32_t(axis) * d.pool_cells + index];
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t flags = fls[axis];
            if ((flags & known) != 0u) continue;
            const uint32_t f = uint32_t(axis) * d.pool_cells + index;
            // the face's value and all six neighbours' flags and values are loaded before any is tested (an
            // out-of-grid neighbour reads the null slot and is then skipped)
            const float center = vel[f];
            uint32_t nf[6];
            float nv[6];
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const uint32_t ni = uint32_t(axis) * d.pool_cells + nbr_index_cta(index, c, n);
                nf[n] = d.face_flags[ni];
                nv[n] = vel[ni];
            }
            float sum = 0.0f, count = 0.0f;
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                if (!in_grid(d, add3(c, nbr_off(n)))) continue;
                if ((nf[n] & known) != 0u && (nf[n] & FACE_SOLID) == 0u) { sum = sum + nv[n]; count = count + 1.0f; }
            }
            if (count > 0.0f) {
                vel[f] = sum / count;
                d.face_flags[f] = flags | new_bit;
            } else if (__float_as_uint(center) != 0u) {
                vel[f] = 0.0f;
            }
        }
    });
}

}  // namespace

int launch_pool_update(const Dev& d, cudaStream_t s) {
    const uint32_t nc = (d.num_bricks + POOL_CTA - 1u) / POOL_CTA;
    k_pool_flags<<<nc, POOL_CTA, 0, s>>>(d);
    k_pool_plan<<<1, 1024, 0, s>>>(d);
    k_pool_free<<<nc, POOL_CTA, 0, s>>>(d);
    k_pool_alloc<<<nc, POOL_CTA, 0, s>>>(d);
    return 4;
}
size_t pool_scratch_words(uint32_t num_bricks) { return 6u * size_t((num_bricks + POOL_CTA - 1u) / POOL_CTA) + 2u; }
int launch_clear_new_slots(const Dev& d, const Shape& sh, cudaStream_t s) {
    k_clear_new_slots<<<sh.brick_ctas, 256, 0, s>>>(d);
    return 1;
}
int launch_mark_cells(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s) {
    k_mark_cells<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p);
    return 1;
}
int launch_normalize_faces(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s) {
    k_normalize<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, vel);
    return 1;
}
int launch_viscosity(const Dev& d, const Pass& p, const float* ustar, const float* src, float* dst, const Shape& sh, cudaStream_t s) {
    k_viscosity<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, ustar, src, dst);
    return 1;
}
int launch_divergence(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s) {
    k_divergence<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, vel);
    return 1;
}
int launch_rbgs(const Dev& d, float* pres, const float* rhs, uint32_t parity, float omega, const Shape& sh, cudaStream_t s) {
    k_rbgs<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, pres, rhs, parity, omega);
    return 1;
}
int launch_project(const Dev& d, const Pass& p, float* vel, const Shape& sh, cudaStream_t s) {
    k_project<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, vel);
    return 1;
}
int launch_coupling(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s) {
    if (p.num_colliders == 0u) return 0;
    k_coupling_faces<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, vel);
    if (p.smooth_coupling == 0u) return 1;
    k_coupling_force<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p);
    return 2;
}
int launch_submerged(const Dev& d, const Shape& sh, cudaStream_t s) {
    k_submerged<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d);
    return 1;
}
int launch_residual(const Dev& d, const Pass& p, const float* vel, const Shape& sh, cudaStream_t s) {
    k_residual<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p, vel);
    return 1;
}
int launch_density_rhs(const Dev& d, const Pass& p, const Shape& sh, cudaStream_t s) {
    k_density_rhs<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, p);
    return 1;
}
int launch_density_displacement(const Dev& d, float* dst, const Shape& sh, cudaStream_t s) {
    k_density_displacement<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, dst);
    return 1;
}
int launch_extrapolate(const Dev& d, float* vel, uint32_t iteration, const Shape& sh, cudaStream_t s) {
    k_extrapolate<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, vel, iteration);
    return 1;
}

}  // namespace slosh
