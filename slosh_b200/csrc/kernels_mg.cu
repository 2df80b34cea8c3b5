// Sparse-brick MGPCG pressure solve (sm_100a): McAdams-style multigrid-preconditioned CG with level 0
// in the brick pool and dense coarse levels.
//
// Reference: PLUG/Shaders/Private/SloshPressureMG.usf -- FINE_STENCIL (:142-157), MGBuildTypeCS
// (:256-278), PCGInitCS (:284-305), MGSmoothCS (:311-338), MGRestrictCS (:343-381), MGCoarseSolveCS
// (:386-413), MGProlongCS (:418-433), PCGApplyACS (:438-454), PCGFinalizeDotCS (:457-492),
// PCGUpdatePRCS (:495-524), PCGUpdateDCS (:527-543); driver SloshProxy.cpp:807-1020.
//
// Differences in form, not in result: the dot products are accumulated in FP64 through one fixed tree
// (a partial per active brick, then the last CTA to finish reduces the partials in a fixed order), so
// they are deterministic and need no separate finalize launch; alpha and beta are formed in FP64 and
// rounded to FP32. PCGInit and PCGUpdatePR also reduce ||b||^2 and ||r||^2 for the relative-residual
// stopping test.
#include "kernels.h"

namespace slosh {

namespace {

__device__ __forceinline__ uint32_t lin3(int3 c, int3 dim) { return uint32_t(c.x + dim.x * (c.y + dim.y * c.z)); }
__device__ __forceinline__ int3 coord3(uint32_t i, int3 dim) {
    return make_int3(int(i % uint32_t(dim.x)), int((i / uint32_t(dim.x)) % uint32_t(dim.y)), int(i / uint32_t(dim.x * dim.y)));
}
__device__ __forceinline__ bool inside3(int3 c, int3 dim) {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < dim.x && c.y < dim.y && c.z < dim.z;
}
__device__ __forceinline__ bool is_red(int3 c) { return (uint32_t(c.x + c.y + c.z) & 1u) == 0u; }

// Level-0 stencil (ghost-fluid diagonal DiagF + epsilon, sum of fluid neighbours of buf).
__device__ __forceinline__ void stencil0(const Dev& d, const float* __restrict__ buf, uint32_t i, int3 c, float& diag, float& sum) {
    sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        if (!in_grid(d, add3(c, nbr_off(n)))) continue;
        const uint32_t ni = nbr_index(d, i, c, n);
        if ((d.cell_type[ni] & CELL_TYPE_MASK) == CELL_FLUID) sum = sum + buf[ni];
    }
    diag = d.cell_diag[i] + DIAG_EPSILON;
}
// Dense coarse-level stencil (counted non-solid neighbours + epsilon).
__device__ __forceinline__ void stencil_dense(const MGLevel& L, const float* __restrict__ buf, int3 c, float& diag, float& sum) {
    diag = DIAG_EPSILON;
    sum = 0.0f;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const int3 nb = add3(c, nbr_off(n));
        if (!inside3(nb, L.dim)) continue;
        const uint32_t ni = lin3(nb, L.dim);
        const uint32_t t = L.type[ni] & CELL_TYPE_MASK;
        if (t != CELL_SOLID) diag = diag + 1.0f;
        if (t == CELL_FLUID) sum = sum + buf[ni];
    }
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
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t t = threadIdx.x + 256u * uint32_t(k);
        double acc = 0.0;
        for (uint32_t e = t; e < n; e += 1024u) acc = acc + __ldcg(partials + e);
        sm.lanes[t] = acc;
    }
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

// Level-0 pass over the active bricks producing up to two dot products. fn(i, c, v0, v1) handles one
// in-grid cell and sets its contributions; every thread runs the same number of brick iterations.
// The last CTA to finish reduces the partials and calls store(t0, t1) in thread 0.
template <int NDOT, class Fn, class Store>
__device__ __forceinline__ void level0_dot_pass(const Dev& d, const MGState& m, uint32_t counter, Fn fn, Store store) {
    __shared__ DotSmem sm;
    const uint32_t active = d.active_bricks[0];
    const uint32_t cap = d.num_pool_bricks;
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
        double a0[2] = {0.0, 0.0}, a1[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t l = threadIdx.x + uint32_t(k) * 256u;
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            if (in_grid(d, c)) fn(slot * BRICK_CELLS + l, c, a0[k], a1[k]);
        }
        const double t0 = brick_reduce(a0[0] + a0[1], sm.w8);
        if (threadIdx.x == 0) m.partials[e] = t0;
        if (NDOT > 1) {
            const double t1 = brick_reduce(a1[0] + a1[1], sm.w8);
            if (threadIdx.x == 0) m.partials[cap + e] = t1;
        }
    }
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

__device__ __forceinline__ float ratio_f(double num, double den) { return fabs(den) > 1e-30 ? float(num / den) : 0.0f; }

// ---- MGBuildTypeCS: coarse cell = air if any child is air, else fluid if any child is fluid ---------------
__global__ void k_build_type(Dev d, MGLevel fine, MGLevel coarse, int fine_is_pool) {
    const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= coarse.cells) return;
    const int3 c = coord3(ci, coarse.dim);
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

// ---- PCGInitCS (+ ||r0||^2 and ||b||^2) --------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_pcg_init(Dev d, MGState m, const float* __restrict__ p, const float* __restrict__ div) {
    level0_dot_pass<2>(d, m, 0,
        [&](uint32_t i, int3 c, double& v0, double& v1) {
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) {
                m.r[i] = 0.0f; m.z[i] = 0.0f; m.dvec[i] = 0.0f;
                return;
            }
            float diag, sum;
            stencil0(d, p, i, c, diag, sum);
            const float ri = -div[i] - (diag * p[i] - sum);
            m.r[i] = ri;
            m.z[i] = is_red(c) ? ri / diag : 0.0f;
            v0 = double(ri * ri);
            const float b = -div[i];
            v1 = double(b * b);
        },
        [&](double rr, double bb) { m.scalars[5] = rr; m.scalars[4] = bb; });
}

// ---- MGSmoothCS on level 0 (z as x, r as b); with dot the r.z reduction shifts rho -----------------------
__global__ void __launch_bounds__(GRID_THREADS) k_smooth0(Dev d, MGState m, uint32_t parity, int dot) {
    if (dot) {
        level0_dot_pass<1>(d, m, 1,
            [&](uint32_t i, int3 c, double& v0, double&) {
                if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
                if ((is_red(c) ? 0u : 1u) == parity) {
                    float diag, sum;
                    stencil0(d, m.z, i, c, diag, sum);
                    const float b = m.r[i];
                    const float x = (b + sum) / diag;
                    m.z[i] = x;
                    v0 = double(b * x);
                } else {
                    v0 = double(m.r[i] * m.z[i]);
                }
            },
            [&](double rho, double) { m.scalars[3] = m.scalars[0]; m.scalars[0] = rho; });
        return;
    }
    const uint32_t active = d.active_bricks[0];
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t l = threadIdx.x + uint32_t(k) * 256u;
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            if (!in_grid(d, c) || (is_red(c) ? 0u : 1u) != parity) continue;
            const uint32_t i = slot * BRICK_CELLS + l;
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) continue;
            float diag, sum;
            stencil0(d, m.z, i, c, diag, sum);
            m.z[i] = (m.r[i] + sum) / diag;
        }
    }
}

// ---- MGSmoothCS on a dense level -------------------------------------------------------------------------
__global__ void k_smooth_dense(MGLevel L, uint32_t parity) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.cells) return;
    if ((L.type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
    const int3 c = coord3(i, L.dim);
    if ((is_red(c) ? 0u : 1u) != parity) return;
    float diag, sum;
    stencil_dense(L, L.x, c, diag, sum);
    L.x[i] = (L.b[i] + sum) / diag;
}

// ---- MGRestrictCS -----------------------------------------------------------------------------------
__device__ __forceinline__ void restrict_store(MGLevel& C, uint32_t ci, int3 c, float sum) {
    const float b = 0.25f * sum;
    C.b[ci] = b;
    float cdiag = DIAG_EPSILON;
#pragma unroll
    for (int n = 0; n < 6; ++n) {
        const int3 nb = add3(c, nbr_off(n));
        const uint32_t t = inside3(nb, C.dim) ? (C.type[lin3(nb, C.dim)] & CELL_TYPE_MASK) : CELL_SOLID;
        cdiag = cdiag + (t != CELL_SOLID ? 1.0f : 0.0f);
    }
    C.x[ci] = is_red(c) ? b / cdiag : 0.0f;
}
// Level 0 -> 1 over the 4^3 level-1 cells of every active brick (SparseCoarse).
__global__ void k_restrict0(Dev d, MGState m) {
    MGLevel C = m.lv[1];
    const uint32_t active = d.active_bricks[0];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < active * 64u; t += gridDim.x * blockDim.x) {
        const uint32_t e = t >> 6, lc = t & 63u;
        const uint32_t brick = d.active_bricks[1u + e];
        const int3 bc = brick_coord_of(d, brick);
        const int3 c = make_int3(bc.x * 4 + int(lc & 3u), bc.y * 4 + int((lc >> 2) & 3u), bc.z * 4 + int(lc >> 4));
        if (!inside3(c, C.dim)) continue;
        const uint32_t ci = lin3(c, C.dim);
        if ((C.type[ci] & CELL_TYPE_MASK) != CELL_FLUID) { C.b[ci] = 0.0f; C.x[ci] = 0.0f; continue; }
        const uint32_t slot = __ldg(d.brick_table + brick);
        float sum = 0.0f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const int3 f = make_int3(c.x * 2 + (o & 1), c.y * 2 + ((o >> 1) & 1), c.z * 2 + ((o >> 2) & 1));
            if (!in_grid(d, f)) continue;
            const uint32_t fi = slot * BRICK_CELLS + local_index_of(f);
            if ((d.cell_type[fi] & CELL_TYPE_MASK) != CELL_FLUID) continue;
            float diag, nbsum;
            stencil0(d, m.z, fi, f, diag, nbsum);
            sum = sum + (m.r[fi] - (diag * m.z[fi] - nbsum));
        }
        restrict_store(C, ci, c, sum);
    }
}
__global__ void k_restrict_dense(MGLevel F, MGLevel C) {
    const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= C.cells) return;
    const int3 c = coord3(ci, C.dim);
    if ((C.type[ci] & CELL_TYPE_MASK) != CELL_FLUID) { C.b[ci] = 0.0f; C.x[ci] = 0.0f; return; }
    float sum = 0.0f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int3 f = make_int3(c.x * 2 + (o & 1), c.y * 2 + ((o >> 1) & 1), c.z * 2 + ((o >> 2) & 1));
        if (!inside3(f, F.dim)) continue;
        const uint32_t fi = lin3(f, F.dim);
        if ((F.type[fi] & CELL_TYPE_MASK) != CELL_FLUID) continue;
        float diag, nbsum;
        stencil_dense(F, F.x, f, diag, nbsum);
        sum = sum + (F.b[fi] - (diag * F.x[fi] - nbsum));
    }
    restrict_store(C, ci, c, sum);
}

// ---- MGCoarseSolveCS: red-black sweeps inside one CTA ------------------------------------------------------
__global__ void __launch_bounds__(1024) k_coarse_solve(Dev d, MGState m, int level, int iterations) {
    const bool pool = level == 0;
    const MGLevel L = m.lv[level];
    float* x = pool ? m.z : L.x;
    const float* b = pool ? m.r : L.b;
    for (int it = 0; it < iterations; ++it) {
        for (uint32_t colour = 0; colour < 2u; ++colour) {
            for (uint32_t li = threadIdx.x; li < L.cells; li += blockDim.x) {
                const int3 c = coord3(li, L.dim);
                if ((is_red(c) ? 0u : 1u) != colour) continue;
                if (pool) {
                    const uint32_t i = cell_index(d, c);
                    if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) continue;
                    float diag, sum;
                    stencil0(d, x, i, c, diag, sum);
                    x[i] = (b[i] + sum) / diag;
                } else {
                    if ((L.type[li] & CELL_TYPE_MASK) != CELL_FLUID) continue;
                    float diag, sum;
                    stencil_dense(L, x, c, diag, sum);
                    x[li] = (b[li] + sum) / diag;
                }
            }
            __syncthreads();
        }
    }
}

// ---- MGProlongCS: x_f += x_c(parent) on fluid cells whose parent is fluid ------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_prolong0(Dev d, MGState m) {
    const MGLevel C = m.lv[1];
    const uint32_t active = d.active_bricks[0];
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t l = threadIdx.x + uint32_t(k) * 256u;
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            if (!in_grid(d, c)) continue;
            const uint32_t i = slot * BRICK_CELLS + l;
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) continue;
            const uint32_t pi = lin3(make_int3(c.x / 2, c.y / 2, c.z / 2), C.dim);
            if ((C.type[pi] & CELL_TYPE_MASK) == CELL_FLUID) m.z[i] = m.z[i] + C.x[pi];
        }
    }
}
__global__ void k_prolong_dense(MGLevel F, MGLevel C) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.cells) return;
    if ((F.type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
    const int3 c = coord3(i, F.dim);
    const uint32_t pi = lin3(make_int3(c.x / 2, c.y / 2, c.z / 2), C.dim);
    if ((C.type[pi] & CELL_TYPE_MASK) == CELL_FLUID) F.x[i] = F.x[i] + C.x[pi];
}

// ---- PCGApplyACS: q = A d, d.q --------------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_apply_a(Dev d, MGState m) {
    level0_dot_pass<1>(d, m, 2,
        [&](uint32_t i, int3 c, double& v0, double&) {
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
            float diag, sum;
            stencil0(d, m.dvec, i, c, diag, sum);
            const float qi = diag * m.dvec[i] - sum;
            m.q[i] = qi;
            v0 = double(m.dvec[i] * qi);
        },
        [&](double dq, double) { m.scalars[2] = dq; });
}

// ---- PCGUpdatePRCS: p += alpha d, r -= alpha q, red pre-smooth; ||r||^2 ----------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_update_pr(Dev d, MGState m, float* __restrict__ p) {
    const float alpha = ratio_f(m.scalars[0], m.scalars[2]);
    level0_dot_pass<1>(d, m, 3,
        [&](uint32_t i, int3 c, double& v0, double&) {
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
            p[i] = p[i] + alpha * m.dvec[i];
            const float ri = m.r[i] - alpha * m.q[i];
            m.r[i] = ri;
            const float diag = d.cell_diag[i] + DIAG_EPSILON;
            m.z[i] = is_red(c) ? ri / diag : 0.0f;
            v0 = double(ri * ri);
        },
        [&](double rr, double) { m.scalars[5] = rr; });
}

// ---- PCGUpdateDCS: d = z + beta d ----------------------------------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_update_d(Dev d, MGState m, int first) {
    const float beta = first ? 0.0f : ratio_f(m.scalars[0], m.scalars[3]);
    const uint32_t active = d.active_bricks[0];
    for (uint32_t e = blockIdx.x; e < active; e += gridDim.x) {
        const uint32_t brick = d.active_bricks[1u + e];
        const uint32_t slot = __ldg(d.brick_table + brick);
        const int3 bc = brick_coord_of(d, brick);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t l = threadIdx.x + uint32_t(k) * 256u;
            const int3 lc = local_coord_of(l);
            const int3 c = make_int3(bc.x * 8 + lc.x, bc.y * 8 + lc.y, bc.z * 8 + lc.z);
            if (!in_grid(d, c)) continue;
            const uint32_t i = slot * BRICK_CELLS + l;
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) continue;
            m.dvec[i] = m.z[i] + beta * m.dvec[i];
        }
    }
}

// ---- ||b - A p||^2 and ||b||^2 of a finished solve (diagnostic) ---------------------------------------------
__global__ void __launch_bounds__(GRID_THREADS) k_true_residual(Dev d, MGState m, const float* __restrict__ p,
                                                                const float* __restrict__ div) {
    level0_dot_pass<2>(d, m, 4,
        [&](uint32_t i, int3 c, double& v0, double& v1) {
            if ((d.cell_type[i] & CELL_TYPE_MASK) != CELL_FLUID) return;
            float diag, sum;
            stencil0(d, p, i, c, diag, sum);
            const float r = -div[i] - (diag * p[i] - sum);
            v0 = double(r * r);
            const float b = -div[i];
            v1 = double(b * b);
        },
        [&](double num, double den) { m.scalars[6] = num; m.scalars[7] = den; });
}

inline int blocks_for(uint32_t n, int threads) { return int((n + uint32_t(threads) - 1u) / uint32_t(threads)); }

}  // namespace

int launch_mg_build_type(const Dev& d, const MGState& m, int l, cudaStream_t s) {
    const MGLevel& C = m.lv[l + 1];
    k_build_type<<<blocks_for(C.cells, 256), 256, 0, s>>>(d, m.lv[l], C, l == 0 ? 1 : 0);
    return 1;
}
int launch_pcg_init(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s) {
    k_pcg_init<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m, p, div);
    return 1;
}
int launch_mg_smooth(const Dev& d, const MGState& m, int l, uint32_t parity, bool dot, const Shape& sh, cudaStream_t s) {
    if (l == 0) {
        k_smooth0<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m, parity, dot ? 1 : 0);
    } else {
        k_smooth_dense<<<blocks_for(m.lv[l].cells, 256), 256, 0, s>>>(m.lv[l], parity);
    }
    return 1;
}
int launch_mg_restrict(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s) {
    if (l == 0) {
        k_restrict0<<<sh.brick_ctas, 256, 0, s>>>(d, m);
    } else {
        k_restrict_dense<<<blocks_for(m.lv[l + 1].cells, 256), 256, 0, s>>>(m.lv[l], m.lv[l + 1]);
    }
    return 1;
}
int launch_mg_coarse_solve(const Dev& d, const MGState& m, int l, int iterations, cudaStream_t s) {
    k_coarse_solve<<<1, 1024, 0, s>>>(d, m, l, iterations);
    return 1;
}
int launch_mg_prolong(const Dev& d, const MGState& m, int l, const Shape& sh, cudaStream_t s) {
    if (l == 0) {
        k_prolong0<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m);
    } else {
        k_prolong_dense<<<blocks_for(m.lv[l].cells, 256), 256, 0, s>>>(m.lv[l], m.lv[l + 1]);
    }
    return 1;
}
int launch_pcg_apply_a(const Dev& d, const MGState& m, const Shape& sh, cudaStream_t s) {
    k_apply_a<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m);
    return 1;
}
int launch_pcg_update_pr(const Dev& d, const MGState& m, float* p, const Shape& sh, cudaStream_t s) {
    k_update_pr<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m, p);
    return 1;
}
int launch_pcg_update_d(const Dev& d, const MGState& m, bool first, const Shape& sh, cudaStream_t s) {
    k_update_d<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m, first ? 1 : 0);
    return 1;
}
int launch_true_residual(const Dev& d, const MGState& m, const float* p, const float* div, const Shape& sh, cudaStream_t s) {
    k_true_residual<<<sh.brick_ctas, GRID_THREADS, 0, s>>>(d, m, p, div);
    return 1;
}
int launch_shift_rho(const MGState&, cudaStream_t) { return 0; }

}  // namespace slosh
