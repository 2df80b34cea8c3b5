// Kernels of the learned warm start (sm_100a): TMA + tcgen05 implicit-GEMM convolution and weight
// gradient, pooling / upsampling and their gradients, the 1x1 head with the masked MSE loss, Adam,
// and the dense input / guess exchange with the sparse brick pool. Layouts and forms: unet.h.
#include <cstdlib>

#include "tc.cuh"
#include "unet.h"

namespace slosh {
namespace unet {
namespace {

using namespace tc;

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }

// Tile t of the volume: its origin and batch entry.
struct TileOrigin {
    int x0, y0, z0, b;
    uint64_t v0;  // linear voxel of row 0 (rows are consecutive voxels)
};
__device__ __forceinline__ TileOrigin tile_origin(const Vol& v, uint32_t t) {
    const uint32_t tx = v.W / v.bx, ty = v.H / v.by, tz = v.D / v.bz;
    TileOrigin o;
    o.x0 = int((t % tx) * v.bx);
    t /= tx;
    o.y0 = int((t % ty) * v.by);
    t /= ty;
    o.z0 = int((t % tz) * v.bz);
    o.b = int(t / tz);
    o.v0 = ((uint64_t(o.b) * v.D + uint64_t(o.z0)) * v.H + uint64_t(o.y0)) * v.W + uint64_t(o.x0);
    return o;
}
__device__ __forceinline__ void tap_offset(uint32_t tap, int& dx, int& dy, int& dz) {
    dx = int(tap % 3u) - 1;
    dy = int((tap / 3u) % 3u) - 1;
    dz = int(tap / 9u) - 1;
}
__device__ __forceinline__ uint8_t* align1024(uint8_t* p) { return p + ((1024u - (smem_u32(p) & 1023u)) & 1023u); }
__device__ __forceinline__ uint32_t tmem_cols(uint32_t n) { return n <= 32u ? 32u : (n <= 64u ? 64u : (n <= 128u ? 128u : 256u)); }

// ---- implicit-GEMM convolution -----------------------------------------------------------------------
// Persistent and warp-specialised: CTA b takes tiles b, b + gridDim.x, ...; warp 0 (one lane) loads with
// TMA, warp 1 (one lane) issues the MMAs, warps 2-5 run the epilogue (warp w reads TMEM lanes 32 (w % 4)
// .. +31, so tile row r = 32 (w % 4) + lane is that thread's voxel). The stage ring runs across tiles;
// the accumulator is double-buffered in TMEM (2 x N columns), so one tile's epilogue overlaps the next
// tile's loads and MMAs; several such CTAs share an SM. Stage s holds A (128 rows x C of one tap and K-block) at stage offset 0 and B
// (N rows x C) at a_region; both are K-major with the swizzle of their row length (2 C bytes): 8-row
// groups 16 C bytes apart (SBO), the K = 16 steps 32 bytes apart.
constexpr int CONV_THREADS = 192;
constexpr int CONV_MAX_STAGES = 8;
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__global__ void __launch_bounds__(CONV_THREADS) k_conv3d(const __grid_constant__ ConvArgs a, uint32_t stage_bytes, uint32_t a_region,
                                                        uint32_t stages) {
    extern __shared__ uint8_t dsm[];
    __shared__ __align__(8) uint64_t full[CONV_MAX_STAGES], empty[CONV_MAX_STAGES], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    uint8_t* base = align1024(dsm);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t ncols = tmem_cols(a.n);
    const uint32_t tiles = a.vol.tiles();
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&acc_full[k], 1);
            mbar_init(&acc_empty[k], 128);
        }
        fence_mbar_init();
        for (uint32_t k = 0; k < a.nblocks; ++k) {
            prefetch_map(&a.act[k]);
            prefetch_map(&a.wgt[k]);
        }
    }
    if (warp == 0) tmem_alloc(&tmem_slot, 2u * ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t niter = 27u * a.nblocks;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t g = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                const TileOrigin o = tile_origin(a.vol, t);
                for (uint32_t it = 0; it < niter; ++it, ++g) {
                    const uint32_t s = g % stages;
                    if (g >= stages && !mbar_wait(&empty[s], ((g / stages) - 1u) & 1u, a.error, 1u)) {
                        ok = false;
                        break;
                    }
                    const uint32_t tap = it / a.nblocks, blk = it % a.nblocks, cb = a.cb[blk];
                    int dx, dy, dz;
                    tap_offset(tap, dx, dy, dz);
                    uint8_t* sa = base + s * stage_bytes;
                    mbar_arrive_expect_tx(&full[s], cb * 256u + cb * a.n * 2u);
                    tma_load_5d(sa, &a.act[blk], 0, o.x0 + dx, o.y0 + dy, o.z0 + dz, o.b, &full[s]);
                    tma_load_2d(sa + a_region, &a.wgt[blk], 0, int(tap * a.n), &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(128u, a.n, 0u, 0u);
            uint32_t g = 0, tl = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++tl) {
                const uint32_t acc = tl & 1u;
                if (tl >= 2u && !mbar_wait(&acc_empty[acc], ((tl >> 1) - 1u) & 1u, a.error, 2u)) break;
                tc_fence_after();
                const uint32_t dcol = tmem + acc * ncols;
                for (uint32_t it = 0; it < niter; ++it, ++g) {
                    const uint32_t s = g % stages;
                    if (!mbar_wait(&full[s], (g / stages) & 1u, a.error, 2u)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t cb = a.cb[it % a.nblocks];
                    const uint32_t row = cb * 2u, layout = swizzle_of_row_bytes(row);
                    const uint32_t sa = smem_u32(base + s * stage_bytes), sb = sa + a_region;
                    for (uint32_t k = 0; k < cb / 16u; ++k)
                        mma_bf16(dcol, smem_desc(sa + 32u * k, 16u, 8u * row, layout), smem_desc(sb + 32u * k, 16u, 8u * row, layout),
                                 idesc, (it | k) != 0u ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                mma_commit(&acc_full[acc]);
            }
        }
    } else {
        const uint32_t q = warp & 3u;  // TMEM lane quarter of this warp
        const uint32_t r = q * 32u + lane;
        uint32_t tl = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
            const uint32_t acc = tl & 1u;
            const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait(&acc_full[acc], (tl >> 1) & 1u, a.error, 4u));
            tc_fence_after();
            if (!ok) break;
            const TileOrigin o = tile_origin(a.vol, t);
            const uint64_t v = o.v0 + r;
            for (uint32_t c0 = 0; c0 < a.n; c0 += 16u) {
                float x[16];
                tmem_ld16(tmem + acc * ncols + ((q * 32u) << 16) + c0, x);
                if (a.bias)
#pragma unroll
                    for (int j = 0; j < 16; ++j) x[j] = x[j] + a.bias[c0 + uint32_t(j)];
                if (a.relu)
#pragma unroll
                    for (int j = 0; j < 16; ++j) x[j] = fmaxf(x[j], 0.0f);
                const uint32_t oi = c0 < a.oc[0] ? 0u : 1u;
                const uint32_t cc = oi == 0u ? c0 : c0 - a.oc[0];
                const uint64_t e = v * a.oc[oi] + cc;
                uint4* dst = reinterpret_cast<uint4*>(a.out[oi] + e);
                if (a.accumulate) {
                    const uint4 w0 = dst[0], w1 = dst[1];
                    const bf16* old0 = reinterpret_cast<const bf16*>(&w0);
                    const bf16* old1 = reinterpret_cast<const bf16*>(&w1);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        x[j] = x[j] + bf(old0[j]);
                        x[8 + j] = x[8 + j] + bf(old1[j]);
                    }
                }
                if (a.mask[oi]) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask[oi] + e);
                    const uint4 m0 = mp[0], m1 = mp[1];
                    const bf16* mk0 = reinterpret_cast<const bf16*>(&m0);
                    const bf16* mk1 = reinterpret_cast<const bf16*>(&m1);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        if (!(bf(mk0[j]) > 0.0f)) x[j] = 0.0f;
                        if (!(bf(mk1[j]) > 0.0f)) x[8 + j] = 0.0f;
                    }
                }
                uint4 w[2];
                bf16* wb = reinterpret_cast<bf16*>(w);
#pragma unroll
                for (int j = 0; j < 16; ++j) wb[j] = __float2bfloat16_rn(x[j]);
                dst[0] = w[0];
                dst[1] = w[1];
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[acc]);
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2u * ncols);
    }
}

// ---- halo-box implicit-GEMM convolution ------------------------------------------------------------------
// Tile = 8 (x) x 16 (y) x 1 (z) output voxels; TMEM row r = x + 8 y. Per tile and 8-channel plane of each
// K-block, one TMA load brings the 10 x 18 x 3 halo box (zero-filled outside the volume) into shared memory
// as [z][y][x][8 channels], 16 bytes per voxel: in the no-swizzle K-major layout every 8 consecutive x of
// one (y, z) line are a contiguous 128-byte core matrix. The A operand of tap (dx, dy, dz) is the box shifted
// by ((dz + 1) 18 + dy + 1) 160 + (dx + 1) 16 bytes: 8-row groups (the tile's y lines) 160 bytes apart (SBO),
// the two planes of a K = 16 step one plane apart (LBO). The weights of all taps sit in shared memory as
// [tap][plane][n][8 channels] (core matrices of 8 output channels, LBO = one plane of n rows, SBO = 128).
// Warp 0 loads halo boxes (nbuf = 1 or 2 buffers across tiles), warp 1 issues the 27 x K / 16 MMAs of a tile,
// warps 2-5 run the same epilogue as k_conv3d. Every wait is bounded.
constexpr uint32_t HALO_X = 10u, HALO_Y = 18u, HALO_Z = 3u;
constexpr uint32_t HALO_PLANE_BYTES = HALO_X * HALO_Y * HALO_Z * 16u;  // 8640
constexpr uint32_t HALO_PLANE = 8704u;                                 // plane stride, a multiple of 128
__global__ void __launch_bounds__(CONV_THREADS) k_conv3d_halo(const __grid_constant__ ConvArgs a, uint32_t wbytes, uint32_t hbytes,
                                                             uint32_t nbuf) {
    extern __shared__ uint8_t dsm[];
    __shared__ __align__(8) uint64_t hfull[2], hempty[2], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    uint8_t* base = align1024(dsm);
    uint8_t* wsm = base;
    uint8_t* hsm = base + ((wbytes + 1023u) & ~1023u);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t ncols = tmem_cols(a.n);
    const uint32_t tiles = a.vol.tiles();
    uint32_t planes[2] = {a.cb[0] / 8u, a.nblocks > 1u ? a.cb[1] / 8u : 0u};
    const uint32_t wk1 = 27u * planes[0] * a.n * 16u;  // byte offset of K-block 1's weights
    // weights [27][n][cb] -> [tap][plane][n][8], 16-byte chunks
    for (uint32_t k = 0; k < a.nblocks; ++k) {
        const uint32_t cb = a.cb[k], pk = planes[k];
        const uint32_t chunks = 27u * a.n * pk;
        const uint4* src = reinterpret_cast<const uint4*>(a.w_ptr[k]);
        uint8_t* dst = wsm + (k ? wk1 : 0u);
        for (uint32_t c = threadIdx.x; c < chunks; c += blockDim.x) {
            const uint32_t p = c % pk, row = c / pk;  // row = tap n + nn
            const uint32_t tap = row / a.n, nn = row % a.n;
            *reinterpret_cast<uint4*>(dst + ((tap * pk + p) * a.n + nn) * 16u) = src[(size_t(row) * cb) / 8u + p];
        }
    }
    fence_async_shared();  // the MMAs read the weights through the async proxy
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; ++k) {
            mbar_init(&hfull[k], 1);
            mbar_init(&hempty[k], 1);
            mbar_init(&acc_full[k], 1);
            mbar_init(&acc_empty[k], 128);
        }
        fence_mbar_init();
        for (uint32_t k = 0; k < a.nblocks; ++k) prefetch_map(&a.halo[k]);
    }
    if (warp == 0) tmem_alloc(&tmem_slot, 2u * ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t ptotal = planes[0] + planes[1];

    if (warp == 0) {
        if (lane == 0) {
            uint32_t tl = 0;
            for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
                const uint32_t hb = tl % nbuf;
                if (tl >= nbuf && !mbar_wait(&hempty[hb], ((tl / nbuf) - 1u) & 1u, a.error, 64u)) break;
                const TileOrigin o = tile_origin(a.vol, t);
                uint8_t* h = hsm + hb * hbytes;
                mbar_arrive_expect_tx(&hfull[hb], ptotal * HALO_PLANE_BYTES);
                uint32_t pl = 0;
                for (uint32_t k = 0; k < a.nblocks; ++k)
                    for (uint32_t p = 0; p < planes[k]; ++p, ++pl)
                        tma_load_5d(h + pl * HALO_PLANE, &a.halo[k], int(8u * p), o.x0 - 1, o.y0 - 1, o.z0 - 1, o.b, &hfull[hb]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(128u, a.n, 0u, 0u);
            const uint32_t wsa = smem_u32(wsm), hsa = smem_u32(hsm);
            uint32_t tl = 0;
            for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
                const uint32_t acc = tl & 1u, hb = tl % nbuf;
                if (tl >= 2u && !mbar_wait(&acc_empty[acc], ((tl >> 1) - 1u) & 1u, a.error, 2u)) break;
                if (!mbar_wait(&hfull[hb], (tl / nbuf) & 1u, a.error, 2u)) break;
                tc_fence_after();
                const uint32_t dcol = tmem + acc * ncols;
                const uint32_t h = hsa + hb * hbytes;
                uint32_t accumulate = 0u;
                for (uint32_t tap = 0; tap < 27u; ++tap) {
                    int dx, dy, dz;
                    tap_offset(tap, dx, dy, dz);
                    const uint32_t shift = (uint32_t(dz + 1) * HALO_Y + uint32_t(dy + 1)) * HALO_X * 16u + uint32_t(dx + 1) * 16u;
                    uint32_t pl = 0;
                    for (uint32_t k = 0; k < a.nblocks; ++k) {
                        const uint32_t wb = wsa + (k ? wk1 : 0u) + tap * planes[k] * a.n * 16u;
                        for (uint32_t ks = 0; ks < planes[k] / 2u; ++ks) {
                            const uint64_t ad = smem_desc(h + (pl + 2u * ks) * HALO_PLANE + shift, HALO_PLANE, HALO_X * 16u, SWZ_NONE);
                            const uint64_t bd = smem_desc(wb + 2u * ks * a.n * 16u, a.n * 16u, 128u, SWZ_NONE);
                            mma_bf16(dcol, ad, bd, idesc, accumulate);
                            accumulate = 1u;
                        }
                        pl += planes[k];
                    }
                }
                mma_commit(&hempty[hb]);
                mma_commit(&acc_full[acc]);
            }
        }
    } else {
        const uint32_t q = warp & 3u;  // TMEM lane quarter of this warp
        const uint32_t r = q * 32u + lane;
        uint32_t tl = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
            const uint32_t acc = tl & 1u;
            const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait(&acc_full[acc], (tl >> 1) & 1u, a.error, 4u));
            tc_fence_after();
            if (!ok) break;
            const TileOrigin o = tile_origin(a.vol, t);
            const uint64_t v = o.v0 + uint64_t(r >> 3) * a.vol.W + (r & 7u);
            for (uint32_t c0 = 0; c0 < a.n; c0 += 16u) {
                float x[16];
                tmem_ld16(tmem + acc * ncols + ((q * 32u) << 16) + c0, x);
                if (a.bias)
#pragma unroll
                    for (int j = 0; j < 16; ++j) x[j] = x[j] + a.bias[c0 + uint32_t(j)];
                if (a.relu)
#pragma unroll
                    for (int j = 0; j < 16; ++j) x[j] = fmaxf(x[j], 0.0f);
                const uint32_t oi = c0 < a.oc[0] ? 0u : 1u;
                const uint32_t cc = oi == 0u ? c0 : c0 - a.oc[0];
                const uint64_t e = v * a.oc[oi] + cc;
                uint4* dst = reinterpret_cast<uint4*>(a.out[oi] + e);
                if (a.accumulate) {
                    const uint4 w0 = dst[0], w1 = dst[1];
                    const bf16* old0 = reinterpret_cast<const bf16*>(&w0);
                    const bf16* old1 = reinterpret_cast<const bf16*>(&w1);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        x[j] = x[j] + bf(old0[j]);
                        x[8 + j] = x[8 + j] + bf(old1[j]);
                    }
                }
                if (a.mask[oi]) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask[oi] + e);
                    const uint4 m0 = mp[0], m1 = mp[1];
                    const bf16* mk0 = reinterpret_cast<const bf16*>(&m0);
                    const bf16* mk1 = reinterpret_cast<const bf16*>(&m1);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        if (!(bf(mk0[j]) > 0.0f)) x[j] = 0.0f;
                        if (!(bf(mk1[j]) > 0.0f)) x[8 + j] = 0.0f;
                    }
                }
                uint4 w[2];
                bf16* wb = reinterpret_cast<bf16*>(w);
#pragma unroll
                for (int j = 0; j < 16; ++j) wb[j] = __float2bfloat16_rn(x[j]);
                dst[0] = w[0];
                dst[1] = w[1];
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[acc]);
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2u * ncols);
    }
}

// ---- weight gradient ------------------------------------------------------------------------------------
// CTA (chunk, group): taps g*T .. g*T+T-1 (T = 128 / c) over the chunk's voxel tiles. Stage s: A =
// T regions of 128 voxel rows x c (tap t's shifted input), B = 128 voxel rows x n (dZ). Both are
// MN-major: A's MN atoms (c channels, one per tap) are 256 c bytes apart (LBO), 8-voxel groups 16 c
// bytes apart (SBO); B has one atom, 8-voxel groups 16 n bytes apart. K = 16 voxels per MMA.
__global__ void __launch_bounds__(128) k_wgrad(const __grid_constant__ WgradArgs a, uint32_t stage_bytes, uint32_t a_region) {
    extern __shared__ uint8_t dsm[];
    __shared__ __align__(8) uint64_t full[WGRAD_STAGES], empty[WGRAD_STAGES], done;
    __shared__ uint32_t tmem_slot;
    uint8_t* base = align1024(dsm);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t T = 128u / a.c, g = blockIdx.y, chunk = blockIdx.x;
    const uint32_t tiles = a.vol.tiles();
    const uint32_t t_begin = chunk * a.tiles_per_chunk;
    const uint32_t t_end = min(tiles, t_begin + a.tiles_per_chunk);
    const uint32_t ncols = tmem_cols(a.n);
    if (threadIdx.x == 0) {
        for (int s = 0; s < WGRAD_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        fence_mbar_init();
        prefetch_map(&a.act);
        prefetch_map(&a.grad);
    }
    if (warp == 0) tmem_alloc(&tmem_slot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t niter = t_end > t_begin ? t_end - t_begin : 0u;
    const uint32_t region = 256u * a.c;  // one tap's 128 rows x c channels

    if (warp == 0 && lane == 0) {
        for (uint32_t it = 0; it < niter; ++it) {
            const uint32_t s = it % WGRAD_STAGES;
            if (it >= uint32_t(WGRAD_STAGES) && !mbar_wait(&empty[s], ((it / WGRAD_STAGES) - 1u) & 1u, a.error, 8u)) break;
            const TileOrigin o = tile_origin(a.vol, t_begin + it);
            uint8_t* sa = base + s * stage_bytes;
            uint32_t taps = 0;
            for (uint32_t t = 0; t < T; ++t)
                if (g * T + t < 27u) ++taps;
            mbar_arrive_expect_tx(&full[s], taps * region + 256u * a.n);
            for (uint32_t t = 0; t < T; ++t) {
                const uint32_t tap = g * T + t;
                if (tap >= 27u) break;
                int dx, dy, dz;
                tap_offset(tap, dx, dy, dz);
                tma_load_5d(sa + t * region, &a.act, 0, o.x0 + dx, o.y0 + dy, o.z0 + dz, o.b, &full[s]);
            }
            tma_load_5d(sa + a_region, &a.grad, 0, o.x0, o.y0, o.z0, o.b, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16_f32(128u, a.n, 1u, 1u);
        const uint32_t la = swizzle_of_row_bytes(2u * a.c), lb = swizzle_of_row_bytes(2u * a.n);
        for (uint32_t it = 0; it < niter; ++it) {
            const uint32_t s = it % WGRAD_STAGES;
            if (!mbar_wait(&full[s], (it / WGRAD_STAGES) & 1u, a.error, 16u)) break;
            tc_fence_after();
            const uint32_t sa = smem_u32(base + s * stage_bytes), sb = sa + a_region;
#pragma unroll
            for (uint32_t k = 0; k < 8u; ++k)
                mma_bf16(tmem, smem_desc(sa + k * 32u * a.c, region, 16u * a.c, la), smem_desc(sb + k * 32u * a.n, 256u * a.n, 16u * a.n, lb),
                         idesc, (it | k) != 0u ? 1u : 0u);
            mma_commit(&empty[s]);
        }
        mma_commit(&done);
    }
    const bool ok = mbar_wait(&done, 0u, a.error, 32u);
    __syncwarp();
    tc_fence_after();
    if (ok) {
        const uint32_t m = warp * 32u + lane;
        const uint32_t tap = g * T + m / a.c, ci = m % a.c;
        for (uint32_t c0 = 0; c0 < a.n; c0 += 16u) {
            float acc[16];
            tmem_ld16(tmem + ((warp * 32u) << 16) + c0, acc);
            if (tap < 27u) {
                float* dst = a.partial + ((uint64_t(chunk) * 27u + tap) * a.n + c0) * a.c + ci;
#pragma unroll
                for (int j = 0; j < 16; ++j) dst[uint64_t(j) * a.c] = niter ? acc[j] : 0.0f;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// out[i] = sum over chunks of partial[chunk][i], in chunk order.
__global__ void k_reduce_chunks(const float* __restrict__ partial, float* __restrict__ out, uint32_t chunks, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s = s + partial[uint64_t(c) * count + i];
    out[i] = s;
}

// Weight gradient of one K-block: out[(tap n + co) cin + off + cl] = sum over chunks of
// partial[chunk][tap][co][cl], in chunk order.
__global__ void k_reduce_wgrad(const float* __restrict__ partial, float* __restrict__ out, uint32_t chunks, uint32_t n, uint32_t cb,
                               uint32_t cin, uint32_t off) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t count = 27u * n * cb;
    if (i >= count) return;
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s = s + partial[uint64_t(c) * count + i];
    const uint32_t cl = i % cb, row = i / cb;
    out[row * cin + off + cl] = s;
}

// Bias gradient partials: chunk c sums channel j over its voxel range (thread j + n * q takes voxels
// q, q + 256 / n, ...; the per-thread sums are added in thread order).
__global__ void k_bias_partial(const bf16* __restrict__ g, uint32_t n, uint64_t voxels, uint64_t per_chunk, float* __restrict__ partial) {
    __shared__ float s_sum[256];
    const uint32_t q = threadIdx.x / n, j = threadIdx.x % n, lanes = 256u / n;
    const uint64_t v0 = uint64_t(blockIdx.x) * per_chunk;
    const uint64_t v1 = min(voxels, v0 + per_chunk);
    float s = 0.0f;
    if (q < lanes)
        for (uint64_t v = v0 + q; v < v1; v += lanes) s = s + bf(g[v * n + j]);
    s_sum[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < n) {
        float t = 0.0f;
        for (uint32_t k = 0; k < lanes; ++k) t = t + s_sum[k * n + threadIdx.x];
        partial[uint64_t(blockIdx.x) * n + threadIdx.x] = t;
    }
}

// ---- pooling and upsampling (8 channels per thread) ----------------------------------------------------
struct V8 {
    float f[8];
};
__device__ __forceinline__ V8 ld8(const bf16* p) {
    const uint4 w = *reinterpret_cast<const uint4*>(p);
    const bf16* b = reinterpret_cast<const bf16*>(&w);
    V8 v;
#pragma unroll
    for (int j = 0; j < 8; ++j) v.f[j] = bf(b[j]);
    return v;
}
__device__ __forceinline__ void st8(bf16* p, const V8& v) {
    uint4 w;
    bf16* b = reinterpret_cast<bf16*>(&w);
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = __float2bfloat16_rn(v.f[j]);
    *reinterpret_cast<uint4*>(p) = w;
}
__device__ __forceinline__ void mask8(V8& v, const bf16* m) {
    const V8 mv = ld8(m);
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (!(mv.f[j] > 0.0f)) v.f[j] = 0.0f;
}
// Linear voxel of the fine child o (x fastest) of coarse voxel (b, z, y, x).
__device__ __forceinline__ uint64_t child_of(const Vol& f, uint32_t b, uint32_t z, uint32_t y, uint32_t x, int o) {
    return ((uint64_t(b) * f.D + 2u * z + uint32_t((o >> 2) & 1)) * f.H + 2u * y + uint32_t((o >> 1) & 1)) * f.W + 2u * x + uint32_t(o & 1);
}
__device__ __forceinline__ bool coarse_coord(const Vol& f, uint64_t i, uint32_t& b, uint32_t& z, uint32_t& y, uint32_t& x) {
    const uint32_t W = f.W / 2u, H = f.H / 2u, D = f.D / 2u;
    x = uint32_t(i % W);
    i /= W;
    y = uint32_t(i % H);
    i /= H;
    z = uint32_t(i % D);
    b = uint32_t(i / D);
    return b < f.B;
}
__global__ void k_pool(const bf16* __restrict__ in, bf16* __restrict__ out, Vol f, uint32_t c) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t g8 = c / 8u;
    uint32_t b, z, y, x;
    if (!coarse_coord(f, t / g8, b, z, y, x)) return;
    const uint32_t cg = uint32_t(t % g8) * 8u;
    V8 s;
#pragma unroll
    for (int j = 0; j < 8; ++j) s.f[j] = 0.0f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const V8 v = ld8(in + child_of(f, b, z, y, x, o) * c + cg);
#pragma unroll
        for (int j = 0; j < 8; ++j) s.f[j] = s.f[j] + v.f[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) s.f[j] = s.f[j] * 0.125f;
    st8(out + (t / g8) * c + cg, s);
}
__global__ void k_pool_bwd(const bf16* __restrict__ gout, bf16* __restrict__ gin, Vol f, uint32_t c, uint32_t accumulate,
                           const bf16* __restrict__ mask) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t g8 = c / 8u;
    uint32_t b, z, y, x;
    if (!coarse_coord(f, t / g8, b, z, y, x)) return;
    const uint32_t cg = uint32_t(t % g8) * 8u;
    const V8 gv = ld8(gout + (t / g8) * c + cg);
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const uint64_t e = child_of(f, b, z, y, x, o) * c + cg;
        V8 v;
#pragma unroll
        for (int j = 0; j < 8; ++j) v.f[j] = gv.f[j] * 0.125f;
        if (accumulate) {
            const V8 old = ld8(gin + e);
#pragma unroll
            for (int j = 0; j < 8; ++j) v.f[j] = old.f[j] + v.f[j];
        }
        if (mask) mask8(v, mask + e);
        st8(gin + e, v);
    }
}
__global__ void k_upsample(const bf16* __restrict__ in, bf16* __restrict__ out, Vol f, uint32_t c) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t g8 = c / 8u;
    uint32_t b, z, y, x;
    if (!coarse_coord(f, t / g8, b, z, y, x)) return;
    const uint32_t cg = uint32_t(t % g8) * 8u;
    const uint4 w = *reinterpret_cast<const uint4*>(in + (t / g8) * c + cg);
#pragma unroll
    for (int o = 0; o < 8; ++o) *reinterpret_cast<uint4*>(out + child_of(f, b, z, y, x, o) * c + cg) = w;
}
__global__ void k_upsample_bwd(const bf16* __restrict__ gout, bf16* __restrict__ gin, Vol f, uint32_t c, const bf16* __restrict__ mask) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t g8 = c / 8u;
    uint32_t b, z, y, x;
    if (!coarse_coord(f, t / g8, b, z, y, x)) return;
    const uint32_t cg = uint32_t(t % g8) * 8u;
    V8 s;
#pragma unroll
    for (int j = 0; j < 8; ++j) s.f[j] = 0.0f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const V8 v = ld8(gout + child_of(f, b, z, y, x, o) * c + cg);
#pragma unroll
        for (int j = 0; j < 8; ++j) s.f[j] = s.f[j] + v.f[j];
    }
    const uint64_t e = (t / g8) * c + cg;
    if (mask) mask8(s, mask + e);
    st8(gin + e, s);
}

// ---- head (16 -> 1), loss and its gradients ------------------------------------------------------------
// head_w = [w0..w15, bias]. Chunk partials per CTA: [17 head gradients, loss]; the CTA's 256 threads
// take voxels v0 + t, v0 + t + 256, ... and their sums are folded in thread order.
constexpr uint32_t HEAD_THREADS = 256;
__global__ void __launch_bounds__(HEAD_THREADS) k_head(const bf16* __restrict__ d0, const bf16* __restrict__ input,
                                                       const float* __restrict__ hw, float* __restrict__ out, const float* __restrict__ target,
                                                       const uint32_t* __restrict__ nfluid, bf16* __restrict__ g_d0, float* __restrict__ partial,
                                                       uint64_t voxels, uint64_t per_chunk) {
    __shared__ float s_part[HEAD_THREADS][18];
    float w[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) w[j] = hw[j];
    const float bias = hw[16];
    const float inv_n = target ? 1.0f / float(max(nfluid[0], 1u)) : 0.0f;
    float acc[18];
#pragma unroll
    for (int j = 0; j < 18; ++j) acc[j] = 0.0f;
    const uint64_t v0 = uint64_t(blockIdx.x) * per_chunk;
    const uint64_t v1 = min(voxels, v0 + per_chunk);
    for (uint64_t v = v0 + threadIdx.x; v < v1; v += HEAD_THREADS) {
        const V8 a = ld8(d0 + v * 16u), b = ld8(d0 + v * 16u + 8u);
        float h[16];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            h[j] = a.f[j];
            h[8 + j] = b.f[j];
        }
        float y = 0.0f;
#pragma unroll
        for (int j = 0; j < 16; ++j) y = y + w[j] * h[j];
        y = y + bias;
        if (out) out[v] = y;
        if (!target) continue;
        const bool fluid = bf(input[v * IN_CHANNELS + 1u]) > 0.5f;
        const float diff = fluid ? y - target[v] : 0.0f;
        const float dy = 2.0f * diff * inv_n;
        V8 ga, gb;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            ga.f[j] = h[j] > 0.0f ? dy * w[j] : 0.0f;
            gb.f[j] = h[8 + j] > 0.0f ? dy * w[8 + j] : 0.0f;
        }
        st8(g_d0 + v * 16u, ga);
        st8(g_d0 + v * 16u + 8u, gb);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[j] = acc[j] + dy * h[j];
        acc[16] = acc[16] + dy;
        acc[17] = acc[17] + diff * diff * inv_n;
    }
    if (!target) return;
#pragma unroll
    for (int j = 0; j < 18; ++j) s_part[threadIdx.x][j] = acc[j];
    __syncthreads();
    if (threadIdx.x < 18) {
        float s = 0.0f;
        for (uint32_t t = 0; t < HEAD_THREADS; ++t) s = s + s_part[t][threadIdx.x];
        partial[uint64_t(blockIdx.x) * 18u + threadIdx.x] = s;
    }
}

// ---- Adam ----------------------------------------------------------------------------------------------
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, uint64_t count,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// ---- BF16 weight copies ----------------------------------------------------------------------------------
struct ConvWeightArgs {
    const float* w;
    uint32_t n, cin, nblocks;
    uint32_t cb[2];
    bf16* fwd[2];
    bf16* dgrad;
};
__global__ void k_conv_weights(ConvWeightArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = 27u * a.n * a.cin;
    if (i >= total) return;
    const uint32_t ci = i % a.cin, co = (i / a.cin) % a.n, tap = i / (a.cin * a.n);
    const bf16 v = __float2bfloat16_rn(a.w[i]);
    const uint32_t blk = (a.nblocks > 1u && ci >= a.cb[0]) ? 1u : 0u;
    const uint32_t cl = blk ? ci - a.cb[0] : ci;
    a.fwd[blk][(tap * a.n + co) * a.cb[blk] + cl] = v;
    a.dgrad[((26u - tap) * a.cin + ci) * a.n + co] = v;
}

// ---- exchange with the simulation's brick pool -------------------------------------------------------
__device__ __forceinline__ uint32_t float_order_key(float f) { return __float_as_uint(fabsf(f)); }
// Pass 1: max |divergence| over fluid cells and the fluid count of the dense grid.
__global__ void k_pack_scan(Dev d, const float* __restrict__ div, uint32_t* __restrict__ meta, uint32_t slot) {
    const uint32_t W = uint32_t(d.grid.x), H = uint32_t(d.grid.y), D = uint32_t(d.grid.z);
    const uint64_t n = uint64_t(W) * H * D;
    uint32_t kmax = 0u, cnt = 0u;
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += uint64_t(gridDim.x) * blockDim.x) {
        const int3 c = make_int3(int(v % W), int((v / W) % H), int(v / (uint64_t(W) * H)));
        const uint32_t ci = cell_index(d, c);
        if (is_null_cell(ci) || type_of(d.cell_type[ci]) != CELL_FLUID) continue;
        kmax = max(kmax, float_order_key(div[ci]));
        ++cnt;
    }
    kmax = __reduce_max_sync(0xFFFFFFFFu, kmax);
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    if ((threadIdx.x & 31u) == 0u) {
        if (kmax) atomicMax(meta + 2u * slot, kmax);
        if (cnt) atomicAdd(meta + 2u * slot + 1u, cnt);
    }
}
__device__ __forceinline__ float slot_scale(const uint32_t* meta, uint32_t slot) {
    const float s = __uint_as_float(meta[2u * slot]);
    return s > 0.0f ? s : 1.0f;
}
// Pass 2: the dense input (and target) of the slot.
__global__ void k_pack(Dev d, const float* __restrict__ div, const float* __restrict__ pressure, bf16* __restrict__ input,
                       float* __restrict__ target, const uint32_t* __restrict__ meta, uint32_t slot) {
    const uint32_t W = uint32_t(d.grid.x), H = uint32_t(d.grid.y), D = uint32_t(d.grid.z);
    const uint64_t n = uint64_t(W) * H * D;
    const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float scale = slot_scale(meta, slot);
    const int3 c = make_int3(int(v % W), int((v / W) % H), int(v / (uint64_t(W) * H)));
    const uint32_t ci = cell_index(d, c);
    const bool border = c.x == 0 || c.y == 0 || c.z == 0 || c.x == d.grid.x - 1 || c.y == d.grid.y - 1 || c.z == d.grid.z - 1;
    uint32_t type = border ? CELL_SOLID : CELL_AIR;
    float dv = 0.0f, pv = 0.0f;
    if (!is_null_cell(ci)) {
        type = type_of(d.cell_type[ci]);
        if (type == CELL_FLUID) {
            dv = div[ci] / scale;
            if (pressure) pv = pressure[ci] / scale;
        }
    }
    uint4 w[2] = {make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u)};
    bf16* wb = reinterpret_cast<bf16*>(w);
    wb[0] = __float2bfloat16_rn(dv);
    wb[1] = __float2bfloat16_rn(type == CELL_FLUID ? 1.0f : 0.0f);
    wb[2] = __float2bfloat16_rn(type == CELL_SOLID ? 1.0f : 0.0f);
    uint4* dst = reinterpret_cast<uint4*>(input + (uint64_t(slot) * n + v) * IN_CHANNELS);
    dst[0] = w[0];
    dst[1] = w[1];
    if (target) target[uint64_t(slot) * n + v] = pv;
}
// Energy-optimal scale of the guess g (the network's output on the dense grid): with x0 = beta g, beta =
// (g . b) / (g . A g) minimises the A-norm error ||x0 - x||_A over the line through g, so the solve never
// starts worse (in that norm) than from zero. A and b are level 0 of the solve: (A g)_i = (diag_i +
// DiagEpsilon) g_i - sum of g over the fluid neighbours, b_i = -div_i, over the fluid cells. Chunk c of
// the dense voxels gives partial[2c] = sum g.b, partial[2c + 1] = sum g.Ag (FP64, threads folded in order).
constexpr uint32_t ENERGY_THREADS = 256;
__global__ void __launch_bounds__(ENERGY_THREADS) k_energy_partial(Dev d, const float* __restrict__ guess, const bf16* __restrict__ input,
                                                                   const float* __restrict__ div, double* __restrict__ partial,
                                                                   uint64_t per_chunk) {
    __shared__ double s_gb[ENERGY_THREADS], s_gag[ENERGY_THREADS];
    const uint32_t W = uint32_t(d.grid.x), H = uint32_t(d.grid.y), D = uint32_t(d.grid.z);
    const uint64_t n = uint64_t(W) * H * D;
    const uint64_t v0 = uint64_t(blockIdx.x) * per_chunk;
    const uint64_t v1 = min(n, v0 + per_chunk);
    double gb = 0.0, gag = 0.0;
    auto fluid = [&](uint64_t v) { return bf(input[v * IN_CHANNELS + 1u]) > 0.5f; };
    for (uint64_t v = v0 + threadIdx.x; v < v1; v += ENERGY_THREADS) {
        if (!fluid(v)) continue;
        const int3 c = make_int3(int(v % W), int((v / W) % H), int(v / (uint64_t(W) * H)));
        const uint32_t ci = cell_index(d, c);
        const float g = guess[v];
        float nb = 0.0f;
        const uint64_t sx = 1u, sy = W, sz = uint64_t(W) * H;
        if (c.x > 0 && fluid(v - sx)) nb = nb + guess[v - sx];
        if (c.x + 1 < d.grid.x && fluid(v + sx)) nb = nb + guess[v + sx];
        if (c.y > 0 && fluid(v - sy)) nb = nb + guess[v - sy];
        if (c.y + 1 < d.grid.y && fluid(v + sy)) nb = nb + guess[v + sy];
        if (c.z > 0 && fluid(v - sz)) nb = nb + guess[v - sz];
        if (c.z + 1 < d.grid.z && fluid(v + sz)) nb = nb + guess[v + sz];
        const float ag = (d.cell_diag[ci] + DIAG_EPSILON) * g - nb;
        gb += double(g) * double(-div[ci]);
        gag += double(g) * double(ag);
    }
    s_gb[threadIdx.x] = gb;
    s_gag[threadIdx.x] = gag;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (uint32_t t = 0; t < ENERGY_THREADS; ++t) {
            a += s_gb[t];
            b += s_gag[t];
        }
        partial[2u * blockIdx.x] = a;
        partial[2u * blockIdx.x + 1u] = b;
    }
}
__global__ void k_energy_finish(const double* __restrict__ partial, uint32_t chunks, float* __restrict__ beta) {
    double a = 0.0, b = 0.0;
    for (uint32_t c = 0; c < chunks; ++c) {
        a += partial[2u * c];
        b += partial[2u * c + 1u];
    }
    *beta = b > 0.0 ? float(a / b) : 0.0f;
}
__global__ void k_scatter_guess(Dev d, const float* __restrict__ guess, const float* __restrict__ beta, float* __restrict__ pressure) {
    const uint32_t W = uint32_t(d.grid.x), H = uint32_t(d.grid.y), D = uint32_t(d.grid.z);
    const uint64_t n = uint64_t(W) * H * D;
    const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int3 c = make_int3(int(v % W), int((v / W) % H), int(v / (uint64_t(W) * H)));
    const uint32_t ci = cell_index(d, c);
    if (is_null_cell(ci) || type_of(d.cell_type[ci]) != CELL_FLUID) return;
    pressure[ci] = guess[v] * beta[0];
}

uint32_t blocks_for(uint64_t n, uint32_t threads) { return uint32_t((n + threads - 1u) / threads); }
uint32_t tmem_cols_host(uint32_t n) { return n <= 32u ? 32u : (n <= 64u ? 64u : (n <= 128u ? 128u : 256u)); }

}  // namespace

static size_t wgrad_smem_bytes(uint32_t n) {
    const size_t a_region = 128u * 128u * 2u;  // T taps x 128 rows x c channels, T c = 128
    const size_t b_region = (256u * size_t(n) + 1023u) / 1024u * 1024u;
    return WGRAD_STAGES * (a_region + b_region) + 1024u;
}

// The halo-box form applies when every K-block has 16 or 32 channels, n <= 64, the weights of all taps fit
// in 64 KB, the volume tiles into 8 x 16 x 1 boxes and two halo buffers still leave three CTAs per SM (the
// configurations where it measured faster than the streamed-tap kernel: 1.6-2x on the 16-channel 128^3 layers;
// at one CTA per SM it was slower, and a one-buffer form at two CTAs per SM gained nothing). SLOSH_CONV_HALO=0
// turns it off.
static int conv_halo_mode() {
    static const int v = [] {
        const char* e = std::getenv("SLOSH_CONV_HALO");
        return e ? std::atoi(e) : 1;
    }();
    return v;
}
static int launch_conv_halo(const ConvArgs& in, cudaStream_t s) {
    const int mode = conv_halo_mode();
    if (mode == 0 || !in.in_ptr[0] || !in.w_ptr[0] || in.n > 64u || in.n % 16u) return 0;
    uint32_t wbytes = 0, hbytes = 0;
    for (uint32_t k = 0; k < in.nblocks; ++k) {
        if ((in.cb[k] != 16u && in.cb[k] != 32u) || !in.in_ptr[k] || !in.w_ptr[k]) return 0;
        wbytes += 27u * in.cb[k] * in.n * 2u;
        hbytes += (in.cb[k] / 8u) * HALO_PLANE;
    }
    if (wbytes > 64u * 1024u || in.vol.W % 8u || in.vol.H % 16u) return 0;
    ConvArgs a = in;
    a.vol.bx = 8u;
    a.vol.by = 16u;
    a.vol.bz = 1u;
    if (!halo_maps(a)) return 0;
    const uint32_t nbuf = 2u;
    const size_t smem = size_t((wbytes + 1023u) & ~1023u) + 2u * size_t(hbytes) + 1024u;
    if ((227u * 1024u) / (smem + 1024u) < 3u) return 0;
    static int num_sms = 0;
    if (!num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (num_sms <= 0) num_sms = 148;
        cudaFuncSetAttribute(k_conv3d_halo, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    }
    uint32_t per_sm = uint32_t((227u * 1024u) / (smem + 1024u));
    const uint32_t by_tmem = 512u / (2u * tmem_cols_host(a.n));
    if (per_sm > by_tmem) per_sm = by_tmem;
    if (per_sm > 2048u / CONV_THREADS) per_sm = 2048u / CONV_THREADS;
    if (per_sm < 1u) per_sm = 1u;
    const uint32_t tiles = a.vol.tiles();
    uint32_t grid = uint32_t(num_sms) * per_sm;
    if (grid > tiles) grid = tiles;
    k_conv3d_halo<<<grid, CONV_THREADS, smem, s>>>(a, wbytes, hbytes, nbuf);
    return 1;
}

int launch_conv(const ConvArgs& a, cudaStream_t s) {
    if (launch_conv_halo(a, s)) return 1;
    uint32_t cbmax = a.cb[0];
    if (a.nblocks > 1u) cbmax = a.cb[0] > a.cb[1] ? a.cb[0] : a.cb[1];
    const uint32_t a_region = 256u * cbmax;
    const uint32_t b_region = (a.n * cbmax * 2u + 1023u) / 1024u * 1024u;
    const uint32_t stage = a_region + b_region;
    // The loads are L2-latency bound, so what counts is the number of stages in flight per SM: 3-8
    // stages in about 48 KB per CTA, and as many persistent CTAs per SM as shared memory (227 KB),
    // TMEM (512 columns, two accumulators per CTA) and threads (2048) allow.
    uint32_t stages = (48u * 1024u) / stage;
    stages = stages < 3u ? 3u : (stages > uint32_t(CONV_MAX_STAGES) ? uint32_t(CONV_MAX_STAGES) : stages);
    const size_t smem = size_t(stages) * stage + 1024u;
    static int num_sms = 0;
    if (!num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (num_sms <= 0) num_sms = 148;
        cudaFuncSetAttribute(k_conv3d, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    }
    const uint32_t tiles = a.vol.tiles();
    uint32_t per_sm = uint32_t((227u * 1024u) / (smem + 1024u));
    const uint32_t by_tmem = 512u / (2u * tmem_cols_host(a.n));
    if (per_sm > by_tmem) per_sm = by_tmem;
    if (per_sm > 2048u / CONV_THREADS) per_sm = 2048u / CONV_THREADS;
    if (per_sm < 1u) per_sm = 1u;
    uint32_t grid = uint32_t(num_sms) * per_sm;
    if (grid > tiles) grid = tiles;
    k_conv3d<<<grid, CONV_THREADS, smem, s>>>(a, stage, a_region, stages);
    return 1;
}
int launch_wgrad(const WgradArgs& a, uint32_t chunks, cudaStream_t s) {
    const uint32_t a_region = 128u * 128u * 2u;
    const uint32_t b_region = (256u * a.n + 1023u) / 1024u * 1024u;
    const size_t smem = wgrad_smem_bytes(a.n);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        configured = true;
    }
    const uint32_t T = 128u / a.c;
    k_wgrad<<<dim3(chunks, (27u + T - 1u) / T), 128, smem, s>>>(a, a_region + b_region, a_region);
    return 1;
}
int launch_reduce_chunks(const float* partial, float* out, uint32_t chunks, uint32_t count, cudaStream_t s) {
    k_reduce_chunks<<<blocks_for(count, 256), 256, 0, s>>>(partial, out, chunks, count);
    return 1;
}
int launch_reduce_wgrad(const float* partial, float* out, uint32_t chunks, uint32_t n, uint32_t cb, uint32_t cin, uint32_t off,
                        cudaStream_t s) {
    k_reduce_wgrad<<<blocks_for(27ull * n * cb, 256), 256, 0, s>>>(partial, out, chunks, n, cb, cin, off);
    return 1;
}
int launch_bias_grad(const bf16* g, uint32_t n, uint64_t voxels, float* partial, uint32_t chunks, float* out, cudaStream_t s) {
    const uint64_t per = (voxels + chunks - 1u) / chunks;
    k_bias_partial<<<chunks, 256, 0, s>>>(g, n, voxels, per, partial);
    k_reduce_chunks<<<1, 256, 0, s>>>(partial, out, chunks, n);
    return 2;
}
int launch_pool(const bf16* in, bf16* out, Vol f, uint32_t c, cudaStream_t s) {
    const uint64_t n = f.voxels() / 8u * (c / 8u);
    k_pool<<<blocks_for(n, 256), 256, 0, s>>>(in, out, f, c);
    return 1;
}
int launch_pool_bwd(const bf16* gout, bf16* gin, Vol f, uint32_t c, uint32_t accumulate, const bf16* mask, cudaStream_t s) {
    const uint64_t n = f.voxels() / 8u * (c / 8u);
    k_pool_bwd<<<blocks_for(n, 256), 256, 0, s>>>(gout, gin, f, c, accumulate, mask);
    return 1;
}
int launch_upsample(const bf16* in, bf16* out, Vol f, uint32_t c, cudaStream_t s) {
    const uint64_t n = f.voxels() / 8u * (c / 8u);
    k_upsample<<<blocks_for(n, 256), 256, 0, s>>>(in, out, f, c);
    return 1;
}
int launch_upsample_bwd(const bf16* gout, bf16* gin, Vol f, uint32_t c, const bf16* mask, cudaStream_t s) {
    const uint64_t n = f.voxels() / 8u * (c / 8u);
    k_upsample_bwd<<<blocks_for(n, 256), 256, 0, s>>>(gout, gin, f, c, mask);
    return 1;
}
int launch_head(const bf16* d0, const bf16* input, const float* head_w, float* out, const float* target, const uint32_t* nfluid,
                bf16* g_d0, float* partial, uint32_t chunks, float* head_grad, uint64_t voxels, cudaStream_t s) {
    const uint64_t per = (voxels + chunks - 1u) / chunks;
    k_head<<<chunks, HEAD_THREADS, 0, s>>>(d0, input, head_w, out, target, nfluid, g_d0, partial, voxels, per);
    if (!target) return 1;
    k_reduce_chunks<<<1, 32, 0, s>>>(partial, head_grad, chunks, 18u);  // head_grad[0..16] gradients, [17] the loss
    return 2;
}
int launch_adam(float* p, const float* g, float* m, float* v, uint64_t count, float lr, float b1, float b2, float eps, float c1,
                float c2, cudaStream_t s) {
    k_adam<<<blocks_for(count, 256), 256, 0, s>>>(p, g, m, v, count, lr, b1, b2, eps, c1, c2);
    return 1;
}
int launch_conv_weights(const float* w, uint32_t n, uint32_t cin, const uint32_t* cb, uint32_t nblocks, bf16* const* fwd, bf16* dgrad,
                        cudaStream_t s) {
    ConvWeightArgs a;
    a.w = w;
    a.n = n;
    a.cin = cin;
    a.nblocks = nblocks;
    a.cb[0] = cb[0];
    a.cb[1] = nblocks > 1u ? cb[1] : 0u;
    a.fwd[0] = fwd[0];
    a.fwd[1] = nblocks > 1u ? fwd[1] : nullptr;
    a.dgrad = dgrad;
    k_conv_weights<<<blocks_for(27ull * n * cin, 256), 256, 0, s>>>(a);
    return 1;
}
int launch_pack_input(const Dev& d, const float* divergence, const float* pressure, bf16* input, float* target, uint32_t* meta,
                      uint32_t slot, cudaStream_t s) {
    const uint64_t n = uint64_t(d.grid.x) * d.grid.y * d.grid.z;
    k_pack_scan<<<592, 256, 0, s>>>(d, divergence, meta, slot);
    k_pack<<<blocks_for(n, 256), 256, 0, s>>>(d, divergence, pressure, input, target, meta, slot);
    return 2;
}
int launch_scatter_guess(const Dev& d, const float* guess, const bf16* input, const float* divergence, double* partial, uint32_t chunks,
                         float* beta, float* pressure, cudaStream_t s) {
    const uint64_t n = uint64_t(d.grid.x) * d.grid.y * d.grid.z;
    k_energy_partial<<<chunks, ENERGY_THREADS, 0, s>>>(d, guess, input, divergence, partial, (n + chunks - 1u) / chunks);
    k_energy_finish<<<1, 1, 0, s>>>(partial, chunks, beta);
    k_scatter_guess<<<blocks_for(n, 256), 256, 0, s>>>(d, guess, beta, pressure);
    return 3;
}

}  // namespace unet
}  // namespace slosh
