// The learned warm start of the pressure solve: a 3-D convolutional U-Net (4 levels, 16/32/64/64
// channels, 3x3x3 kernels, BF16 weights and activations, FP32 accumulation) that maps the divergence
// and the fluid / solid masks to an initial pressure guess for MGPCG, trained on the GPU with the
// kernels below. Activations are dense NDHWC BF16 ([batch][z][y][x][channel]); channel counts are
// 16, 32 or 64 per tensor (a 128-channel convolution input is two tensors, a "K-block" each).
//
// Kernel forms (kernels_unet.cu):
//   k_conv3d   implicit-GEMM 3x3x3 convolution, stride 1, zero padding 1, persistent: a CTA takes
//              tiles of 128 output voxels x N channels in turn; per (tap, K-block) TMA loads the 128
//              shifted input rows and the tap's N x C weights into swizzled shared memory and one
//              thread issues tcgen05.mma (M = 128, K = 16) into one of two TMEM accumulators; four
//              epilogue warps add the bias, apply ReLU, split the channels over one or two output
//              tensors, optionally add to them and mask them (ReLU backward) while the next tile's
//              loads and MMAs run. With flipped, transposed weights it is also the data gradient.
//   k_conv3d_halo  the same convolution for the layers whose weights fit in shared memory (K-blocks of 16 or
//              32 channels): a tile is an 8 x 16 x 1 box of voxels, and one TMA load per 8-channel plane brings
//              its 10 x 18 x 3 halo box into shared memory in the no-swizzle core-matrix layout (16 bytes per
//              voxel and plane); each of the 27 taps is then just an operand descriptor whose start address is
//              shifted by the tap inside the halo box (8-row groups 160 bytes apart, planes one halo box apart).
//              The weights of all taps stay in shared memory for the CTA's lifetime.
//   k_wgrad    weight gradient dW[tap][n][c] = sum_v X[v + tap][c] dZ[v][n] as tcgen05.mma with both
//              operands MN-major: M = 128 rows are (tap, c) pairs of 128 / C taps, N = output
//              channels, K = 128 voxels per stage; per-chunk partials are summed in chunk order.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace slosh {
namespace unet {

typedef __nv_bfloat16 bf16;

constexpr int WGRAD_STAGES = 4;
constexpr uint32_t IN_CHANNELS = 16;  // divergence, fluid, solid, zero padding to the MMA's K of 16

// Dense volume geometry and its 128-voxel tiles: a tile is the box (bx, by, bz) at (x0, y0, z0) of
// one batch entry; bx = min(W, 128), by = min(H, 128 / bx), bz = 128 / (bx * by), so the tile's rows
// are 128 consecutive voxels in (z, y, x) order.
struct Vol {
    uint32_t W, H, D, B;
    uint32_t bx, by, bz;
    __host__ __device__ uint64_t voxels() const { return uint64_t(W) * H * D * B; }
    __host__ __device__ uint32_t tiles() const { return uint32_t(voxels() / 128u); }
};

struct alignas(64) ConvArgs {
    CUtensorMap act[2];  // K-block inputs: 5-D (C, W, H, D, B), box (C, bx, by, bz, 1)
    CUtensorMap wgt[2];  // K-block weights: 2-D (C, 27 N), box (C, N); rows tap * N + n
    uint32_t cb[2];      // channels of each K-block (16, 32 or 64)
    uint32_t nblocks;
    uint32_t n;          // output channels (multiple of 16, <= 128)
    Vol vol;
    const float* bias;   // [n] or null
    uint32_t relu;
    bf16* out[2];        // output channels [0, oc[0]) -> out[0], [oc[0], n) -> out[1]
    uint32_t oc[2];
    const bf16* mask[2]; // multiply by (mask > 0) after the optional add
    uint32_t accumulate; // add to the outputs' current values
    uint32_t* error;
    // for the halo-box form (k_conv3d_halo): the K-block inputs and weights as plain pointers; the
    // launcher builds the halo tensor maps itself
    const bf16* in_ptr[2];   // [B][D][H][W][cb]
    const bf16* w_ptr[2];    // [27][n][cb]
    CUtensorMap halo[2];     // 5-D (C, W, H, D, B), box (8, 10, 18, 3, 1), no swizzle (set by launch_conv)
};

struct alignas(64) WgradArgs {
    CUtensorMap act;     // X: box (c, bx, by, bz, 1)
    CUtensorMap grad;    // dZ: box (n, bx, by, bz, 1)
    uint32_t c, n;
    Vol vol;
    uint32_t tiles_per_chunk;
    float* partial;      // [chunks][27][n][c]
    uint32_t* error;
};

int launch_conv(const ConvArgs& a, cudaStream_t s);
// Halo tensor maps of a convolution's K-block inputs (box 8 channels x 10 x 18 x 3, no swizzle), for
// k_conv3d_halo; false if a map is rejected.
bool halo_maps(ConvArgs& a);
int launch_wgrad(const WgradArgs& a, uint32_t chunks, cudaStream_t s);
int launch_reduce_chunks(const float* partial, float* out, uint32_t chunks, uint32_t count, cudaStream_t s);
int launch_reduce_wgrad(const float* partial, float* out, uint32_t chunks, uint32_t n, uint32_t cb, uint32_t cin, uint32_t off,
                        cudaStream_t s);
int launch_bias_grad(const bf16* g, uint32_t n, uint64_t voxels, float* partial, uint32_t chunks, float* out, cudaStream_t s);
int launch_pool(const bf16* in, bf16* out, Vol fine, uint32_t c, cudaStream_t s);
int launch_pool_bwd(const bf16* gout, bf16* gin, Vol fine, uint32_t c, uint32_t accumulate, const bf16* mask, cudaStream_t s);
int launch_upsample(const bf16* in, bf16* out, Vol fine, uint32_t c, cudaStream_t s);
int launch_upsample_bwd(const bf16* gout, bf16* gin, Vol fine, uint32_t c, const bf16* mask, cudaStream_t s);
// 1x1 head (16 -> 1) on the last decoder tensor; with a target also the masked MSE over fluid voxels,
// the head's gradients and the gradient of the decoder tensor (ReLU-masked): head_grad[0..16] =
// d loss / d (w0..w15, bias), head_grad[17] = the loss.
int launch_head(const bf16* d0, const bf16* input, const float* head_w, float* out, const float* target, const uint32_t* nfluid,
                bf16* g_d0, float* partial, uint32_t chunks, float* head_grad, uint64_t voxels, cudaStream_t s);
int launch_adam(float* p, const float* g, float* m, float* v, uint64_t count, float lr, float b1, float b2, float eps, float c1,
                float c2, cudaStream_t s);
// BF16 weight copies of one convolution from its FP32 master [27][n][cin]: the forward K-blocks
// [27][n][cb] and the data-gradient weights [27][cin][n] (tap mirrored).
int launch_conv_weights(const float* w, uint32_t n, uint32_t cin, const uint32_t* cb, uint32_t nblocks, bf16* const* fwd, bf16* dgrad,
                        cudaStream_t s);

// Dense network input of batch entry `slot` from a simulation state: channel 0 = divergence / scale,
// 1 = fluid, 2 = solid; scale = max |divergence| over the fluid cells (1 when there is none). With
// target != null also the dense target pressure / scale (0 outside the fluid). meta[2 slot] = scale
// bits, meta[2 slot + 1] = fluid voxel count (accumulated; the caller clears it).
int launch_pack_input(const Dev& d, const float* divergence, const float* pressure, bf16* input, float* target, uint32_t* meta,
                      uint32_t slot, cudaStream_t s);
// Initial pressure from slot 0's guess: pressure[fluid cells] = beta * guess[v], beta = (g . b) / (g . A g)
// of the solve's level-0 system (energy-optimal scale, deterministic FP64 sums over `chunks` chunks).
int launch_scatter_guess(const Dev& d, const float* guess, const bf16* input, const float* divergence, double* partial, uint32_t chunks,
                         float* beta, float* pressure, cudaStream_t s);

}  // namespace unet
}  // namespace slosh
