// Host side of the learned warm start: the U-Net's tensors, tensor maps, parameters and the forward /
// backward / Adam schedule on one stream, plus its C ABI (include/slosh_cuda.h) and the hook the
// simulation calls before a pressure solve when warm_start = LEARNED.
//
// Network (grid W x H x D, each a multiple of 8; level l has dimensions >> l):
//   encoder  l0: in(16) -> e0a(16) -> e0(16)     pool -> p1(16)
//            l1: p1 -> e1a(32) -> e1(32)          pool -> p2(32)
//            l2: p2 -> e2a(64) -> e2(64)          pool -> p3(64)
//            l3: p3 -> e3a(64) -> e3(64)
//   decoder  l2: [up(e3), e2] -> d2a(64) -> d2(64)
//            l1: [up(d2), e1] -> d1a(32) -> d1(32)
//            l0: [up(d1), e0] -> d0a(16) -> d0(16)
//   head     guess = w . d0 + b (1x1, FP32)
// Every convolution is 3x3x3 with bias and ReLU; pooling is the mean of 2^3 children, upsampling
// repeats the parent. Loss: mean over fluid voxels of (guess - pressure / scale)^2.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/slosh_cuda.h"
#include "unet.h"

namespace slosh {
namespace unet {

void* sim_ctx_dev(void* ctx, Dev* out, float** divergence, float** pressure, cudaStream_t* stream);  // driver.cu

struct CudaFail {
    cudaError_t code;
    const char* what;
};
#define UCK(x)                                                          \
    do {                                                                \
        cudaError_t e_ = (x);                                           \
        if (e_ != cudaSuccess) throw slosh::unet::CudaFail{e_, #x};     \
    } while (0)

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        UCK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
CUtensorMapSwizzle swizzle_for(uint32_t row_bytes) {
    return row_bytes == 128u ? CU_TENSOR_MAP_SWIZZLE_128B : (row_bytes == 64u ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}
// 5-D map of a dense NDHWC BF16 tensor with C channels; box = one 128-voxel tile.
CUtensorMap act_map(const bf16* p, uint32_t C, const Vol& v) {
    CUtensorMap m;
    const cuuint64_t dims[5] = {C, v.W, v.H, v.D, v.B};
    const cuuint64_t strides[4] = {uint64_t(C) * 2u, uint64_t(C) * 2u * v.W, uint64_t(C) * 2u * v.W * v.H,
                                   uint64_t(C) * 2u * v.W * v.H * v.D};
    const cuuint32_t box[5] = {C, v.bx, v.by, v.bz, 1u};
    const cuuint32_t es[5] = {1u, 1u, 1u, 1u, 1u};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(p), dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(2u * C), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("tensor map (activations) rejected");
    return m;
}
// 2-D map of a weight tensor [27 rows_per_tap][C]; box = one tap's rows.
CUtensorMap wgt_map(const bf16* p, uint32_t C, uint32_t rows_per_tap) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {C, 27ull * rows_per_tap};
    const cuuint64_t strides[1] = {uint64_t(C) * 2u};
    const cuuint32_t box[2] = {C, rows_per_tap};
    const cuuint32_t es[2] = {1u, 1u};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(p), dims, strides, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(2u * C), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("tensor map (weights) rejected");
    return m;
}
// 5-D map of a dense NDHWC BF16 tensor with C channels whose box is the 10 x 18 x 3 halo of an 8 x 16 x 1
// tile, 8 channels at a time, unswizzled (16 bytes per voxel in shared memory).
bool halo_map(CUtensorMap* m, const bf16* p, uint32_t C, const Vol& v) {
    const cuuint64_t dims[5] = {C, v.W, v.H, v.D, v.B};
    const cuuint64_t strides[4] = {uint64_t(C) * 2u, uint64_t(C) * 2u * v.W, uint64_t(C) * 2u * v.W * v.H,
                                   uint64_t(C) * 2u * v.W * v.H * v.D};
    const cuuint32_t box[5] = {8u, 10u, 18u, 3u, 1u};
    const cuuint32_t es[5] = {1u, 1u, 1u, 1u, 1u};
    return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(p), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
Vol make_vol(uint32_t W, uint32_t H, uint32_t D, uint32_t B) {
    Vol v{W, H, D, B, 0, 0, 0};
    v.bx = W < 128u ? W : 128u;
    v.by = H < 128u / v.bx ? H : 128u / v.bx;
    v.bz = 128u / (v.bx * v.by);
    if (v.bx * v.by * v.bz != 128u || W % v.bx || H % v.by || D % v.bz || v.bz > D)
        throw std::invalid_argument("volume cannot be tiled by 128-voxel boxes");
    return v;
}
template <class T>
T* dmalloc(size_t n, bool zero = true) {
    void* p = nullptr;
    UCK(cudaMalloc(&p, n * sizeof(T) + 16));
    if (zero) UCK(cudaMemset(p, 0, n * sizeof(T) + 16));
    return static_cast<T*>(p);
}

struct Tensor {
    uint32_t c = 0, level = 0;
    bf16* act = nullptr;
    bf16* grad = nullptr;
    CUtensorMap map_act, map_grad;
    bool relu = false;  // produced by a ReLU convolution (its gradient is masked by act > 0)
};
struct Conv {
    int in[2] = {-1, -1};
    uint32_t nblocks = 1, cb[2] = {0, 0}, cin = 0, n = 0;
    int out = -1;
    uint64_t w_off = 0, b_off = 0;  // in the parameter vector
    bf16* wf[2] = {nullptr, nullptr};
    bf16* wd = nullptr;
    CUtensorMap map_wf[2], map_wd;
};

// Chunking of a voxel reduction: about two CTAs per SM over all groups.
uint32_t chunks_for(uint32_t tiles, uint32_t groups) {
    uint32_t c = (296u + groups - 1u) / groups;
    if (c > tiles) c = tiles;
    return c < 1u ? 1u : c;
}

}  // namespace

bool halo_maps(ConvArgs& a) {
    for (uint32_t k = 0; k < a.nblocks; ++k)
        if (!a.in_ptr[k] || !halo_map(&a.halo[k], a.in_ptr[k], a.cb[k], a.vol)) return false;
    return true;
}

struct Net {
    slosh_unet_config_t cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    Vol vol[4];
    std::vector<Tensor> T;
    std::vector<Conv> C;
    int t_in = -1, t_e0 = -1, t_d0 = -1;
    uint64_t num_params = 0, head_off = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    float *target = nullptr, *guess = nullptr;
    uint32_t* meta = nullptr;    // per slot: scale bits, fluid count
    uint32_t* nfluid = nullptr;  // total fluid voxels of the batch
    uint32_t* error = nullptr;
    float *wpartial = nullptr, *bpartial = nullptr, *hpartial = nullptr, *head_grad = nullptr;
    double* energy = nullptr;  // warm-start scale partials
    float* beta = nullptr;     // warm-start scale of the last guess
    uint32_t head_chunks = 0, bias_chunks = 0;
    uint64_t step = 0;
    uint64_t launches = 0;

    int add_tensor(uint32_t c, uint32_t level, bool relu) {
        Tensor t;
        t.c = c;
        t.level = level;
        t.relu = relu;
        const size_t n = size_t(vol[level].voxels()) * c;
        t.act = dmalloc<bf16>(n);
        t.grad = dmalloc<bf16>(n);
        t.map_act = act_map(t.act, c, vol[level]);
        t.map_grad = act_map(t.grad, c, vol[level]);
        T.push_back(t);
        return int(T.size()) - 1;
    }
    int add_conv(int in0, int in1, uint32_t n) {
        Conv c;
        c.in[0] = in0;
        c.in[1] = in1;
        c.nblocks = in1 >= 0 ? 2u : 1u;
        c.cb[0] = T[size_t(in0)].c;
        c.cb[1] = in1 >= 0 ? T[size_t(in1)].c : 0u;
        c.cin = c.cb[0] + c.cb[1];
        c.n = n;
        c.out = add_tensor(n, T[size_t(in0)].level, true);
        c.w_off = num_params;
        num_params += 27ull * n * c.cin;
        c.b_off = num_params;
        num_params += n;
        for (uint32_t k = 0; k < c.nblocks; ++k) {
            c.wf[k] = dmalloc<bf16>(27ull * n * c.cb[k]);
            c.map_wf[k] = wgt_map(c.wf[k], c.cb[k], n);
        }
        c.wd = dmalloc<bf16>(27ull * n * c.cin);
        c.map_wd = wgt_map(c.wd, n, c.cin);
        C.push_back(c);
        return int(C.size()) - 1;
    }

    Net(const slosh_unet_config_t& config, int dev) : cfg(config), device(dev) {
        if (device < 0) UCK(cudaGetDevice(&device));  // -1: the calling thread's current device
        UCK(cudaSetDevice(device));
        UCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const uint32_t W = cfg.dim[0], H = cfg.dim[1], D = cfg.dim[2], B = cfg.batch ? cfg.batch : 1u;
        if (W % 8u || H % 8u || D % 8u || !W || !H || !D) throw std::invalid_argument("grid dimensions must be multiples of 8");
        for (uint32_t l = 0; l < 4; ++l) vol[l] = make_vol(W >> l, H >> l, D >> l, B);
        t_in = add_tensor(IN_CHANNELS, 0, false);
        const int e0a = C[size_t(add_conv(t_in, -1, 16))].out;
        t_e0 = C[size_t(add_conv(e0a, -1, 16))].out;
        const int p1 = add_tensor(16, 1, false);
        const int e1a = C[size_t(add_conv(p1, -1, 32))].out;
        const int e1 = C[size_t(add_conv(e1a, -1, 32))].out;
        const int p2 = add_tensor(32, 2, false);
        const int e2a = C[size_t(add_conv(p2, -1, 64))].out;
        const int e2 = C[size_t(add_conv(e2a, -1, 64))].out;
        const int p3 = add_tensor(64, 3, false);
        const int e3a = C[size_t(add_conv(p3, -1, 64))].out;
        add_conv(e3a, -1, 64);
        const int u2 = add_tensor(64, 2, false);
        const int d2a = C[size_t(add_conv(u2, e2, 64))].out;
        add_conv(d2a, -1, 64);
        const int u1 = add_tensor(64, 1, false);
        const int d1a = C[size_t(add_conv(u1, e1, 32))].out;
        add_conv(d1a, -1, 32);
        const int u0 = add_tensor(32, 0, false);
        const int d0a = C[size_t(add_conv(u0, t_e0, 16))].out;
        t_d0 = C[size_t(add_conv(d0a, -1, 16))].out;
        head_off = num_params;
        num_params += 17;
        params = dmalloc<float>(num_params);
        grads = dmalloc<float>(num_params);
        adam_m = dmalloc<float>(num_params);
        adam_v = dmalloc<float>(num_params);
        const uint64_t v0 = vol[0].voxels();
        target = dmalloc<float>(v0);
        guess = dmalloc<float>(v0);
        meta = dmalloc<uint32_t>(2ull * B);
        nfluid = dmalloc<uint32_t>(1);
        error = dmalloc<uint32_t>(1);
        size_t wp = 0;
        for (const Conv& c : C)
            for (uint32_t k = 0; k < c.nblocks; ++k) {
                const uint32_t Tt = 128u / c.cb[k];
                const uint32_t groups = (27u + Tt - 1u) / Tt;
                const size_t need = size_t(chunks_for(vol[T[size_t(c.in[k])].level].tiles(), groups)) * 27u * c.n * c.cb[k];
                if (need > wp) wp = need;
            }
        wpartial = dmalloc<float>(wp);
        bias_chunks = 256;
        bpartial = dmalloc<float>(size_t(bias_chunks) * 64u);
        head_chunks = 592;
        hpartial = dmalloc<float>(size_t(head_chunks) * 18u);
        head_grad = dmalloc<float>(18);
        energy = dmalloc<double>(2u * 592u);
        beta = dmalloc<float>(1);
        // dmalloc clears on the legacy default stream, which `stream` (non-blocking) does not wait for
        UCK(cudaDeviceSynchronize());
        init_params();
    }
    ~Net() {
        cudaSetDevice(device);
        cudaStreamSynchronize(stream);
        for (Tensor& t : T) {
            cudaFree(t.act);
            cudaFree(t.grad);
        }
        for (Conv& c : C) {
            for (uint32_t k = 0; k < c.nblocks; ++k) cudaFree(c.wf[k]);
            cudaFree(c.wd);
        }
        for (void* p : {(void*)params, (void*)grads, (void*)adam_m, (void*)adam_v, (void*)target, (void*)guess, (void*)meta, (void*)nfluid,
                        (void*)error, (void*)wpartial, (void*)bpartial, (void*)hpartial, (void*)head_grad, (void*)energy, (void*)beta})
            cudaFree(p);
        cudaStreamDestroy(stream);
    }

    // He-normal weights (std sqrt(2 / fan_in), fan_in = 27 x real input channels), zero biases.
    void init_params() {
        std::vector<float> h(num_params, 0.0f);
        std::mt19937 rng(cfg.seed);
        for (size_t i = 0; i < C.size(); ++i) {
            const Conv& c = C[i];
            const uint32_t fan_cin = i == 0 ? 3u : c.cin;
            std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / float(27u * fan_cin)));
            for (uint64_t j = 0; j < 27ull * c.n * c.cin; ++j) h[c.w_off + j] = nd(rng);
        }
        std::normal_distribution<float> nh(0.0f, std::sqrt(1.0f / 16.0f));
        for (int j = 0; j < 16; ++j) h[head_off + uint64_t(j)] = nh(rng);
        set_params(h.data());
    }
    void set_params(const float* h) {
        UCK(cudaMemcpyAsync(params, h, num_params * 4, cudaMemcpyHostToDevice, stream));
        UCK(cudaMemsetAsync(adam_m, 0, num_params * 4, stream));
        UCK(cudaMemsetAsync(adam_v, 0, num_params * 4, stream));
        step = 0;
        refresh_weights();
        UCK(cudaStreamSynchronize(stream));
    }
    void refresh_weights() {
        for (const Conv& c : C) launches += launch_conv_weights(params + c.w_off, c.n, c.cin, c.cb, c.nblocks, c.wf, c.wd, stream);
    }

    ConvArgs conv_args(const Conv& c) const {
        ConvArgs a;
        std::memset(static_cast<void*>(&a), 0, sizeof(a));
        a.nblocks = c.nblocks;
        a.n = c.n;
        for (uint32_t k = 0; k < c.nblocks; ++k) {
            a.act[k] = T[size_t(c.in[k])].map_act;
            a.wgt[k] = c.map_wf[k];
            a.cb[k] = c.cb[k];
            a.in_ptr[k] = T[size_t(c.in[k])].act;
            a.w_ptr[k] = c.wf[k];
        }
        a.vol = vol[T[size_t(c.out)].level];
        a.bias = params + c.b_off;
        a.relu = 1;
        a.out[0] = T[size_t(c.out)].act;
        a.oc[0] = c.n;
        a.error = error;
        return a;
    }
    void forward() {
        for (size_t i = 0; i < C.size(); ++i) {
            launches += launch_conv(conv_args(C[i]), stream);
            after_conv(i);
        }
        launches += launch_head(T[size_t(t_d0)].act, T[size_t(t_in)].act, params + head_off, guess, nullptr, nullptr, nullptr, nullptr,
                                head_chunks, nullptr, vol[0].voxels(), stream);
    }
    // The resampling step that follows convolution i in the forward order.
    void after_conv(size_t i) {
        switch (i) {
            case 1: launches += launch_pool(T[size_t(C[1].out)].act, T[size_t(C[2].in[0])].act, vol[0], 16, stream); break;
            case 3: launches += launch_pool(T[size_t(C[3].out)].act, T[size_t(C[4].in[0])].act, vol[1], 32, stream); break;
            case 5: launches += launch_pool(T[size_t(C[5].out)].act, T[size_t(C[6].in[0])].act, vol[2], 64, stream); break;
            case 7: launches += launch_upsample(T[size_t(C[7].out)].act, T[size_t(C[8].in[0])].act, vol[2], 64, stream); break;
            case 9: launches += launch_upsample(T[size_t(C[9].out)].act, T[size_t(C[10].in[0])].act, vol[1], 64, stream); break;
            case 11: launches += launch_upsample(T[size_t(C[11].out)].act, T[size_t(C[12].in[0])].act, vol[0], 32, stream); break;
            default: break;
        }
    }

    // Weight and bias gradients of convolution c from its (masked) output gradient.
    void conv_param_grads(const Conv& c) {
        const Tensor& out = T[size_t(c.out)];
        const Vol& v = vol[out.level];
        for (uint32_t k = 0; k < c.nblocks; ++k) {
            WgradArgs w;
            std::memset(static_cast<void*>(&w), 0, sizeof(w));
            w.act = T[size_t(c.in[k])].map_act;
            w.grad = out.map_grad;
            w.c = c.cb[k];
            w.n = c.n;
            w.vol = v;
            const uint32_t Tt = 128u / c.cb[k], groups = (27u + Tt - 1u) / Tt;
            const uint32_t chunks = chunks_for(v.tiles(), groups);
            w.tiles_per_chunk = (v.tiles() + chunks - 1u) / chunks;
            const uint32_t used = (v.tiles() + w.tiles_per_chunk - 1u) / w.tiles_per_chunk;
            w.partial = wpartial;
            w.error = error;
            launches += launch_wgrad(w, used, stream);
            launches += launch_reduce_wgrad(wpartial, grads + c.w_off, used, c.n, c.cb[k], c.cin, k == 0 ? 0u : c.cb[0], stream);
        }
        launches += launch_bias_grad(out.grad, c.n, v.voxels(), bpartial, bias_chunks, grads + c.b_off, stream);
    }
    // Data gradient of convolution c into its inputs' gradients (write or add, masked where asked).
    void conv_data_grad(const Conv& c, const uint32_t accumulate[2], const bf16* const mask[2]) {
        ConvArgs a;
        std::memset(static_cast<void*>(&a), 0, sizeof(a));
        const Tensor& out = T[size_t(c.out)];
        a.nblocks = 1;
        a.act[0] = out.map_grad;
        a.wgt[0] = c.map_wd;
        a.cb[0] = c.n;
        a.n = c.cin;
        a.in_ptr[0] = out.grad;
        a.w_ptr[0] = c.wd;
        a.vol = vol[out.level];
        a.bias = nullptr;
        a.relu = 0;
        a.out[0] = T[size_t(c.in[0])].grad;
        a.oc[0] = c.cb[0];
        a.mask[0] = mask[0];
        if (c.nblocks > 1) {
            a.out[1] = T[size_t(c.in[1])].grad;
            a.oc[1] = c.cb[1];
            a.mask[1] = mask[1];
        }
        a.accumulate = accumulate[0];
        if (c.nblocks > 1 && accumulate[1] != accumulate[0]) throw std::logic_error("mixed accumulation");
        a.error = error;
        launches += launch_conv(a, stream);
    }

    float backward_and_grads() {
        UCK(cudaMemsetAsync(grads, 0, num_params * 4, stream));
        launches += launch_head(T[size_t(t_d0)].act, T[size_t(t_in)].act, params + head_off, guess, target, nfluid, T[size_t(t_d0)].grad,
                                hpartial, head_chunks, head_grad, vol[0].voxels(), stream);
        UCK(cudaMemcpyAsync(grads + head_off, head_grad, 17 * 4, cudaMemcpyDeviceToDevice, stream));
        const uint32_t wr[2] = {0u, 0u};
        // convolutions in reverse; the gradient of every ReLU tensor is masked by its last contribution
        for (int i = int(C.size()) - 1; i >= 0; --i) {
            const Conv& c = C[size_t(i)];
            conv_param_grads(c);
            if (i == 0) break;
            const Tensor& in0 = T[size_t(c.in[0])];
            const bf16* mask[2] = {in0.relu ? in0.act : nullptr, nullptr};
            // skip-connection inputs (block 1) get their first contribution here, unmasked (the pooling
            // gradient adds the second one and masks)
            if (c.nblocks > 1) mask[1] = nullptr;
            conv_data_grad(c, wr, mask);
            // the resampling step before convolution i, backwards
            switch (i) {
                case 12: launches += launch_upsample_bwd(T[size_t(C[12].in[0])].grad, T[size_t(C[11].out)].grad, vol[0], 32, T[size_t(C[11].out)].act, stream); break;
                case 10: launches += launch_upsample_bwd(T[size_t(C[10].in[0])].grad, T[size_t(C[9].out)].grad, vol[1], 64, T[size_t(C[9].out)].act, stream); break;
                case 8: launches += launch_upsample_bwd(T[size_t(C[8].in[0])].grad, T[size_t(C[7].out)].grad, vol[2], 64, T[size_t(C[7].out)].act, stream); break;
                case 6: launches += launch_pool_bwd(T[size_t(C[6].in[0])].grad, T[size_t(C[5].out)].grad, vol[2], 64, 1u, T[size_t(C[5].out)].act, stream); break;
                case 4: launches += launch_pool_bwd(T[size_t(C[4].in[0])].grad, T[size_t(C[3].out)].grad, vol[1], 32, 1u, T[size_t(C[3].out)].act, stream); break;
                case 2: launches += launch_pool_bwd(T[size_t(C[2].in[0])].grad, T[size_t(C[1].out)].grad, vol[0], 16, 1u, T[size_t(C[1].out)].act, stream); break;
                default: break;
            }
        }
        float loss = 0.0f;
        UCK(cudaMemcpyAsync(&loss, head_grad + 17, 4, cudaMemcpyDeviceToHost, stream));
        UCK(cudaStreamSynchronize(stream));
        check_error();
        return loss;
    }
    void adam_step() {
        ++step;
        const float b1 = cfg.beta1, b2 = cfg.beta2;
        const float c1 = 1.0f / (1.0f - std::pow(b1, float(step)));
        const float c2 = 1.0f / (1.0f - std::pow(b2, float(step)));
        launches += launch_adam(params, grads, adam_m, adam_v, num_params, cfg.learning_rate, b1, b2, cfg.eps, c1, c2, stream);
        refresh_weights();
    }
    void check_error() {
        uint32_t e = 0;
        UCK(cudaMemcpy(&e, error, 4, cudaMemcpyDeviceToHost));
        if (e) {
            UCK(cudaMemsetAsync(error, 0, 4, stream));
            UCK(cudaStreamSynchronize(stream));
            throw std::runtime_error("tensor-core pipeline wait timed out (error bits " + std::to_string(e) + ")");
        }
    }
    // Batch totals after the samples were packed: fluid voxel count over all slots.
    void finish_batch() {
        std::vector<uint32_t> m(2ull * vol[0].B);
        UCK(cudaMemcpyAsync(m.data(), meta, m.size() * 4, cudaMemcpyDeviceToHost, stream));
        UCK(cudaStreamSynchronize(stream));
        uint32_t total = 0;
        for (uint32_t b = 0; b < vol[0].B; ++b) total += m[2u * b + 1u];
        UCK(cudaMemcpyAsync(nfluid, &total, 4, cudaMemcpyHostToDevice, stream));
        UCK(cudaStreamSynchronize(stream));
    }
};

// Warm start of a simulation's pressure solve (slot 0 of the network's batch).
int warm_start(Net* net, const Dev& d, const float* divergence, float* pressure, cudaStream_t s) {
    if (uint32_t(d.grid.x) != net->vol[0].W || uint32_t(d.grid.y) != net->vol[0].H || uint32_t(d.grid.z) != net->vol[0].D)
        throw std::invalid_argument("warm-start network grid differs from the simulation grid");
    cudaStream_t keep = net->stream;
    net->stream = s;
    int n = 0;
    UCK(cudaMemsetAsync(net->meta, 0, 8, s));
    n += launch_pack_input(d, divergence, nullptr, net->T[size_t(net->t_in)].act, nullptr, net->meta, 0u, s);
    const uint64_t before = net->launches;
    net->forward();
    n += int(net->launches - before);
    n += launch_scatter_guess(d, net->guess, net->T[size_t(net->t_in)].act, divergence, net->energy, 592u, net->beta, pressure, s);
    net->stream = keep;
    return n;
}

}  // namespace unet
}  // namespace slosh

using slosh::unet::Net;

namespace {
thread_local std::string g_unet_error;
template <class F>
slosh_status unet_guard(F&& f) {
    try {
        return f();
    } catch (const slosh::unet::CudaFail& e) {
        g_unet_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return SLOSH_ERR_CUDA;
    } catch (const std::invalid_argument& e) {
        g_unet_error = e.what();
        return SLOSH_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        g_unet_error = e.what();
        return SLOSH_ERR_CUDA;
    }
}
Net* as_net(void* p) {
    if (!p) throw std::invalid_argument("network is NULL");
    return static_cast<Net*>(p);
}
}  // namespace

SLOSH_API const char* slosh_unet_last_error(void) { return g_unet_error.c_str(); }

SLOSH_API void slosh_unet_config_default(slosh_unet_config_t* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->dim[0] = out->dim[1] = out->dim[2] = 128;
    out->batch = 1;
    out->seed = 10000;
    out->learning_rate = 1e-3f;
    out->beta1 = 0.9f;
    out->beta2 = 0.999f;
    out->eps = 1e-8f;
}
SLOSH_API slosh_status slosh_unet_create(const slosh_unet_config_t* config, int32_t device, void** out_net) {
    return unet_guard([&]() -> slosh_status {
        if (!config || !out_net) throw std::invalid_argument("NULL argument");
        *out_net = new Net(*config, device);
        return SLOSH_OK;
    });
}
SLOSH_API void slosh_unet_destroy(void* net) { delete static_cast<Net*>(net); }
SLOSH_API uint64_t slosh_unet_num_params(void* net) { return net ? static_cast<Net*>(net)->num_params : 0; }
SLOSH_API slosh_status slosh_unet_get_params(void* net, float* host, uint64_t count) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        if (!host || count != n->num_params) throw std::invalid_argument("parameter count mismatch");
        UCK(cudaMemcpyAsync(host, n->params, count * 4, cudaMemcpyDeviceToHost, n->stream));
        UCK(cudaStreamSynchronize(n->stream));
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_set_params(void* net, const float* host, uint64_t count) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        if (!host || count != n->num_params) throw std::invalid_argument("parameter count mismatch");
        n->set_params(host);
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_set_sample(void* net, uint32_t slot, const uint16_t* input_bf16, const float* target, uint32_t fluid_voxels) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        if (slot >= n->vol[0].B || !input_bf16) throw std::invalid_argument("bad slot or input");
        const uint64_t v = n->vol[0].W * uint64_t(n->vol[0].H) * n->vol[0].D;
        UCK(cudaMemcpyAsync(n->T[size_t(n->t_in)].act + slot * v * slosh::unet::IN_CHANNELS, input_bf16, v * slosh::unet::IN_CHANNELS * 2,
                            cudaMemcpyHostToDevice, n->stream));
        if (target) UCK(cudaMemcpyAsync(n->target + slot * v, target, v * 4, cudaMemcpyHostToDevice, n->stream));
        const uint32_t m[2] = {0x3F800000u, fluid_voxels};  // scale 1
        UCK(cudaMemcpyAsync(n->meta + 2u * slot, m, 8, cudaMemcpyHostToDevice, n->stream));
        UCK(cudaStreamSynchronize(n->stream));
        n->finish_batch();
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_capture_sample(void* net, void* sim_ctx, uint32_t slot) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        if (slot >= n->vol[0].B) throw std::invalid_argument("bad slot");
        slosh::Dev d;
        float *div = nullptr, *pres = nullptr;
        cudaStream_t s = nullptr;
        if (!slosh::unet::sim_ctx_dev(sim_ctx, &d, &div, &pres, &s)) throw std::invalid_argument("bad simulation context");
        if (uint32_t(d.grid.x) != n->vol[0].W || uint32_t(d.grid.y) != n->vol[0].H || uint32_t(d.grid.z) != n->vol[0].D)
            throw std::invalid_argument("network grid differs from the simulation grid");
        UCK(cudaStreamSynchronize(s));
        UCK(cudaMemsetAsync(n->meta + 2u * slot, 0, 8, n->stream));
        const uint64_t v = uint64_t(d.grid.x) * d.grid.y * d.grid.z;
        n->launches += slosh::unet::launch_pack_input(d, div, pres, n->T[size_t(n->t_in)].act, n->target, n->meta, slot, n->stream);
        (void)v;
        UCK(cudaStreamSynchronize(n->stream));
        n->finish_batch();
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_forward(void* net, float* host_guess) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        n->forward();
        if (host_guess)
            UCK(cudaMemcpyAsync(host_guess, n->guess, n->vol[0].voxels() * 4, cudaMemcpyDeviceToHost, n->stream));
        UCK(cudaStreamSynchronize(n->stream));
        n->check_error();
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_backward(void* net, float* out_loss, float* host_grads) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        const float loss = n->backward_and_grads();
        if (out_loss) *out_loss = loss;
        if (host_grads) {
            UCK(cudaMemcpyAsync(host_grads, n->grads, n->num_params * 4, cudaMemcpyDeviceToHost, n->stream));
            UCK(cudaStreamSynchronize(n->stream));
        }
        return SLOSH_OK;
    });
}
SLOSH_API slosh_status slosh_unet_train_step(void* net, float* out_loss) {
    return unet_guard([&]() -> slosh_status {
        Net* n = as_net(net);
        n->forward();
        const float loss = n->backward_and_grads();
        n->adam_step();
        if (out_loss) *out_loss = loss;
        return SLOSH_OK;
    });
}
SLOSH_API uint64_t slosh_unet_launch_count(void* net) { return net ? static_cast<Net*>(net)->launches : 0; }

// One convolution through the same kernels, on host arrays: y = relu(conv(x) + b), the data gradient
// dx of dz = dy (no mask), dW and db. For parity tests of the kernels.
SLOSH_API slosh_status slosh_unet_conv_test(const slosh_conv_test_t* t) {
    using namespace slosh::unet;
    return unet_guard([&]() -> slosh_status {
        if (!t || !t->x[0] || !t->w || !t->dy) throw std::invalid_argument("NULL argument");
        const uint32_t nb = t->nblocks == 2u ? 2u : 1u;
        const Vol v = make_vol(t->dim[0], t->dim[1], t->dim[2], t->batch ? t->batch : 1u);
        const uint64_t nv = v.voxels();
        const uint32_t n = t->cout, cin = t->cin[0] + (nb > 1 ? t->cin[1] : 0u);
        for (uint32_t k = 0; k < nb; ++k)
            if (t->cin[k] != 16u && t->cin[k] != 32u && t->cin[k] != 64u) throw std::invalid_argument("block channels must be 16, 32 or 64");
        if (n != 16u && n != 32u && n != 64u) throw std::invalid_argument("cout must be 16, 32 or 64");
        cudaStream_t s;
        UCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        std::vector<void*> owned;
        auto alloc = [&](size_t bytes) {
            void* p = nullptr;
            UCK(cudaMalloc(&p, bytes + 16));
            UCK(cudaMemsetAsync(p, 0, bytes + 16, s));  // on the work stream, so it is ordered before the uploads
            owned.push_back(p);
            return p;
        };
        slosh_status st = SLOSH_OK;
        try {
            bf16* x[2] = {nullptr, nullptr};
            bf16* dx[2] = {nullptr, nullptr};
            for (uint32_t k = 0; k < nb; ++k) {
                x[k] = static_cast<bf16*>(alloc(nv * t->cin[k] * 2));
                dx[k] = static_cast<bf16*>(alloc(nv * t->cin[k] * 2));
                UCK(cudaMemcpyAsync(x[k], t->x[k], nv * t->cin[k] * 2, cudaMemcpyHostToDevice, s));
            }
            bf16* y = static_cast<bf16*>(alloc(nv * n * 2));
            bf16* dz = static_cast<bf16*>(alloc(nv * n * 2));
            UCK(cudaMemcpyAsync(dz, t->dy, nv * n * 2, cudaMemcpyHostToDevice, s));
            float* w = static_cast<float*>(alloc(27ull * n * cin * 4));
            float* b = static_cast<float*>(alloc(n * 4));
            UCK(cudaMemcpyAsync(w, t->w, 27ull * n * cin * 4, cudaMemcpyHostToDevice, s));
            if (t->bias) UCK(cudaMemcpyAsync(b, t->bias, n * 4, cudaMemcpyHostToDevice, s));
            bf16* wf[2] = {nullptr, nullptr};
            for (uint32_t k = 0; k < nb; ++k) wf[k] = static_cast<bf16*>(alloc(27ull * n * t->cin[k] * 2));
            bf16* wd = static_cast<bf16*>(alloc(27ull * n * cin * 2));
            uint32_t* err = static_cast<uint32_t*>(alloc(4));
            launch_conv_weights(w, n, cin, t->cin, nb, wf, wd, s);
            ConvArgs a;
            std::memset(static_cast<void*>(&a), 0, sizeof(a));
            a.nblocks = nb;
            a.n = n;
            for (uint32_t k = 0; k < nb; ++k) {
                a.act[k] = act_map(x[k], t->cin[k], v);
                a.wgt[k] = wgt_map(wf[k], t->cin[k], n);
                a.cb[k] = t->cin[k];
                a.in_ptr[k] = x[k];
                a.w_ptr[k] = wf[k];
            }
            a.vol = v;
            a.bias = b;
            a.relu = 1;
            a.out[0] = y;
            a.oc[0] = n;
            a.error = err;
            launch_conv(a, s);
            ConvArgs g;
            std::memset(static_cast<void*>(&g), 0, sizeof(g));
            g.nblocks = 1;
            g.act[0] = act_map(dz, n, v);
            g.wgt[0] = wgt_map(wd, n, cin);
            g.cb[0] = n;
            g.n = cin;
            g.in_ptr[0] = dz;
            g.w_ptr[0] = wd;
            g.vol = v;
            g.out[0] = dx[0];
            g.oc[0] = t->cin[0];
            if (nb > 1) {
                g.out[1] = dx[1];
                g.oc[1] = t->cin[1];
            }
            g.error = err;
            launch_conv(g, s);
            float* dw = static_cast<float*>(alloc(27ull * n * cin * 4));
            float* db = static_cast<float*>(alloc(n * 4));
            for (uint32_t k = 0; k < nb; ++k) {
                WgradArgs wa;
                std::memset(static_cast<void*>(&wa), 0, sizeof(wa));
                wa.act = a.act[k];
                wa.grad = g.act[0];
                wa.c = t->cin[k];
                wa.n = n;
                wa.vol = v;
                const uint32_t Tt = 128u / t->cin[k], groups = (27u + Tt - 1u) / Tt;
                const uint32_t chunks = chunks_for(v.tiles(), groups);
                wa.tiles_per_chunk = (v.tiles() + chunks - 1u) / chunks;
                const uint32_t used = (v.tiles() + wa.tiles_per_chunk - 1u) / wa.tiles_per_chunk;
                wa.partial = static_cast<float*>(alloc(size_t(used) * 27u * n * t->cin[k] * 4));
                wa.error = err;
                launch_wgrad(wa, used, s);
                launch_reduce_wgrad(wa.partial, dw, used, n, t->cin[k], cin, k == 0 ? 0u : t->cin[0], s);
            }
            float* bp = static_cast<float*>(alloc(64ull * 64u * 4));
            launch_bias_grad(dz, n, nv, bp, 64, db, s);
            UCK(cudaGetLastError());
            UCK(cudaStreamSynchronize(s));
            uint32_t e = 0;
            UCK(cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost));
            if (e) throw std::runtime_error("tensor-core pipeline wait timed out (error bits " + std::to_string(e) + ")");
            if (t->y) UCK(cudaMemcpy(t->y, y, nv * n * 2, cudaMemcpyDeviceToHost));
            for (uint32_t k = 0; k < nb; ++k)
                if (t->dx[k]) UCK(cudaMemcpy(t->dx[k], dx[k], nv * t->cin[k] * 2, cudaMemcpyDeviceToHost));
            if (t->dw) UCK(cudaMemcpy(t->dw, dw, 27ull * n * cin * 4, cudaMemcpyDeviceToHost));
            if (t->db) UCK(cudaMemcpy(t->db, db, n * 4, cudaMemcpyDeviceToHost));
        } catch (...) {
            for (void* p : owned) cudaFree(p);
            cudaStreamDestroy(s);
            throw;
        }
        for (void* p : owned) cudaFree(p);
        cudaStreamDestroy(s);
        return st;
    });
}
