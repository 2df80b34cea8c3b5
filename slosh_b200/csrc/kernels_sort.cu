// Spatial sort of particles by 4^3 block key with compaction of dead slots (sm_100a).
//
// Reference: PLUG/Shaders/Private/SloshSort.usf (SortKey :36-47, SortCountCS :65-76, scans :78-132,
// SortScatterCS :134-146, SortWriteCountCS :149-154) and AddSpatialSort, SloshProxy.cpp:1022-1087.
//
// The reference ranks particles inside a key with an atomic counter, so its permutation depends on
// thread timing. This sort is stable: it orders by key and, inside a key, by source slot -- the order
// the reference produces when its atomics resolve in ascending thread order. It is an LSD radix sort of
// (key, slot) pairs with 8-bit digits; each pass is reduce-then-scan:
//   upsweep   per 4096-item tile, a shared-memory histogram of the digit (tile_hist[digit][tile]);
//   scan      exclusive scan of tile_hist in digit-major order = each tile's first output position;
//   scatter   each warp ranks its 512 contiguous items in order (warp match + per-warp counters), the
//             per-warp counters are prefixed across warps, and items go to tile base + rank.
// No step waits on another CTA. Per-key counts come from warp-aggregated atomics (integer, exact),
// and their exclusive scan gives the key offsets and the live count.
#include "kernels.h"

namespace slosh {

namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_ROUNDS = 16;                      // items per lane
constexpr int SORT_TILE = SORT_THREADS * SORT_ROUNDS;  // 4096 items per tile
constexpr int WARP_ITEMS = 32 * SORT_ROUNDS;           // 512 contiguous items per warp
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t sort_key_of(const Dev& d, float4 a, int3 sdim, uint32_t num_keys) {
    if (is_dead_age(a.w)) return num_keys - 1u;
    const int cx = clampi(int(floorf(a.x * d.inv_h)), 0, d.grid.x - 1);
    const int cy = clampi(int(floorf(a.y * d.inv_h)), 0, d.grid.y - 1);
    const int cz = clampi(int(floorf(a.z * d.inv_h)), 0, d.grid.z - 1);
    const uint32_t k = uint32_t((cx >> 2) + sdim.x * ((cy >> 2) + sdim.y * (cz >> 2)));
    return min(k, num_keys - 2u);
}

__device__ __forceinline__ uint32_t tile_item(uint32_t tile, int r) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return tile * uint32_t(SORT_TILE) + uint32_t(warp * WARP_ITEMS + r * 32 + lane);
}

// Keys, per-key counts and the digit-0 tile histogram.
__global__ void __launch_bounds__(SORT_THREADS) k_keys(Dev d, const slosh_particle_t* __restrict__ particles, uint32_t n,
                                                       uint32_t* __restrict__ keys, uint32_t* __restrict__ counts,
                                                       uint32_t* __restrict__ tile_hist, uint32_t num_tiles, int3 sdim,
                                                       uint32_t num_keys) {
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const int lane = threadIdx.x & 31;
#pragma unroll 4
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        const uint32_t i = tile_item(tile, r);
        const bool valid = i < n;
        uint32_t key = 0xFFFFFFFFu;
        if (valid) {
            key = sort_key_of(d, __ldg(reinterpret_cast<const float4*>(particles + i)), sdim, num_keys);
            keys[i] = key;
            atomicAdd(hist + (key & 0xFFu), 1u);
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(counts + key, uint32_t(__popc(peers)));
    }
    __syncthreads();
    tile_hist[threadIdx.x * num_tiles + tile] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(SORT_THREADS) k_upsweep(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ tile_hist,
                                                          uint32_t num_tiles, uint32_t shift) {
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
#pragma unroll 4
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        const uint32_t i = tile_item(tile, r);
        if (i < n) atomicAdd(hist + ((__ldg(keys + i) >> shift) & 0xFFu), 1u);
    }
    __syncthreads();
    tile_hist[threadIdx.x * num_tiles + tile] = hist[threadIdx.x];
}

// Stable scatter of one digit. vals_in == nullptr means the identity (source slot = item index);
// keys_out == nullptr skips writing keys (last pass).
__global__ void __launch_bounds__(SORT_THREADS) k_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                          uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                                                          const uint32_t* __restrict__ tile_scan, uint32_t num_tiles, uint32_t shift) {
    __shared__ uint32_t whist[SORT_WARPS][256];
    for (int t = threadIdx.x; t < SORT_WARPS * 256; t += SORT_THREADS) (&whist[0][0])[t] = 0u;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t key[SORT_ROUNDS], val[SORT_ROUNDS], rank[SORT_ROUNDS];
#pragma unroll
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        const uint32_t i = tile_item(tile, r);
        const bool valid = i < n;
        key[r] = valid ? __ldg(keys_in + i) : 0u;
        val[r] = valid ? (vals_in ? __ldg(vals_in + i) : i) : 0u;
        const uint32_t digit = valid ? ((key[r] >> shift) & 0xFFu) : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
        uint32_t before = 0u;
        if (valid) before = whist[warp][digit];
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) whist[warp][digit] = before + uint32_t(__popc(peers));
        __syncwarp();
        rank[r] = valid ? before + uint32_t(__popc(peers & lt_mask)) : 0xFFFFFFFFu;
    }
    __syncthreads();
    {
        const uint32_t dgt = threadIdx.x;
        uint32_t run = tile_scan[dgt * num_tiles + tile];
#pragma unroll
        for (int w = 0; w < SORT_WARPS; ++w) {
            const uint32_t t = whist[w][dgt];
            whist[w][dgt] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        if (rank[r] == 0xFFFFFFFFu) continue;
        const uint32_t dst = whist[warp][(key[r] >> shift) & 0xFFu] + rank[r];
        if (keys_out) keys_out[dst] = key[r];
        vals_out[dst] = val[r];
    }
}

// Gather of the 48-byte records in sorted order; perm keeps the source slot of every output.
__global__ void k_gather(const slosh_particle_t* __restrict__ in, slosh_particle_t* __restrict__ out, const uint32_t* __restrict__ vals,
                         uint32_t* __restrict__ perm, uint32_t n) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t src = __ldg(vals + j);
    const float4* s = reinterpret_cast<const float4*>(in + src);
    float4* o = reinterpret_cast<float4*>(out + j);
    const float4 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2);
    o[0] = a;
    o[1] = b;
    o[2] = c;
    perm[j] = src;
}

// ---- exclusive scan of u32 (three kernels, in place allowed) ----------------------------------------
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
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
        const int nw = blockDim.x / 32;
        uint32_t w = lane < nw ? s_warp[lane] : 0u;
        uint32_t ws = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, ws, off);
            if (lane >= off) ws += y;
        }
        if (lane < nw) s_warp[lane] = ws - w;
        if (lane == 31) s_warp[32] = ws;
    }
    __syncthreads();
    const uint32_t ex = s_warp[warp] + x - v;
    *total = s_warp[32];
    __syncthreads();
    return ex;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ sums) {
    __shared__ uint32_t s_warp[33];
    const uint32_t base = blockIdx.x * uint32_t(SCAN_TILE) + threadIdx.x * uint32_t(SCAN_ITEMS);
    uint32_t v = 0u;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + uint32_t(k) < n) v += in[base + uint32_t(k)];
    uint32_t total;
    block_excl_scan(v, s_warp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t* sums, uint32_t nb) {
    __shared__ uint32_t s_warp[33];
    const uint32_t per = (nb + blockDim.x - 1u) / blockDim.x;
    const uint32_t b0 = min(threadIdx.x * per, nb), b1 = min(b0 + per, nb);
    uint32_t v = 0u;
    for (uint32_t b = b0; b < b1; ++b) v += sums[b];
    uint32_t total;
    uint32_t run = block_excl_scan(v, s_warp, &total);
    for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t t = sums[b];
        sums[b] = run;
        run += t;
    }
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const uint32_t* in, uint32_t* out, uint32_t n, const uint32_t* __restrict__ sums) {
    __shared__ uint32_t s_warp[33];
    const uint32_t base = blockIdx.x * uint32_t(SCAN_TILE) + threadIdx.x * uint32_t(SCAN_ITEMS);
    uint32_t vals[SCAN_ITEMS];
    uint32_t v = 0u;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        vals[k] = base + uint32_t(k) < n ? in[base + uint32_t(k)] : 0u;
        v += vals[k];
    }
    uint32_t total;
    uint32_t run = block_excl_scan(v, s_warp, &total) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + uint32_t(k) < n) out[base + uint32_t(k)] = run;
        run += vals[k];
    }
}

int exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s) {
    const uint32_t nb = (n + uint32_t(SCAN_TILE) - 1u) / uint32_t(SCAN_TILE);
    if (nb == 0) return 0;
    k_scan_reduce<<<nb, SCAN_THREADS, 0, s>>>(in, n, tmp);
    k_scan_sums<<<1, 1024, 0, s>>>(tmp, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, s>>>(in, out, n, tmp);
    return 3;
}

__global__ void k_live_count(const uint32_t* offsets, uint32_t num_keys, uint32_t* pc) {
    pc[0] = offsets[num_keys - 1u];
}

}  // namespace

int launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s) {
    return exclusive_scan(in, out, n, tmp, s);
}
size_t exclusive_scan_tmp_size(uint32_t n) { return (size_t(n) + SCAN_TILE - 1) / SCAN_TILE + 1; }

int3 sort_brick_dim(int3 g) { return make_int3((g.x + 3) / 4, (g.y + 3) / 4, (g.z + 3) / 4); }

size_t sort_tile_hist_size(uint32_t capacity) {
    const size_t tiles = (size_t(capacity) + SORT_TILE - 1) / SORT_TILE;
    return 256 * (tiles > 0 ? tiles : 1);
}
size_t sort_scan_tmp_size(uint32_t capacity, uint32_t num_sort_keys) {
    const size_t a = (sort_tile_hist_size(capacity) + SCAN_TILE - 1) / SCAN_TILE;
    const size_t b = (size_t(num_sort_keys) + SCAN_TILE - 1) / SCAN_TILE;
    return (a > b ? a : b) + 1;
}

int launch_sort(const Dev& d, const SortBuffers& b, const slosh_particle_t* in, slosh_particle_t* out, uint32_t n,
                uint32_t num_keys, int3 sdim, cudaStream_t s) {
    int launches = 0;
    cudaMemsetAsync(b.counts, 0, sizeof(uint32_t) * num_keys, s);
    if (n == 0) {
        launches += exclusive_scan(b.counts, b.offsets, num_keys, b.scan_tmp, s);
        k_live_count<<<1, 1, 0, s>>>(b.offsets, num_keys, b.particle_count);
        return launches + 1;
    }
    const uint32_t num_tiles = (n + uint32_t(SORT_TILE) - 1u) / uint32_t(SORT_TILE);
    const uint32_t hist_n = 256u * num_tiles;
    uint32_t bits = 0;
    while ((1u << bits) < num_keys && bits < 32) ++bits;  // keys are < num_keys
    const int passes = bits <= 8 ? 1 : int((bits + 7) / 8);
    k_keys<<<num_tiles, SORT_THREADS, 0, s>>>(d, in, n, b.keys[0], b.counts, b.tile_hist, num_tiles, sdim, num_keys);
    ++launches;
    int cur = 0;
    for (int pass = 0; pass < passes; ++pass) {
        const uint32_t shift = uint32_t(pass) * 8u;
        if (pass > 0) {
            k_upsweep<<<num_tiles, SORT_THREADS, 0, s>>>(b.keys[cur], n, b.tile_hist, num_tiles, shift);
            ++launches;
        }
        launches += exclusive_scan(b.tile_hist, b.tile_hist, hist_n, b.scan_tmp, s);
        const bool last = pass == passes - 1;
        k_scatter<<<num_tiles, SORT_THREADS, 0, s>>>(b.keys[cur], pass == 0 ? nullptr : b.vals[cur], last ? nullptr : b.keys[cur ^ 1],
                                                     b.vals[cur ^ 1], n, b.tile_hist, num_tiles, shift);
        ++launches;
        cur ^= 1;
    }
    k_gather<<<(n + 255u) / 256u, 256, 0, s>>>(in, out, b.vals[cur], b.perm, n);
    ++launches;
    launches += exclusive_scan(b.counts, b.offsets, num_keys, b.scan_tmp, s);
    k_live_count<<<1, 1, 0, s>>>(b.offsets, num_keys, b.particle_count);
    return launches + 1;
}

}  // namespace slosh
