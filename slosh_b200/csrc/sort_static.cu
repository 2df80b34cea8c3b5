// Allocation-free spatial sort of caller-owned particle records (slosh_sort_particles_static).
//
// The context's sort (slosh_sort_particles) keeps its radix scratch in buffers that slosh_create
// allocates. This entry point runs the same kernels (launch_sort: keys, digit histograms, scans, stable
// scatter, gather) on particle arrays that the caller owns, without a context and without allocating
// anything: its scratch is the one static device array below, sized for at most
// SLOSH_STATIC_SORT_MAX_PARTICLES particles and SLOSH_STATIC_SORT_MAX_KEYS sort keys (7.4 MB per device).
//
// Who cannot allocate here, and why:
//   * an engine that reserves its device memory once at start-up and afterwards hands the simulation
//     only fixed buffers of its own (a render-graph transient heap, a pooled allocator): a stray
//     cudaMalloc breaks its budget and its residency accounting;
//   * a frame loop that must not stall: cudaFree synchronises the whole device, and a first-time
//     cudaMalloc can take milliseconds;
//   * a tool that re-sorts a particle snapshot without creating a simulation context (whose creation
//     allocates the whole brick pool).
//
// Set-up: a __device__ array has its own address in every CUDA context, so the address is resolved per
// context. Each call looks up the current context's unique ID (cuCtxGetId, fetched through
// cudaGetDriverEntryPoint, so the library needs no link against the driver library) in a small cache; on a
// miss it resolves the array's address with cudaGetSymbolAddress in that context and caches it. A host that
// runs in its own context (cuCtxCreate, an engine's or a green context), or that resets a device and starts
// again, therefore gets the address of its current context, never a stale one. The first call in a context
// also loads this library's device code there if it is not loaded yet (CUDA loads modules lazily by default),
// which commits the static scratch and the code on that device: that first call allocates, every later one
// does not. Make it during start-up, before any stream capture begins in that context; with
// CUDA_MODULE_LOADING=EAGER the load happens when the context is created instead.
//
// Races: there is one scratch per device. Calls that overlap on a device -- two streams, or two host
// threads, with nothing ordering them -- race on it and corrupt each other's results. Issue them on one
// stream, or order them with events or a lock.
//
// What must start at zero: only the per-key counts, which launch_sort clears on the stream at the start of
// every call; every other scratch word is written before it is read within the call.
#include <cuda.h>  // CUcontext and CUresult only: the driver calls are fetched at run time

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "kernels.h"

namespace slosh {

void set_last_error(const char* message);  // driver.cu: text returned by slosh_last_error_string

namespace {

constexpr uint32_t kMaxParticles = SLOSH_STATIC_SORT_MAX_PARTICLES;
constexpr uint32_t kMaxKeys = SLOSH_STATIC_SORT_MAX_KEYS;
constexpr size_t kAlignWords = 64;  // 256-byte sub-buffers
constexpr size_t round_up(size_t w) { return (w + kAlignWords - 1) / kAlignWords * kAlignWords; }
// Tile histogram: 256 digits x one 4096-particle tile; scan block sums: one per 4096 scanned words.
constexpr size_t kTileHistWords = round_up(256 * ((size_t(kMaxParticles) + 4095) / 4096));
constexpr size_t kScanTmpWords = round_up(((kTileHistWords > kMaxKeys ? kTileHistWords : kMaxKeys) + 4095) / 4096 + 1);
constexpr size_t kParticleWords = round_up(kMaxParticles);
constexpr size_t kKeyWords = round_up(kMaxKeys);
// keys[2], vals[2], perm | counts, offsets | tile histogram | scan sums | live count
constexpr size_t kScratchWords = 5 * kParticleWords + 2 * kKeyWords + kTileHistWords + kScanTmpWords + kAlignWords;

static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

// Scratch addresses per CUDA context, keyed by the context's process-unique ID (IDs are never reused, so an
// entry can go stale only by its context being destroyed, and then no call can run in it again).
struct ScratchEntry {
    unsigned long long context_id;
    uint32_t* ptr;
};
constexpr size_t kMaxCachedContexts = 64;
std::mutex g_setup_mutex;
ScratchEntry g_scratch_cache[kMaxCachedContexts] = {};
size_t g_scratch_entries = 0, g_scratch_next = 0;  // filled entries; next slot to overwrite when full

using CtxGetCurrentFn = CUresult(CUDAAPI*)(CUcontext*);
using CtxGetIdFn = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// ID of the context current on this thread, or 0 when none is current. Call with g_setup_mutex held.
cudaError_t current_context_id(unsigned long long* id) {
    *id = 0;
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e != cudaSuccess) return e;
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1) return cudaErrorSymbolNotFound;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    if (!ctx) return cudaSuccess;
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

// Address of g_sort_scratch in the current context, resolved once per context.
cudaError_t scratch_in_current_context(uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = 0;
    cudaError_t e = current_context_id(&id);
    if (e != cudaSuccess) return e;
    void* p = nullptr;
    if (id == 0) {
        // No context is current yet: resolving the symbol makes the current device's primary context current.
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
        e = current_context_id(&id);
        if (e != cudaSuccess) return e;
        if (id == 0) return cudaErrorDeviceUninitialized;
    }
    for (size_t k = 0; k < g_scratch_entries; ++k)
        if (g_scratch_cache[k].context_id == id) {
            *out = g_scratch_cache[k].ptr;
            return cudaSuccess;
        }
    if (!p) {
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
    }
    const size_t k = g_scratch_entries < kMaxCachedContexts ? g_scratch_entries++ : (g_scratch_next++ % kMaxCachedContexts);
    g_scratch_cache[k] = ScratchEntry{id, static_cast<uint32_t*>(p)};
    *out = g_scratch_cache[k].ptr;
    return cudaSuccess;
}

// True when p is device (or managed) memory that kernels on `device` can address.
bool device_addressable(const void* p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

slosh_status fail(slosh_status code, const std::string& message) {
    set_last_error(message.c_str());
    return code;
}

}  // namespace
}  // namespace slosh

using namespace slosh;

SLOSH_API slosh_status slosh_sort_particles_static(const slosh_particle_t* particles_in, slosh_particle_t* particles_out,
                                                   uint32_t count, const int32_t grid_dim[3], float cell_size,
                                                   uint32_t* perm_out, uint32_t* key_offsets_out, uint32_t* live_count_out,
                                                   void* cuda_stream) {
    const char* fn = "slosh_sort_particles_static: ";
    if (!grid_dim || grid_dim[0] <= 0 || grid_dim[1] <= 0 || grid_dim[2] <= 0)
        return fail(SLOSH_ERR_INVALID_ARG, std::string(fn) + "grid_dim must hold three positive extents");
    if (!(cell_size > 0.0f) || !std::isfinite(cell_size))
        return fail(SLOSH_ERR_INVALID_ARG, std::string(fn) + "cell_size must be positive and finite");
    if (count > kMaxParticles)
        return fail(SLOSH_ERR_CAPACITY, std::string(fn) + "count " + std::to_string(count) +
                                            " exceeds the static scratch maximum of " + std::to_string(kMaxParticles) +
                                            " particles; use a context (slosh_sort_particles) for larger arrays");
    const int3 grid = make_int3(grid_dim[0], grid_dim[1], grid_dim[2]);
    const int3 sdim = sort_brick_dim(grid);
    const uint64_t keys64 = uint64_t(sdim.x) * uint64_t(sdim.y) * uint64_t(sdim.z) + 1u;
    if (keys64 > kMaxKeys)
        return fail(SLOSH_ERR_CAPACITY, std::string(fn) + "the grid needs " + std::to_string(keys64) +
                                            " sort keys, above the static scratch maximum of " + std::to_string(kMaxKeys));
    const uint32_t num_keys = uint32_t(keys64);
    if (count > 0 && (!particles_in || !particles_out))
        return fail(SLOSH_ERR_INVALID_ARG, std::string(fn) + "particles_in and particles_out are required");
    if (count > 0 && particles_in == particles_out)
        return fail(SLOSH_ERR_INVALID_ARG, std::string(fn) + "particles_out must not alias particles_in");

    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(e == cudaErrorNoDevice ? SLOSH_ERR_NO_DEVICE : SLOSH_ERR_CUDA, std::string(fn) + cudaGetErrorString(e));
    const void* ptrs[5] = {particles_in, particles_out, perm_out, key_offsets_out, live_count_out};
    const char* names[5] = {"particles_in", "particles_out", "perm_out", "key_offsets_out", "live_count_out"};
    for (int k = 0; k < 5; ++k)
        if (ptrs[k] && !device_addressable(ptrs[k], device))
            return fail(SLOSH_ERR_INVALID_ARG, std::string(fn) + names[k] + " is not device memory of the current device");

    uint32_t* base = nullptr;
    e = scratch_in_current_context(&base);
    if (e != cudaSuccess) return fail(SLOSH_ERR_CUDA, std::string(fn) + "resolving the static scratch: " + cudaGetErrorString(e));

    SortBuffers b{};
    uint32_t* w = base;
    b.keys[0] = w; w += kParticleWords;
    b.keys[1] = w; w += kParticleWords;
    b.vals[0] = w; w += kParticleWords;
    b.vals[1] = w; w += kParticleWords;
    b.perm = perm_out ? perm_out : w; w += kParticleWords;
    b.counts = w; w += kKeyWords;
    b.offsets = key_offsets_out ? key_offsets_out : w; w += kKeyWords;
    b.tile_hist = w; w += kTileHistWords;
    b.scan_tmp = w; w += kScanTmpWords;
    b.particle_count = live_count_out ? live_count_out : w;
    b.tile_hist_capacity = kTileHistWords;
    b.scan_tmp_capacity = kScanTmpWords;
    if (sort_tile_hist_size(count) > kTileHistWords || sort_scan_tmp_size(count, num_keys) > kScanTmpWords)
        return fail(SLOSH_ERR_CAPACITY, std::string(fn) + "internal scratch layout too small");

    // The sort kernels read only the grid extents and the inverse cell size of the device view.
    Dev d{};
    d.grid = grid;
    d.h = cell_size;
    d.inv_h = 1.0f / cell_size;
    launch_sort(d, b, particles_in, particles_out, count, num_keys, sdim, static_cast<cudaStream_t>(cuda_stream));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SLOSH_ERR_CUDA, std::string(fn) + cudaGetErrorString(e));
    return SLOSH_OK;
}
