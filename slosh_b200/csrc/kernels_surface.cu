// Headless liquid surface from the particles (sm_100a): density splat, field resolve and surface nets,
// written into device buffers (no window, swapchain or graphics API).
//
// Reference: PLUG/Shaders/Private/SloshSurface.usf -- DensitySplatCS (:54-100), FieldResolveCS (:109-149),
// SampleField/FieldGradient (:154-165), SurfaceNetsVerticesCS (:330-399), SurfaceNetsFacesCS (:401-458),
// SurfaceNetsArgsCS (:460-470); ellipsoids from AnisoComputeCS (SloshRender.usf:281-376) in sphere mode
// (AnisoStrength 0: centre = particle position, axes = splat radius along x, y and z); parameters as
// BuildDensityField / FillFieldParameters set them (PLUG/Source/SloshRender/Private/SloshRenderer.cpp:118-170).
//
// Same arithmetic as the reference; deliberate differences, identical in the CPU restatement:
//   * vertices and quads are numbered in cell order (flags, exclusive scan, write), not in the order in which
//     atomic counters hand out slots, so the mesh is deterministic;
//   * the field gradient of a vertex normal samples the f16 field by exact FP32 trilinear interpolation with
//     clamped addressing (the reference uses the texture unit's filter);
//   * normalize(v) is v / sqrt(dot(v, v)); positions are in sim metres (voxel centre v at v + 0.5 voxels).
#include <cuda_fp16.h>

#include "kernels.h"

namespace slosh {

namespace {

constexpr float FIELD_W_FIXED = 1024.0f, FIELD_X_FIXED = 256.0f;
constexpr uint32_t FIELD_MOMENTS = 5u, NO_VERTEX = 0xFFFFFFFFu;
constexpr int SURF_THREADS = 256;

__device__ __forceinline__ uint32_t voxel_index(const SurfaceDev& s, int3 v) { return uint32_t(v.x + s.dim.x * (v.y + s.dim.y * v.z)); }
__device__ __forceinline__ uint32_t field_brick(const SurfaceDev& s, int3 v) {
    const int bx = min(max(v.x >> 3, 0), s.bdim.x - 1), by = min(max(v.y >> 3, 0), s.bdim.y - 1), bz = min(max(v.z >> 3, 0), s.bdim.z - 1);
    return uint32_t(bx + s.bdim.x * (by + s.bdim.y * bz));
}
__device__ __forceinline__ uint32_t cell_of(const SurfaceDev& s, int3 c) {
    return uint32_t(c.x + (s.dim.x - 1) * (c.y + (s.dim.y - 1) * c.z));
}
__device__ __forceinline__ int3 cell_coord(const SurfaceDev& s, uint32_t i) {
    const uint32_t cx = uint32_t(s.dim.x - 1), cy = uint32_t(s.dim.y - 1);
    return make_int3(int(i % cx), int((i / cx) % cy), int(i / (cx * cy)));
}
__device__ __forceinline__ float field_at(const SurfaceDev& s, int3 v) {
    return __half2float(__ushort_as_half(s.field[voxel_index(s, v)]));
}
__device__ __forceinline__ float dot3f(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// ---- DensitySplatCS ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(SURF_THREADS) k_density_splat(SurfaceDev s, const slosh_particle_t* __restrict__ particles, uint32_t n) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(reinterpret_cast<const float4*>(particles + i));
    if (is_dead_age(a.w)) return;  // a removed particle's ellipsoid is all zeros: skipped
    const float r = s.splat_radius;
    const float3 axis[3] = {make_float3(r, 0.0f, 0.0f), make_float3(0.0f, r, 0.0f), make_float3(0.0f, 0.0f, r)};
    const float k = s.support * s.inv_voxel;
    const float3 c = make_float3(a.x * s.inv_voxel, a.y * s.inv_voxel, a.z * s.inv_voxel);
    float3 w[3];
    float amax = 0.0f;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float3 u = make_float3(axis[q].x * k, axis[q].y * k, axis[q].z * k);
        const float aa = fmaxf(dot3f(u, u), 1e-8f);
        w[q] = make_float3(u.x / aa, u.y / aa, u.z / aa);
        amax = q == 0 ? aa : fmaxf(amax, aa);
    }
    const float rr = fminf(sqrtf(amax), s.max_footprint);
    const int3 lo = make_int3(max(int(floorf(c.x - rr - 0.5f)), 0), max(int(floorf(c.y - rr - 0.5f)), 0), max(int(floorf(c.z - rr - 0.5f)), 0));
    const int3 hi = make_int3(min(int(ceilf(c.x + rr - 0.5f)), s.dim.x - 1), min(int(ceilf(c.y + rr - 0.5f)), s.dim.y - 1),
                              min(int(ceilf(c.z + rr - 0.5f)), s.dim.z - 1));
    for (int z = lo.z; z <= hi.z; ++z)
        for (int y = lo.y; y <= hi.y; ++y)
            for (int x = lo.x; x <= hi.x; ++x) {
                const float3 d = make_float3((float(x) + 0.5f) - c.x, (float(y) + 0.5f) - c.y, (float(z) + 0.5f) - c.z);
                const float3 qv = make_float3(dot3f(d, w[0]), dot3f(d, w[1]), dot3f(d, w[2]));
                const float q2 = dot3f(qv, qv);
                if (q2 < 1.0f) {
                    float wk = 1.0f - q2;
                    wk = wk * wk * wk;
                    int32_t* acc = s.accum + voxel_index(s, make_int3(x, y, z)) * FIELD_MOMENTS;
                    atomicAdd(acc + 0, __float2int_rz(wk * FIELD_W_FIXED + 0.5f));
                    atomicAdd(acc + 1, __float2int_rn(-d.x * wk * FIELD_X_FIXED));
                    atomicAdd(acc + 2, __float2int_rn(-d.y * wk * FIELD_X_FIXED));
                    atomicAdd(acc + 3, __float2int_rn(-d.z * wk * FIELD_X_FIXED));
                    atomicAdd(acc + 4, __float2int_rn(s.radius_voxels * wk * FIELD_X_FIXED));
                }
            }
}

// ---- FieldResolveCS: fixed point -> f16 field (Zhu & Bridson surface) + dilated brick occupancy ---------------
__global__ void __launch_bounds__(SURF_THREADS) k_field_resolve(SurfaceDev s) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    const uint32_t nv = uint32_t(s.dim.x) * uint32_t(s.dim.y) * uint32_t(s.dim.z);
    if (i >= nv) return;
    const int3 v = make_int3(int(i % uint32_t(s.dim.x)), int((i / uint32_t(s.dim.x)) % uint32_t(s.dim.y)), int(i / uint32_t(s.dim.x * s.dim.y)));
    const int32_t* acc = s.accum + i * FIELD_MOMENTS;
    const float w = float(acc[0]) / FIELD_W_FIXED;
    float f = 0.0f;
    if (w > 1e-3f) {
        const float den = FIELD_X_FIXED * w;
        const float3 mo = make_float3(float(acc[1]) / den, float(acc[2]) / den, float(acc[3]) / den);
        const float rbar = fmaxf(float(acc[4]) / den, 1e-3f);
        const float phi = sqrtf(dot3f(mo, mo)) - rbar;
        f = saturatef(0.5f - 0.5f * phi / rbar);
    }
    s.field[i] = __half_as_ushort(__float2half_rn(f));
    if (f <= 0.0f) return;
    const int3 ib = make_int3(v.x & 7, v.y & 7, v.z & 7);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int3 o = make_int3((k & 1) * 2 - 1, ((k >> 1) & 1) * 2 - 1, (k >> 2) * 2 - 1);
        const int3 nb = make_int3(v.x + o.x * int(ib.x == (o.x < 0 ? 0 : 7)), v.y + o.y * int(ib.y == (o.y < 0 ? 0 : 7)),
                                  v.z + o.z * int(ib.z == (o.z < 0 ? 0 : 7)));
        if (nb.x >= 0 && nb.y >= 0 && nb.z >= 0 && nb.x < s.dim.x && nb.y < s.dim.y && nb.z < s.dim.z) atomicOr(s.bricks + field_brick(s, nb), 1u);
    }
}

// The 8 corner values of a cell and their inside mask (corner k at c + (k & 1, (k >> 1) & 1, k >> 2)).
__device__ __forceinline__ uint32_t cell_corners(const SurfaceDev& s, int3 c, float fc[8]) {
    uint32_t mask = 0u;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        fc[k] = field_at(s, make_int3(c.x + (k & 1), c.y + ((k >> 1) & 1), c.z + (k >> 2)));
        mask |= (fc[k] >= s.iso ? 1u : 0u) << k;
    }
    return mask;
}

// ---- SurfaceNetsVerticesCS, split: flags -> scan -> vertices in cell order -----------------------------------
__global__ void __launch_bounds__(SURF_THREADS) k_sn_vertex_flags(SurfaceDev s, uint32_t ncells) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    if (i >= ncells) return;
    const int3 c = cell_coord(s, i);
    uint32_t flag = 0u;
    if (s.bricks[field_brick(s, c)] != 0u) {
        float fc[8];
        const uint32_t mask = cell_corners(s, c, fc);
        flag = (mask != 0u && mask != 0xFFu) ? 1u : 0u;
    }
    s.vflag[i] = flag;
}

// Exact trilinear sample of the f16 field at Pv (voxel units; voxel v's centre at v + 0.5), clamped edges.
__device__ float sample_field(const SurfaceDev& s, float3 pv) {
    const float x = pv.x - 0.5f, y = pv.y - 0.5f, z = pv.z - 0.5f;
    const float fx0 = floorf(x), fy0 = floorf(y), fz0 = floorf(z);
    const float tx = x - fx0, ty = y - fy0, tz = z - fz0;
    const int x0 = int(fx0), y0 = int(fy0), z0 = int(fz0);
    const int xs[2] = {min(max(x0, 0), s.dim.x - 1), min(max(x0 + 1, 0), s.dim.x - 1)};
    const int ys[2] = {min(max(y0, 0), s.dim.y - 1), min(max(y0 + 1, 0), s.dim.y - 1)};
    const int zs[2] = {min(max(z0, 0), s.dim.z - 1), min(max(z0 + 1, 0), s.dim.z - 1)};
    float cz[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        float cy[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float a = field_at(s, make_int3(xs[0], ys[j], zs[k])), b = field_at(s, make_int3(xs[1], ys[j], zs[k]));
            cy[j] = a + tx * (b - a);
        }
        cz[k] = cy[0] + ty * (cy[1] - cy[0]);
    }
    return cz[0] + tz * (cz[1] - cz[0]);
}
__device__ __forceinline__ float3 normalize_div(float3 v) {
    const float l = sqrtf(dot3f(v, v));
    return make_float3(v.x / l, v.y / l, v.z / l);
}

__global__ void __launch_bounds__(SURF_THREADS) k_sn_vertices(SurfaceDev s, uint32_t ncells) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    if (i >= ncells) return;
    uint32_t vi = s.vflag[i] ? s.vbase[i] : NO_VERTEX;
    if (vi != NO_VERTEX && vi >= s.max_vertices) vi = NO_VERTEX;
    s.cell_vertex[i] = vi;
    if (vi == NO_VERTEX) return;
    const int3 c = cell_coord(s, i);
    float fc[8];
    const uint32_t mask = cell_corners(s, c, fc);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, count = 0.0f;
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int bit = 1; bit <= 4; bit <<= 1) {
            if (a & bit) continue;
            const int b = a | bit;
            if (((mask >> a) & 1u) == ((mask >> b) & 1u)) continue;
            const float t = saturatef((s.iso - fc[a]) / (fc[b] - fc[a]));
            // lerp between corners whose coordinates are 0 or 1: the moving coordinate is t or 1 - t
            const float px = (a & 1) == (b & 1) ? float(a & 1) : ((b & 1) ? t : 1.0f - t);
            const float py = ((a >> 1) & 1) == ((b >> 1) & 1) ? float((a >> 1) & 1) : (((b >> 1) & 1) ? t : 1.0f - t);
            const float pz = (a >> 2) == (b >> 2) ? float(a >> 2) : ((b >> 2) ? t : 1.0f - t);
            sx = sx + px;
            sy = sy + py;
            sz = sz + pz;
            count = count + 1.0f;
        }
    const float3 pv = make_float3((float(c.x) + 0.5f) + sx / count, (float(c.y) + 0.5f) + sy / count, (float(c.z) + 0.5f) + sz / count);
    s.positions[3u * vi + 0u] = pv.x * s.voxel;
    s.positions[3u * vi + 1u] = pv.y * s.voxel;
    s.positions[3u * vi + 2u] = pv.z * s.voxel;
    const float3 g = make_float3(sample_field(s, make_float3(pv.x + 1.0f, pv.y, pv.z)) - sample_field(s, make_float3(pv.x - 1.0f, pv.y, pv.z)),
                                 sample_field(s, make_float3(pv.x, pv.y + 1.0f, pv.z)) - sample_field(s, make_float3(pv.x, pv.y - 1.0f, pv.z)),
                                 sample_field(s, make_float3(pv.x, pv.y, pv.z + 1.0f)) - sample_field(s, make_float3(pv.x, pv.y, pv.z - 1.0f)));
    float3 nrm = make_float3(0.0f, 0.0f, 1.0f);
    if (sqrtf(dot3f(g, g)) > 1e-8f) {
        const float3 ng = normalize_div(g);
        nrm = make_float3(-ng.x, -ng.y, -ng.z);
    }
    const float3 ref = fabsf(nrm.z) < 0.9f ? make_float3(0.0f, 0.0f, 1.0f) : make_float3(1.0f, 0.0f, 0.0f);
    const float3 tx = normalize_div(cross3(nrm, ref));
    s.normals[3u * vi + 0u] = nrm.x;
    s.normals[3u * vi + 1u] = nrm.y;
    s.normals[3u * vi + 2u] = nrm.z;
    s.tangents[3u * vi + 0u] = tx.x;
    s.tangents[3u * vi + 1u] = tx.y;
    s.tangents[3u * vi + 2u] = tx.z;
}

// ---- SurfaceNetsFacesCS, split: quad counts -> scan -> quads in cell order ------------------------------------
// Quads of cell c: for each axis whose edge from voxel c to c + e crosses the level, the four cells around
// the edge (c, c - eu, c - eu - ev, c - ev) when all exist and carry a vertex. emit(axis, in0, v00, v10, v11, v01).
template <class Emit>
__device__ __forceinline__ void cell_quads(const SurfaceDev& s, int3 c, Emit emit) {
    if (s.bricks[field_brick(s, c)] == 0u) return;
    const bool in0 = field_at(s, c) >= s.iso;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int3 e = make_int3(axis == 0, axis == 1, axis == 2);
        const bool in1 = field_at(s, make_int3(c.x + e.x, c.y + e.y, c.z + e.z)) >= s.iso;
        if (in0 == in1) continue;
        const int3 eu = make_int3(axis == 2, axis == 0, axis == 1), ev = make_int3(axis == 1, axis == 2, axis == 0);
        const int3 c10 = make_int3(c.x - eu.x, c.y - eu.y, c.z - eu.z);
        const int3 c11 = make_int3(c.x - eu.x - ev.x, c.y - eu.y - ev.y, c.z - eu.z - ev.z);
        const int3 c01 = make_int3(c.x - ev.x, c.y - ev.y, c.z - ev.z);
        if (c11.x < 0 || c11.y < 0 || c11.z < 0) continue;
        const uint32_t v00 = s.cell_vertex[cell_of(s, c)], v10 = s.cell_vertex[cell_of(s, c10)];
        const uint32_t v11 = s.cell_vertex[cell_of(s, c11)], v01 = s.cell_vertex[cell_of(s, c01)];
        if (v00 == NO_VERTEX || v10 == NO_VERTEX || v11 == NO_VERTEX || v01 == NO_VERTEX) continue;
        emit(in0, v00, v10, v11, v01);
    }
}
__global__ void __launch_bounds__(SURF_THREADS) k_sn_quad_counts(SurfaceDev s, uint32_t ncells) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    if (i >= ncells) return;
    uint32_t count = 0u;
    cell_quads(s, cell_coord(s, i), [&](bool, uint32_t, uint32_t, uint32_t, uint32_t) { ++count; });
    s.qflag[i] = count;
}
__global__ void __launch_bounds__(SURF_THREADS) k_sn_faces(SurfaceDev s, uint32_t ncells) {
    const uint32_t i = blockIdx.x * SURF_THREADS + threadIdx.x;
    if (i >= ncells) return;
    uint32_t q = s.qbase[i];
    cell_quads(s, cell_coord(s, i), [&](bool in0, uint32_t v00, uint32_t v10, uint32_t v11, uint32_t v01) {
        const uint32_t base = 6u * q++;
        if (base + 6u > s.max_indices) return;
        uint32_t* o = s.indices + base;
        // winding faces away from the inside voxel
        if (in0) { o[0] = v00; o[1] = v11; o[2] = v10; o[3] = v00; o[4] = v01; o[5] = v11; }
        else { o[0] = v00; o[1] = v10; o[2] = v11; o[3] = v00; o[4] = v11; o[5] = v01; }
    });
}
// Counters: [0] vertices requested, [1] indices requested (SurfaceNetsArgsCS clamps and rounds on the host).
__global__ void k_sn_totals(SurfaceDev s, uint32_t ncells) {
    s.counters[0] = s.vbase[ncells - 1u] + s.vflag[ncells - 1u];
    s.counters[1] = 6u * (s.qbase[ncells - 1u] + s.qflag[ncells - 1u]);
}

int blocks_of(uint64_t n) { return int((n + SURF_THREADS - 1) / SURF_THREADS); }

}  // namespace

int launch_surface(const SurfaceDev& s, const slosh_particle_t* particles, uint32_t n, bool mesh, cudaStream_t st) {
    const uint64_t nv = uint64_t(s.dim.x) * uint64_t(s.dim.y) * uint64_t(s.dim.z);
    const uint64_t nb = uint64_t(s.bdim.x) * uint64_t(s.bdim.y) * uint64_t(s.bdim.z);
    int launches = 0;
    cudaMemsetAsync(s.accum, 0, nv * FIELD_MOMENTS * 4, st);
    cudaMemsetAsync(s.bricks, 0, nb * 4, st);
    cudaMemsetAsync(s.counters, 0, 8, st);
    if (n > 0) {
        k_density_splat<<<blocks_of(n), SURF_THREADS, 0, st>>>(s, particles, n);
        ++launches;
    }
    k_field_resolve<<<blocks_of(nv), SURF_THREADS, 0, st>>>(s);
    ++launches;
    if (!mesh) return launches;
    const uint32_t nc = uint32_t(s.dim.x - 1) * uint32_t(s.dim.y - 1) * uint32_t(s.dim.z - 1);
    if (nc == 0) return launches;
    k_sn_vertex_flags<<<blocks_of(nc), SURF_THREADS, 0, st>>>(s, nc);
    launches += 1 + launch_exclusive_scan(s.vflag, s.vbase, nc, s.scan_tmp, st);
    k_sn_vertices<<<blocks_of(nc), SURF_THREADS, 0, st>>>(s, nc);
    k_sn_quad_counts<<<blocks_of(nc), SURF_THREADS, 0, st>>>(s, nc);
    launches += 2 + launch_exclusive_scan(s.qflag, s.qbase, nc, s.scan_tmp, st);
    k_sn_faces<<<blocks_of(nc), SURF_THREADS, 0, st>>>(s, nc);
    k_sn_totals<<<1, 1, 0, st>>>(s, nc);
    return launches + 2;
}

}  // namespace slosh
