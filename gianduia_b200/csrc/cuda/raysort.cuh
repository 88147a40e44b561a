// Ray keys for reordering ray queries (wavefront.cu: each iteration's closest-hit and
// shadow queries; trace.cu: ray batches). A 16-bit key: the origin's cell in an 8 x 8 x 8
// grid over the scene's bounds (Morton order, high 9 bits) and the direction's cube-map
// bin (dominant axis and sign, then 4 x 4 over the other two components; low 7 bits).
// Rays with equal or adjacent keys start in the same region heading the same way, so a
// warp that takes them visits the same nodes. A counting sort over the keys: histogram
// (the caller's key kernel), kRayScan (exclusive prefix sum in place), the caller's
// scatter, kRayClear. Reordering changes which rays share a warp, never a ray's result.
#pragma once
#include "gnd/layout.h"

namespace gnd {

constexpr uint32_t kRayBins = 1u << 16;

__device__ __forceinline__ uint32_t spread3(uint32_t x) { return (x & 1u) | ((x & 2u) << 2) | ((x & 4u) << 4); }

__device__ __forceinline__ uint32_t rayKey(const SceneView& s, V3 o, V3 d) {
    uint32_t c[3];
    const float oc[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)   // fmaxf / fminf map NaN to the bounds
        c[a] = (uint32_t)fminf(fmaxf((oc[a] - s.keyLo[a]) * s.keyScale[a], 0.0f), 7.0f);
    const uint32_t cell = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    uint32_t face;
    float u, v, m;
    if (ax >= ay && ax >= az) { face = d.x < 0.0f; u = d.y; v = d.z; m = ax; }
    else if (ay >= az) { face = 2u + (d.y < 0.0f); u = d.x; v = d.z; m = ay; }
    else { face = 4u + (d.z < 0.0f); u = d.x; v = d.y; m = az; }
    const float inv = m > 0.0f ? 1.0f / m : 0.0f;
    const uint32_t qu = (uint32_t)fminf(fmaxf((u * inv + 1.0f) * 2.0f, 0.0f), 3.0f);
    const uint32_t qv = (uint32_t)fminf(fmaxf((v * inv + 1.0f) * 2.0f, 0.0f), 3.0f);
    return (cell << 7) | (face << 4) | (qu << 2) | qv;
}

namespace {

// Exclusive prefix sum of the histogram in place (one block of 1024 threads, 64 bins each,
// read and written as 16 uint4 so that the loads are issued back to back).
__global__ void __launch_bounds__(1024) kRayScan(uint32_t* bins) {
    __shared__ uint32_t warpSum[32];
    constexpr uint32_t kPer = kRayBins / 1024u;
    static_assert(kPer % 4 == 0, "bins per thread must fill uint4 loads");
    uint4* b4 = reinterpret_cast<uint4*>(bins + threadIdx.x * kPer);
    uint4 v[kPer / 4];
    uint32_t local = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer / 4; ++k) v[k] = b4[k];
#pragma unroll
    for (uint32_t k = 0; k < kPer / 4; ++k) local += (v[k].x + v[k].y) + (v[k].z + v[k].w);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warpSum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        warpSum[lane] = w;
    }
    __syncthreads();
    uint32_t run = x - local + (warp ? warpSum[warp - 1] : 0u);
#pragma unroll
    for (uint32_t k = 0; k < kPer / 4; ++k) {
        uint4 o;
        o.x = run; run += v[k].x;
        o.y = run; run += v[k].y;
        o.z = run; run += v[k].z;
        o.w = run; run += v[k].w;
        b4[k] = o;
    }
}

// Clears the histogram (the scatter leaves each bin at its end offset).
__global__ void kRayClear(uint32_t* bins) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kRayBins; i += gridDim.x * blockDim.x) bins[i] = 0;
}

}  // namespace

}  // namespace gnd
