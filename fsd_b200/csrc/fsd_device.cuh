// Device helpers shared by the kernels: periodic box arithmetic, table
// interpolation and warp/group reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fsd_internal.h"

namespace fsd {

// Minimum image with an xy tilt, rint based (HOOMD BoxDim::minImage, device path).
__device__ __forceinline__ float3 min_image(float3 w, const Box& b) {
    float img = rintf(w.z * (1.0f / b.Lz));
    w.z -= b.Lz * img;
    img = rintf(w.y * (1.0f / b.Ly));
    w.x -= b.Ly * b.xy * img;
    w.y -= b.Ly * img;
    w.x -= b.Lx * rintf(w.x * (1.0f / b.Lx));
    return w;
}

// Pair separation j - i (or i - j) and its squared length evaluated without
// fused multiply-adds, so that separations and gaps are the correctly rounded
// single-precision values of the reference's arithmetic (minImage, dot,
// sqrtf).  Near contact the lubrication functions are steep in the gap, so
// this rounding is part of the result.
__device__ __forceinline__ float3 min_image_rn(float3 w, const Box& b) {
    float img = rintf(__fmul_rn(w.z, 1.0f / b.Lz));
    w.z = __fsub_rn(w.z, __fmul_rn(b.Lz, img));
    img = rintf(__fmul_rn(w.y, 1.0f / b.Ly));
    w.x = __fsub_rn(w.x, __fmul_rn(__fmul_rn(b.Ly, b.xy), img));
    w.y = __fsub_rn(w.y, __fmul_rn(b.Ly, img));
    w.x = __fsub_rn(w.x, __fmul_rn(b.Lx, rintf(__fmul_rn(w.x, 1.0f / b.Lx))));
    return w;
}

__device__ __forceinline__ float dist2_rn(float3 r) {
    return __fadd_rn(__fadd_rn(__fmul_rn(r.x, r.x), __fmul_rn(r.y, r.y)), __fmul_rn(r.z, r.z));
}

// Fractional coordinates in [0,1) of the sheared box (HOOMD BoxDim::makeFraction).
__device__ __forceinline__ float3 make_fraction(float3 v, const Box& b) {
    float3 d = make_float3(v.x + b.Lx / 2, v.y + b.Ly / 2, v.z + b.Lz / 2);
    d.x -= b.xy * v.y;
    return make_float3(d.x / b.Lx, d.y / b.Ly, d.z / b.Lz);
}

// Wrap a position back into the box, updating its image (HOOMD BoxDim::wrap).
__device__ __forceinline__ void wrap_position(float3& w, int3& img, const Box& b) {
    const float tilt_x = b.xy * w.y;
    if (w.x >= b.Lx / 2 + tilt_x) { w.x -= b.Lx; img.x++; }
    else if (w.x < -b.Lx / 2 + tilt_x) { w.x += b.Lx; img.x--; }
    if (w.y >= b.Ly / 2) { w.y -= b.Ly; w.x -= b.Ly * b.xy; img.y++; }
    else if (w.y < -b.Ly / 2) { w.y += b.Ly; w.x += b.Ly * b.xy; img.y--; }
    if (w.z >= b.Lz / 2) { w.z -= b.Lz; img.z++; }
    else if (w.z < -b.Lz / 2) { w.z += b.Lz; img.z--; }
}

// Interpolated near-field resistance scalars [first, first+count) of the table
// row bracketing distance r.  Pairs at r <= 2.001 use the regularised row 232
// (Lubrication.cu:172-186).  Beyond the last tabulated gap the index reaches
// row 999 whose values are zero; those pairs contribute nothing, which is what
// the reference's read past the last row yields as well.
template <int COUNT>
__device__ __forceinline__ void res_interp(const ResTable& t, float r, int first, float* out) {
    if ((double)r <= 2.001) {
        const float* v = t.vals + 232 * kResFuncs + first;
#pragma unroll
        for (int c = 0; c < COUNT; ++c) out[c] = __ldg(v + c);
        return;
    }
    const float s = (float)(((double)r - 2.0) / (double)kResMin);
    const int ind = (int)(log10f(s) / kResDr);
    if (ind >= kResRows - 1) {
#pragma unroll
        for (int c = 0; c < COUNT; ++c) out[c] = 0.0f;
        return;
    }
    const float dl = __ldg(t.dist + ind), du = __ldg(t.dist + ind + 1);
    const float fac = (r - dl) / (du - dl);
    const float* lo = t.vals + ind * kResFuncs + first;
    const float* hi = lo + kResFuncs;
#pragma unroll
    for (int c = 0; c < COUNT; ++c) {
        const float a = __ldg(lo + c), b = __ldg(hi + c);
        out[c] = a + (b - a) * fac;
    }
}

// Sum over aligned groups of G lanes (G a power of two <= 32).
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int G>
__device__ __forceinline__ double group_sum_d(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Last-block reduction: the threads that wrote this block's partials have
// fenced them; the block that takes the last ticket sees every block's
// partials and resets the ticket.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Sum of part[0:n] in a fixed order by one warp (same result every run).
__device__ __forceinline__ double warp_sum_parts(const double* part, int n) {
    double s = 0.0;
    for (int b = threadIdx.x & 31; b < n; b += 32) s += __ldcg(part + b);
    return group_sum_d<32>(s);
}

// Block sum of v written (and fenced) to part[blockIdx.x].
__device__ __forceinline__ void block_partial(double v, double* part) {
    __shared__ double sh[32];
    v = group_sum_d<32>(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        t = group_sum_d<32>(t);
        if (threadIdx.x == 0) {
            part[blockIdx.x] = t;
            __threadfence();
        }
    }
}

}  // namespace fsd
