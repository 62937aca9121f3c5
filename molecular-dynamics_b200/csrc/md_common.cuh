// md_common.cuh -- device helpers shared by the tinyMD B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tmd {

constexpr int kWarp = 32;
// list entry = slot << kCodeBits | code; code = (dkx+1) | (dky+1) << 2 | (dkz+1) << 4,
// dk = the neighbour's rebasing cell minus the owner's (mixed form only).
constexpr int kCodeBits = 6;
constexpr uint32_t kCodeMask = (1u << kCodeBits) - 1u;
constexpr int kMaxSlots = 1 << (32 - kCodeBits);

// Neighbour-list layout: quads of four consecutive entries of one atom, atom-fastest.
// Entry k of atom i sits at nl_index(k, i, stride); quad b of atom i is uint4 b * stride + i.
__device__ __forceinline__ size_t nl_index(int k, int i, int stride) {
    return (((size_t)(k >> 2) * stride + i) << 2) + (k & 3);
}

// ---- strict FP64 arithmetic (round-to-nearest, never contracted into FMA) --
// The FP64 form evaluates every expression in the reference's operand order
// with these, which makes it bit-identical to the CPU restatement.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// ((x*x + y*y) + z*z) as utils/utilities.impala:49-50 evaluates it
__device__ __forceinline__ double len2_strict(double x, double y, double z) {
    return dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
}

// ---- packed per-atom integer triplets (10 bits per axis, modulo 1024) -----
__device__ __forceinline__ int pack3(int a, int b, int c) {
    return (a & 1023) | ((b & 1023) << 10) | ((c & 1023) << 20);
}
__device__ __forceinline__ int unpack_axis(int p, int axis) { return (p >> (10 * axis)) & 1023; }
// signed difference of two packed axes, wrapped into [-512, 511]
__device__ __forceinline__ int wrap_diff(int a, int b) { return ((a - b + 512) & 1023) - 512; }

// FP32 copy of a position relative to the centre of its cell in the dyadic
// rebasing grid of spacing h (mixed form); w carries the packed rebasing cell
// (bit pattern of rbk), which the staged force kernel decodes
__device__ __forceinline__ float4 rebased32(const double4& p, int rbk, const double* alo, double h) {
    float4 r;
    r.x = (float)(p.x - (alo[0] + ((double)unpack_axis(rbk, 0) + 0.5) * h));
    r.y = (float)(p.y - (alo[1] + ((double)unpack_axis(rbk, 1) + 0.5) * h));
    r.z = (float)(p.z - (alo[2] + ((double)unpack_axis(rbk, 2) + 0.5) * h));
    r.w = __int_as_float(rbk);
    return r;
}

// ghost code: bits 0-5 last-pass shift (2 bits per axis, value + 1), bits 8-13 total shift
__device__ __forceinline__ int shift_axis(int code, int base, int axis) {
    return ((code >> (base + 2 * axis)) & 3) - 1;
}

// ---- warp / block reductions ---------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// compensated sums (Knuth's two-sum: a + b = s + e exactly), for totals whose
// rounding must stay far below their differences (loss values under central differences)
__device__ __forceinline__ void dd_add(double& s, double& c, double t, double d) {
    const double u = s + t;
    const double bp = u - s;
    c = c + d + ((s - (u - bp)) + (t - bp));
    s = u;
}
__device__ __forceinline__ void warp_sum_dd(double& s, double& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_down_sync(0xffffffffu, s, o);
        const double d = __shfl_down_sync(0xffffffffu, c, o);
        dd_add(s, c, t, d);
    }
}
// block total of (s, c) pairs in thread 0 (scratch: 64 doubles)
__device__ __forceinline__ void block_sum_dd(double& s, double& c, double* scratch) {
    warp_sum_dd(s, c);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        scratch[wid] = s;
        scratch[32 + wid] = c;
    }
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (wid == 0) {
        s = lane < nw ? scratch[lane] : 0.0;
        c = lane < nw ? scratch[32 + lane] : 0.0;
        warp_sum_dd(s, c);
    }
    __syncthreads();
}
__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Sums `v` over the block in a fixed order (warp tree, then warp 0 over the
// warp partials); the result is valid in thread 0.  `scratch` needs
// blockDim.x / 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? scratch[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace tmd
