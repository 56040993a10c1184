// vx_layout.cuh — device storage of symmetric 3x3 blocks.
//
// A symmetric block (xx, yy, zz, xy, xz, yz) of n entries is stored so that a
// thread reads its block with two (FP32) or three (FP64) vector loads and a
// warp's loads are contiguous:
//   FP32: float4[n] (xx, yy, zz, xy) followed by float2[n] (xz, yz)  -> 6n floats
//   FP64: double2[n] (xx, yy), double2[n] (zz, xy), double2[n] (xz, yz) -> 6n doubles
// Per-axis bond stiffness uses one such array per axis. In FP64 the axes sit
// at base + axis * 6n; in FP32 at base + axis * 6 * kstride32(n), n rounded up
// to a multiple of 4, so every axis starts on a 16-byte boundary (a float4
// load at 24 n bytes would be misaligned for odd n).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vx {

// REV stride of the per-axis FP32 stiffness arrays.
__host__ __device__ constexpr uint32_t kstride32(uint32_t n) { return (n + 3u) & ~3u; }

template <typename T>
struct Sym {
    T xx, yy, zz, xy, xz, yz;
};

__device__ __forceinline__ Sym<float> load_sym(const float* __restrict__ base, size_t n, size_t i) {
    float4 a = __ldg(reinterpret_cast<const float4*>(base) + i);
    float2 b = __ldg(reinterpret_cast<const float2*>(base + 4 * n) + i);
    return {a.x, a.y, a.z, a.w, b.x, b.y};
}
__device__ __forceinline__ Sym<double> load_sym(const double* __restrict__ base, size_t n, size_t i) {
    double2 a = __ldg(reinterpret_cast<const double2*>(base) + i);
    double2 b = __ldg(reinterpret_cast<const double2*>(base + 2 * n) + i);
    double2 c = __ldg(reinterpret_cast<const double2*>(base + 4 * n) + i);
    return {a.x, a.y, b.x, b.y, c.x, c.y};
}
__device__ __forceinline__ void store_sym(float* base, size_t n, size_t i, double xx, double yy, double zz,
                                          double xy, double xz, double yz) {
    reinterpret_cast<float4*>(base)[i] = make_float4((float)xx, (float)yy, (float)zz, (float)xy);
    reinterpret_cast<float2*>(base + 4 * n)[i] = make_float2((float)xz, (float)yz);
}
__device__ __forceinline__ void store_sym(double* base, size_t n, size_t i, double xx, double yy, double zz,
                                          double xy, double xz, double yz) {
    reinterpret_cast<double2*>(base)[i] = make_double2(xx, yy);
    reinterpret_cast<double2*>(base + 2 * n)[i] = make_double2(zz, xy);
    reinterpret_cast<double2*>(base + 4 * n)[i] = make_double2(xz, yz);
}

}  // namespace vx
