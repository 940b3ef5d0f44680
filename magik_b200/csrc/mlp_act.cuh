// Shared pieces of the surrogate's tensor-core kernels (mlp_tc.cu,
// mlp_train_tc.cu): the tile geometry of the activations and the activation
// functions on FP32 and BF16 pairs.
//
// SiLU and its derivative come from tanh.approx:
//   silu(z) = u + u tanh(u) and sigmoid(z) = (1 + tanh(u)) / 2, u = z / 2;
//   silu'(z) = s (1 + z (1 - s)).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "mlp.h"
#include "tc_sm100.cuh"

namespace mgk {
namespace act {

constexpr int TM = 128;                           // rows per tile
constexpr uint32_t A_BYTES = TM * MLP_HID * 2;    // 64 KB: a 256-column tile
constexpr uint32_t A_SBO = 4096;                  // its 8-row group stride
constexpr uint32_t X_TILE = TM * MLP_IN_PAD * 2;  // 4 KB: a 16-column tile
constexpr uint32_t X_SBO = 256;                   // its 8-row group stride

__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu_f(float z) {
    const float u = 0.5f * z;
    return __fmaf_rn(u, tanh_approx(u), u);
}
__device__ __forceinline__ float silu_grad_f(float z) {
    const float s = __fmaf_rn(0.5f, tanh_approx(0.5f * z), 0.5f);
    return s * __fmaf_rn(z, 1.0f - s, 1.0f);
}
// the two BF16 halves of a word (low half first) as floats
__device__ __forceinline__ float2 unpack_bf16(uint32_t v) {
    return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xFFFF0000u));
}
// silu of both BF16 halves of a word, rounded back to BF16
__device__ __forceinline__ uint32_t silu_bf16x2(uint32_t v) {
    const float2 u = __fmul2_rn(make_float2(0.5f, 0.5f), unpack_bf16(v));
    const float2 h = __ffma2_rn(u, make_float2(tanh_approx(u.x), tanh_approx(u.y)), u);
    return tc::pack_bf16(h.x, h.y);
}
__device__ __forceinline__ void add_bf16x2(float& a, float& b, uint32_t v) {
    const float2 f = unpack_bf16(v);
    a += f.x;
    b += f.y;
}
// silu of a pair given u = z / 2, in BF16x2: u (1 + tanh u), u rounded to
// BF16 first (one tanh.approx.bf16x2 and one fma.rn.bf16x2 per pair)
__device__ __forceinline__ uint32_t silu_half_pair(float u0, float u1) {
    const uint32_t u = tc::pack_bf16(u0, u1);
    uint32_t t, h;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(u));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(u), "r"(t));
    return h;
}

}  // namespace act
}  // namespace mgk
