// Internal interfaces of the surrogate network kernels (mlp.cu) and its
// driver (surrogate.cu).  Not installed.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/mgk.h"

namespace mgk {

// Network shape: 7 -> 256 -> 256 -> 256 -> 256 -> 8, SiLU between layers.
// Inputs are padded to 16 and outputs to 16 for the tensor-core tiles; the
// padding columns of W1 and rows of W5 start at zero and receive zero
// gradients, so they stay zero.
constexpr int MLP_IN = 7, MLP_IN_PAD = 16, MLP_HID = 256, MLP_OUT = 8, MLP_OUT_PAD = 16, MLP_LAYERS = 5;
// Offsets (floats) of the weights ([out][in]) and biases in the flat parameter vector.
__host__ __device__ constexpr uint32_t mlp_w_off(int l) {
    return l == 0 ? 0u : (l == 1 ? 4352u : (l == 2 ? 70144u : (l == 3 ? 135936u : 201728u)));
}
__host__ __device__ constexpr uint32_t mlp_b_off(int l) {
    return l == 0 ? 4096u : (l == 1 ? 69888u : (l == 2 ? 135680u : (l == 3 ? 201472u : 205824u)));
}
constexpr uint32_t MLP_PARAMS = 205840;

enum GemmEpilogue { EPI_FWD_SILU = 0, EPI_FWD_OUT = 1, EPI_DX = 2, EPI_DW = 3 };
enum GemmKind {
    GEMM_FWD_FIRST, GEMM_FWD_HIDDEN, GEMM_FWD_OUT,
    GEMM_DX_FROM_OUT, GEMM_DX_HIDDEN,
    GEMM_DW_HIDDEN, GEMM_DW_FIRST, GEMM_DW_OUT
};

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K, lda, ldb, ldc, k_split;
    const float* bias;            // EPI_FWD_*
    __nv_bfloat16* Z;             // EPI_FWD_SILU: pre-activation
    __nv_bfloat16* H;             // EPI_FWD_SILU: activation; EPI_DX: dZ_prev
    const __nv_bfloat16* Zp;      // EPI_DX: pre-activation of the previous layer
    float* out;                   // EPI_FWD_OUT: outputs; EPI_DW: gradient accumulator
};

// Labels of one training sample: mgk_sample_label (include/mgk.h).
using SampleLabel = mgk_sample_label;

struct LossWeights {
    float cls, r, g, dir, conf;
    float tol_r, tol_g, tol_dir;  // "good prediction" bounds for the confidence target
};

struct AdamStep {
    float lr, b1, b2, eps;
    float c1, c2;     // 1 / (1 - b1^t), 1 / (1 - b2^t)
    float gscale;     // the gradient is grad x gscale (1 / ranks after a sum over ranks)
};

cudaError_t launch_gemm(GemmKind kind, GemmArgs g, cudaStream_t st);
cudaError_t launch_colsum(const __nv_bfloat16* X, int rows, int ld, int cols, float* out, cudaStream_t st);
cudaError_t launch_colsum_f32(const float* X, int rows, int cols, float* out, cudaStream_t st);
cudaError_t launch_loss(const float* out, const SampleLabel* lab, int B, LossWeights w, __nv_bfloat16* dout,
                        float* dout32, float* loss_acc, cudaStream_t st);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, __nv_bfloat16* copy, int n, AdamStep a,
                        cudaStream_t st);
cudaError_t launch_gather(const float* feat, const SampleLabel* lab, const uint32_t* perm, int b0, int B,
                          __nv_bfloat16* x0, SampleLabel* blab, cudaStream_t st);
cudaError_t launch_features_bf16(const float* feat, uint32_t n, uint32_t rows, __nv_bfloat16* x0, cudaStream_t st);

// Fused tensor-core inference (mlp_tc.cu).
size_t mlp_image_bytes();
cudaError_t launch_weight_image(const __nv_bfloat16* wb, void* img, cudaStream_t st);
cudaError_t launch_mlp_infer_tc(const float* feat, uint32_t n, const void* img, const float* params, float* out,
                                uint32_t* status, int sm_count, cudaStream_t st);

}  // namespace mgk
