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

// The weight-gradient kernel's CTAs: `heavy` per layer of W2..W4, `l0` for
// W1 and b1, `l4` for W5 and b5, each job a contiguous range of batch tiles.
struct DwJobs {
    uint32_t heavy, l0, l4;
    __host__ __device__ uint32_t total() const { return 3 * heavy + l0 + l4; }
};

// Device-side position of a training run whose steps are replayed from a
// CUDA graph (mgk_surrogate_train): the kernels read where they are from
// here instead of from their arguments.
struct TrainCounters {
    uint32_t step;   // global step: index into the table of Adam constants
    uint32_t done;   // blocks of the Adam kernel finished in this step (the last one advances)
    uint32_t batch;  // batch within the epoch
    uint32_t epoch;  // epochs begun
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
// Adam on the n FP32 parameters; the new values in BF16 into `copy` and,
// where given, into the forward and transposed weight images.
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, __nv_bfloat16* copy, void* img, void* img_t,
                        int n, AdamStep a, cudaStream_t st);
// The same with the constants of step ctr->step from `table`; the last block
// to finish advances ctr->step and ctr->batch.
// With `part` non-null the gradient is summed from the weight-gradient
// partials (mlp_dw_source) instead of read from g.  pdl (here and in the
// tensor-core launchers): launched as a programmatic dependent of the
// previous kernel in the stream, its set-up overlapping that kernel's tail.
cudaError_t launch_adam_counted(float* p, const float* g, const float* part, const DwJobs& jobs, float* m, float* v,
                                __nv_bfloat16* copy, void* img, void* img_t, int n, const AdamStep* table,
                                TrainCounters* ctr, cudaStream_t st, bool pdl = false);
// Begins an epoch of a counted run: ctr->batch = 0, ++ctr->epoch, and the
// epoch's order perm[0, n) from keys[ctr->epoch - 1].
cudaError_t launch_epoch_begin(uint32_t* perm, uint32_t n, const uint4* keys, TrainCounters* ctr, cudaStream_t st);
cudaError_t launch_gather(const float* feat, const SampleLabel* lab, const uint32_t* perm, int b0, int B,
                          __nv_bfloat16* x0, SampleLabel* blab, cudaStream_t st);
cudaError_t launch_features_bf16(const float* feat, uint32_t n, uint32_t rows, __nv_bfloat16* x0, cudaStream_t st);

// The weight image of the tensor-core kernels (mlp_tc.cu, mlp_train_tc.cu):
// 14 chunks, each stored K-major in the operand layout of the tensor cores.
// Chunk 0 is W1 (256 x 16, 8-row stride 256 B), chunks 1-12 are W2..W4 in
// slices of 64 input columns (256 x 64, 8-row stride 1024 B), chunk 13 is W5
// (16 x 256, 8-row stride 4096 B).  W1..W4 are stored halved (exact in BF16).
constexpr int MLP_IMAGE_CHUNKS = 14;
__host__ __device__ constexpr uint32_t mlp_chunk_offset(int c) {
    return c == 0 ? 0u : (c <= 12 ? 8192u + uint32_t(c - 1) * 32768u : 8192u + 12u * 32768u);
}
__host__ __device__ constexpr uint32_t mlp_chunk_bytes(int c) { return (c == 0 || c == 13) ? 8192u : 32768u; }
constexpr uint32_t MLP_IMAGE_BYTES = 8192u + 12u * 32768u + 8192u;
// Where parameter i (flat index) sits in the forward image and in the
// transposed image of the backward (mlp_t_image_bytes): byte offsets, ~0u
// where it has none (the biases; W1 in the transposed image).  *halved: the
// images hold it halved (the layers followed by SiLU).
__host__ __device__ inline void mlp_image_offsets(uint32_t i, uint32_t* f, uint32_t* t, bool* halved) {
    *f = *t = ~0u;
    *halved = false;
    int l = 0;
    while (l < MLP_LAYERS && !(i >= mlp_w_off(l) && i < mlp_b_off(l))) ++l;
    if (l == MLP_LAYERS) return;
    auto kmaj = [](uint32_t row, uint32_t k, uint32_t sbo) {
        return (row >> 3) * sbo + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
    };
    const uint32_t e = i - mlp_w_off(l), in_dim = l == 0 ? MLP_IN_PAD : MLP_HID;
    const uint32_t out = e / in_dim, in = e % in_dim;
    *halved = l < 4;
    if (l == 0) {
        *f = kmaj(out, in, 256);
    } else if (l == 4) {
        *f = mlp_chunk_offset(13) + kmaj(out, in, 4096);
        *t = kmaj(in, out, 256);
    } else {
        *f = mlp_chunk_offset(1 + 4 * (l - 1) + int(in / 64)) + kmaj(out, in % 64, 1024);
        *t = mlp_chunk_offset(1 + 4 * (3 - l) + int(out / 64)) + kmaj(in, out % 64, 1024);
    }
}

// Fused tensor-core inference and the training chains (mlp_tc.cu).
size_t mlp_image_bytes();
// The transposed image of the backward chain: W5^T (256 x 16, 8-row stride
// 256 B), then W4^T, W3^T, W2^T in slices of 64 output columns (chunks 1-12
// of the same offsets and shapes), halved like the forward image.
size_t mlp_t_image_bytes();
// Both images from the BF16 weights (img_t may be null).
cudaError_t launch_weight_image(const __nv_bfloat16* wb, void* img, void* img_t, cudaStream_t st);
cudaError_t launch_mlp_infer_tc(const float* feat, uint32_t n, const void* img, const float* params, float* out,
                                uint32_t* status, int sm_count, cudaStream_t st);

// Tensor-core training (chains: mlp_tc.cu; weight gradients: mlp_train_tc.cu)
// on tiled activations: 128-row tiles
// in the operand layout (element (row, col) of tile t at
// t * 256 * C + kmaj(row % 128, col, 16 C) bytes for C columns).
// Forward with stash of Z_1..Z_4 of the batch perm[b0 .. b0 + 128 n_tiles)
// of the sample set (feat [.][7], lab), writing its X0 tiles; with labels
// (lab non-null) also the loss (+= *loss_acc, the batch mean) and dOut tiles;
// out (FP32 [rows][16]) may be null.
// With ctr non-null the batch is batch ctr->batch of the epoch (b0 is added)
// and the loss goes to loss_acc[ctr->epoch - 1].
cudaError_t launch_mlp_fwd_stash_tc(const void* img, const float* params, const float* feat, const uint32_t* perm,
                                    uint32_t b0, void* x0_tiles, void* const* z, float* out, const SampleLabel* lab,
                                    const LossWeights& w, void* dout_tiles, float* loss_acc, uint32_t n_tiles,
                                    const TrainCounters* ctr, uint32_t* status, int sm_count, cudaStream_t st,
                                    bool pdl = false);
// The forward (as above, with labels) and the input-gradient chain in one
// kernel: each tile's backward runs right after its forward, dOut handed
// over in shared memory (and written to dout_tiles for the weight gradients).
cudaError_t launch_mlp_fwd_bwd_tc(const void* img, const void* img_t, const float* params, const float* feat,
                                  const uint32_t* perm, uint32_t b0, void* x0_tiles, void* const* z, void* const* dz,
                                  const SampleLabel* lab, const LossWeights& w, void* dout_tiles, float* loss_acc,
                                  uint32_t n_tiles, const TrainCounters* ctr, uint32_t* status, int sm_count,
                                  cudaStream_t st, bool pdl = false);
cudaError_t launch_mlp_bwd_dx_tc(const void* img_t, const void* dout_tiles, void* const* z, void* const* dz,
                                 uint32_t n_tiles, uint32_t* status, int sm_count, cudaStream_t st, bool pdl = false);
DwJobs mlp_dw_jobs(uint32_t n_tiles, int sm_count);
// A job's partial sums: the 256 x 256 (or 256 x 16) weight-gradient block
// row-major, then the 256 (or 16) bias-gradient sums.
constexpr uint32_t MLP_DW_PART = MLP_HID * MLP_HID + MLP_HID;
// Where the gradient of parameter i is in the partials: the sum over jobs
// j0 .. j0 + nj - 1 of part[j * MLP_DW_PART + src].
__host__ __device__ inline void mlp_dw_source(uint32_t i, const DwJobs& jobs, uint32_t* j0, uint32_t* nj,
                                              uint32_t* src) {
    const uint32_t j_l0 = 3 * jobs.heavy, j_l4 = j_l0 + jobs.l0;  // first job of W1 / b1 and of W5 / b5
    int l = 0;
    while (l < MLP_LAYERS - 1 && i >= mlp_w_off(l + 1)) ++l;
    const bool bias = i >= mlp_b_off(l);
    const uint32_t e = bias ? i - mlp_b_off(l) : i - mlp_w_off(l);
    *j0 = l == 0 ? j_l0 : (l == 4 ? j_l4 : (l - 1) * jobs.heavy);
    *nj = l == 0 ? jobs.l0 : (l == 4 ? jobs.l4 : jobs.heavy);
    if (bias) *src = MLP_HID * MLP_HID + e;
    else if (l == 4) *src = (e % MLP_HID) * MLP_OUT_PAD + e / MLP_HID;  // dW5 [16][256] from dW5^T [256][16]
    else *src = e;
}
size_t mlp_dw_partial_floats(uint32_t jobs);
// Weight and bias gradients (all of W1..W5, b1..b5) from dZ_1..dZ_4, Z_1..Z_4,
// X0 and dOut: the jobs' partials, and (reduce) their sums into grad.
cudaError_t launch_mlp_dw_tc(void* const* dz, void* const* z, const void* x0_tiles, const void* dout_tiles,
                             float* part, float* grad, uint32_t n_tiles, const DwJobs& jobs, uint32_t* status,
                             cudaStream_t st, bool reduce = true, bool pdl = false);
// The sample-set order of one epoch (a keyed permutation of [0, n)) on the
// device (mlp.cu).
cudaError_t launch_epoch_perm(uint32_t* perm, uint32_t n, const uint32_t key[4], cudaStream_t st);

}  // namespace mgk
