// Tensor-core kernels of the deflection surrogate (an MLP 7 -> 256^4 -> 8 with
// SiLU activations, BF16 weights and activations, FP32 accumulation).
//
//  k_gemm      C = A * B on BF16 tensor cores (mma.sync m16n8k16, FP32
//              accumulators), operands staged in shared memory with cp.async
//              double buffering and read with ldmatrix (.trans where the operand
//              is stored the other way round), fused epilogues:
//                EPI_FWD_SILU  z = acc + b;  Z = bf16(z);  H = bf16(silu(z))
//                EPI_FWD_OUT   out = acc + b (FP32)
//                EPI_DX        dZ_prev = bf16(acc * silu'(Z_prev))
//                EPI_DW        dW += acc (FP32 atomics; the batch is split over
//                              blockIdx.z)
//  k_colsum    bias gradients
//  k_loss      loss and d(loss)/d(out) of a batch
//  k_adam      Adam update of the FP32 master parameters and the BF16 copies
//  k_gather    batch assembly (features, labels) from a permutation
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.h"
#include "mlp_loss.cuh"
#include "tc_sm100.cuh"

#ifndef MGK_ADAM_BULK_ROWS
#define MGK_ADAM_BULK_ROWS 40u
#endif

namespace mgk {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void ldsm_x4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}


__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// C[M][N] = A[M][K] * B[K][N].
//   A_KMAJ: A is stored [M][K] (row length lda) - else [K][M].
//   B_NK:   B is stored [N][K] (row length ldb) - else [K][N].
// BM x BN tile per CTA, BK per stage, WM x WN warps; M, N and the K range of
// each blockIdx.z are multiples of the tile sizes (checked on the host).
template <bool A_KMAJ, bool B_NK, int EPI, int BM, int BN, int BK, int WM, int WN>
__global__ void __launch_bounds__(WM * WN * 32) k_gemm(GemmArgs g) {
    constexpr int NT_THREADS = WM * WN * 32;
    constexpr int TM = BM / WM, TN = BN / WN;
    constexpr int MT = TM / 16, NT = TN / 8;
    static_assert(TM % 16 == 0 && TN % 16 == 0 && BK % 16 == 0, "tile");
    constexpr int PAD = 8;
    constexpr int A_ROWS = A_KMAJ ? BM : BK, A_COLS = A_KMAJ ? BK : BM;
    constexpr int B_ROWS = B_NK ? BN : BK, B_COLS = B_NK ? BK : BN;
    __shared__ __align__(16) __nv_bfloat16 sA[2][A_ROWS][A_COLS + PAD];
    __shared__ __align__(16) __nv_bfloat16 sB[2][B_ROWS][B_COLS + PAD];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp / WN, wn = warp % WN;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int k_begin = blockIdx.z * g.k_split, k_end = min(g.K, k_begin + g.k_split);
    const __nv_bfloat16* A = g.A;
    const __nv_bfloat16* B = g.B;

    auto load = [&](int stage, int k0) {
        constexpr int A_CH = A_ROWS * A_COLS / 8, B_CH = B_ROWS * B_COLS / 8;
        for (int c = tid; c < A_CH; c += NT_THREADS) {
            int r = c / (A_COLS / 8), c8 = (c % (A_COLS / 8)) * 8;
            const __nv_bfloat16* src = A_KMAJ ? A + size_t(m0 + r) * g.lda + k0 + c8 : A + size_t(k0 + r) * g.lda + m0 + c8;
            cp_async16(&sA[stage][r][c8], src);
        }
        for (int c = tid; c < B_CH; c += NT_THREADS) {
            int r = c / (B_COLS / 8), c8 = (c % (B_COLS / 8)) * 8;
            const __nv_bfloat16* src = B_NK ? B + size_t(n0 + r) * g.ldb + k0 + c8 : B + size_t(k0 + r) * g.ldb + n0 + c8;
            cp_async16(&sB[stage][r][c8], src);
        }
        cp_async_commit();
    };

    float acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

    const int n_k = (k_end - k_begin) / BK;
    if (n_k > 0) load(0, k_begin);
    for (int it = 0; it < n_k; ++it) {
        const int stage = it & 1;
        if (it + 1 < n_k) {
            load(stage ^ 1, k_begin + (it + 1) * BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t af[MT][4];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const int mb = wm * TM + mt * 16;
                const int i = lane & 7, mat = lane >> 3;
                if constexpr (A_KMAJ) {
                    ldsm_x4(af[mt][0], af[mt][1], af[mt][2], af[mt][3],
                            &sA[stage][mb + (lane & 15)][kk + (lane >> 4) * 8]);
                } else {
                    const int k_off = ((mat >> 1) ? 8 : 0) + i, m_off = (mat & 1) ? 8 : 0;
                    ldsm_x4_t(af[mt][0], af[mt][1], af[mt][2], af[mt][3], &sA[stage][kk + k_off][mb + m_off]);
                }
            }
#pragma unroll
            for (int nt = 0; nt < NT; nt += 2) {
                const int nb = wn * TN + nt * 8;
                const int i = lane & 7, mat = lane >> 3;
                uint32_t b0, b1, b2, b3;
                if constexpr (B_NK) {
                    const int n_off = ((mat >> 1) ? 8 : 0) + i, k_off = (mat & 1) ? 8 : 0;
                    ldsm_x4(b0, b1, b2, b3, &sB[stage][nb + n_off][kk + k_off]);
                } else {
                    const int k_off = ((mat & 1) ? 8 : 0) + i, n_off = (mat >> 1) ? 8 : 0;
                    ldsm_x4_t(b0, b1, b2, b3, &sB[stage][kk + k_off][nb + n_off]);
                }
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    mma_bf16(acc[mt][nt], af[mt], b0, b1);
                    mma_bf16(acc[mt][nt + 1], af[mt], b2, b3);
                }
            }
        }
        __syncthreads();
    }

    // ---- epilogue: accumulator (row g / g+8, cols 2t, 2t+1) of each tile
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + wm * TM + mt * 16 + gq + h * 8;
                const int col = n0 + wn * TN + nt * 8 + 2 * tq;
                float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
                if constexpr (EPI == EPI_FWD_SILU) {
                    v0 += g.bias[col];
                    v1 += g.bias[col + 1];
                    const size_t o = size_t(row) * g.ldc + col;
                    if (g.Z) *reinterpret_cast<__nv_bfloat162*>(g.Z + o) = __floats2bfloat162_rn(v0, v1);
                    *reinterpret_cast<__nv_bfloat162*>(g.H + o) = __floats2bfloat162_rn(silu(v0), silu(v1));
                } else if constexpr (EPI == EPI_FWD_OUT) {
                    const size_t o = size_t(row) * g.ldc + col;
                    g.out[o] = v0 + g.bias[col];
                    g.out[o + 1] = v1 + g.bias[col + 1];
                } else if constexpr (EPI == EPI_DX) {
                    const size_t o = size_t(row) * g.ldc + col;
                    const __nv_bfloat162 zp = *reinterpret_cast<const __nv_bfloat162*>(g.Zp + o);
                    const float2 z = __bfloat1622float2(zp);
                    *reinterpret_cast<__nv_bfloat162*>(g.H + o) =
                        __floats2bfloat162_rn(v0 * silu_grad(z.x), v1 * silu_grad(z.y));
                } else {  // EPI_DW
                    atomicAdd(&g.out[size_t(row) * g.ldc + col], v0);
                    atomicAdd(&g.out[size_t(row) * g.ldc + col + 1], v1);
                }
            }
}

template <bool A_KMAJ, bool B_NK, int EPI, int BM, int BN, int BK, int WM, int WN>
static cudaError_t gemm_t(const GemmArgs& g, int splits, cudaStream_t st) {
    if (g.M % BM || g.N % BN || g.k_split % BK || g.K % BK) return cudaErrorInvalidValue;
    dim3 grid(g.N / BN, g.M / BM, splits);
    k_gemm<A_KMAJ, B_NK, EPI, BM, BN, BK, WM, WN><<<grid, WM * WN * 32, 0, st>>>(g);
    return cudaGetLastError();
}

// Picks the tile configuration of each GEMM of the network by shape.
cudaError_t launch_gemm(GemmKind kind, GemmArgs g, cudaStream_t st) {
    switch (kind) {
        case GEMM_FWD_FIRST:   // Z1 = X0 W1^T, K = 16
            g.k_split = g.K;
            return gemm_t<true, true, EPI_FWD_SILU, 128, 128, 16, 2, 4>(g, 1, st);
        case GEMM_FWD_HIDDEN:  // K = N = 256
            g.k_split = g.K;
            return gemm_t<true, true, EPI_FWD_SILU, 128, 128, 32, 2, 4>(g, 1, st);
        case GEMM_FWD_OUT:     // N = 16
            g.k_split = g.K;
            return gemm_t<true, true, EPI_FWD_OUT, 128, 16, 32, 8, 1>(g, 1, st);
        case GEMM_DX_FROM_OUT:  // dH4 = dOut W5, K = 16
            g.k_split = g.K;
            return gemm_t<true, false, EPI_DX, 128, 128, 16, 2, 4>(g, 1, st);
        case GEMM_DX_HIDDEN:
            g.k_split = g.K;
            return gemm_t<true, false, EPI_DX, 128, 128, 32, 2, 4>(g, 1, st);
        case GEMM_DW_HIDDEN: {  // dW = dZ^T H, batch split over blockIdx.z
            int splits = g.K / g.k_split;
            return gemm_t<false, false, EPI_DW, 128, 128, 32, 2, 4>(g, splits, st);
        }
        case GEMM_DW_FIRST: {  // N = 16
            int splits = g.K / g.k_split;
            return gemm_t<false, false, EPI_DW, 128, 16, 32, 8, 1>(g, splits, st);
        }
        case GEMM_DW_OUT: {  // M = 16
            int splits = g.K / g.k_split;
            return gemm_t<false, false, EPI_DW, 16, 128, 32, 1, 4>(g, splits, st);
        }
    }
    return cudaErrorInvalidValue;
}

// ------------------------------------------------------------ small kernels
// Column sums of a BF16 [rows][ld] matrix into an FP32 vector (bias gradients).
__global__ void __launch_bounds__(256) k_colsum(const __nv_bfloat16* __restrict__ X, int rows, int ld, int cols,
                                                int rows_per_block, float* __restrict__ out) {
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r0 = blockIdx.y * rows_per_block;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = r0 + (threadIdx.x >> 5); r < min(rows, r0 + rows_per_block); r += 8)
        s += __bfloat162float(X[size_t(r) * ld + c]);
    __shared__ float red[8][32];
    red[threadIdx.x >> 5][threadIdx.x & 31] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = 0.f;
        for (int i = 0; i < 8; ++i) t += red[i][threadIdx.x];
        atomicAdd(&out[c], t);
    }
}

cudaError_t launch_colsum(const __nv_bfloat16* X, int rows, int ld, int cols, float* out, cudaStream_t st) {
    const int rpb = 1024;
    dim3 grid((cols + 31) / 32, (rows + rpb - 1) / rpb);
    k_colsum<<<grid, 256, 0, st>>>(X, rows, ld, cols, rpb, out);
    return cudaGetLastError();
}


// Loss of one batch and its gradient w.r.t. the outputs (scaled by 1/B):
// mlp_row_loss (mlp_loss.cuh) per row; dout in BF16 and dout32 in FP32,
// row-major.
__global__ void __launch_bounds__(256) k_loss(const float* __restrict__ out, const SampleLabel* __restrict__ lab,
                                              int B, LossWeights w, __nv_bfloat16* __restrict__ dout,
                                              float* __restrict__ dout32, float* __restrict__ loss_acc) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (b < B) {
        float o[MLP_OUT_PAD], d[MLP_OUT_PAD];
#pragma unroll
        for (int i = 0; i < MLP_OUT_PAD; i += 4) {
            const float4 v = *reinterpret_cast<const float4*>(out + size_t(b) * MLP_OUT_PAD + i);
            o[i] = v.x; o[i + 1] = v.y; o[i + 2] = v.z; o[i + 3] = v.w;
        }
        l = mlp_row_loss(o, lab[b], w, d);
        const float inv_b = 1.0f / float(B);
#pragma unroll
        for (int i = 0; i < MLP_OUT_PAD; ++i) {
            dout32[size_t(b) * MLP_OUT_PAD + i] = d[i] * inv_b;
            dout[size_t(b) * MLP_OUT_PAD + i] = __float2bfloat16_rn(d[i] * inv_b);
        }
    }
    // block reduction of the loss
    __shared__ float red[256];
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss_acc, red[0] / float(B));
}

cudaError_t launch_loss(const float* out, const SampleLabel* lab, int B, LossWeights w, __nv_bfloat16* dout,
                        float* dout32, float* loss_acc, cudaStream_t st) {
    k_loss<<<(B + 255) / 256, 256, 0, st>>>(out, lab, B, w, dout, dout32, loss_acc);
    return cudaGetLastError();
}

// Bias gradients of the output layer from the FP32 output gradient.
__global__ void k_colsum_f32(const float* __restrict__ X, int rows, int cols, float* __restrict__ out) {
    const int c = threadIdx.x & 15;
    float s = 0.f;
    for (int r = blockIdx.x * 16 + (threadIdx.x >> 4); r < rows; r += gridDim.x * 16) s += X[size_t(r) * cols + c];
    atomicAdd(&out[c], s);
}

cudaError_t launch_colsum_f32(const float* X, int rows, int cols, float* out, cudaStream_t st) {
    k_colsum_f32<<<256, 256, 0, st>>>(X, rows, cols, out);
    return cudaGetLastError();
}

// Adam on n FP32 parameters; bf16_copy (may be null) receives the new weights.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ bf16_copy, __nv_bfloat16* __restrict__ img,
                       __nv_bfloat16* __restrict__ img_t, int n, AdamStep a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = grad[i] * a.gscale;
    const float mi = a.b1 * m[i] + (1.f - a.b1) * gi;
    const float vi = a.b2 * v[i] + (1.f - a.b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - a.lr * (mi * a.c1) / (sqrtf(vi * a.c2) + a.eps);
    p[i] = pi;
    const __nv_bfloat16 h = __float2bfloat16_rn(pi);
    if (bf16_copy) bf16_copy[i] = h;
    if (img) {
        uint32_t f, t;
        bool halved;
        mlp_image_offsets(uint32_t(i), &f, &t, &halved);
        const __nv_bfloat16 w = halved ? __hmul(h, __float2bfloat16(0.5f)) : h;
        if (f != ~0u) img[f / 2] = w;
        if (img_t && t != ~0u) img_t[t / 2] = w;
    }
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, __nv_bfloat16* copy, void* img, void* img_t,
                        int n, AdamStep a, cudaStream_t st) {
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(p, g, m, v, copy, static_cast<__nv_bfloat16*>(img),
                                             static_cast<__nv_bfloat16*>(img_t), n, a);
    return cudaGetLastError();
}

// Adam with the constants of the current step of a counted run.  Every
// block reads ctr->step before it counts itself done, so the last block's
// advance comes after all reads.
// Launched as the dependent of the weight gradients, a block loads before
// its griddepcontrol.wait what only earlier kernels wrote: the step counter
// and constants, m, v and p (the Adam of the step before, whose completion
// the kernels in between waited for); the partials after it.
__global__ void k_adam_counted(float* __restrict__ p, const float* __restrict__ grad, const float* __restrict__ part,
                               DwJobs jobs, uint32_t max_rows, float* __restrict__ m, float* __restrict__ v,
                               __nv_bfloat16* __restrict__ bf16_copy, __nv_bfloat16* __restrict__ img,
                               __nv_bfloat16* __restrict__ img_t, int n, const AdamStep* __restrict__ table,
                               TrainCounters* ctr) {
    __shared__ AdamStep a;
    __shared__ __align__(8) uint64_t bar;
    extern __shared__ __align__(16) float rows[];  // [jobs of this block's parameters][256]
    const uint32_t step = *reinterpret_cast<volatile uint32_t*>(&ctr->step);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float m_old = 0.f, v_old = 0.f, p_old = 0.f;
    if (i < n) {
        m_old = m[i];
        v_old = v[i];
        p_old = p[i];
    }
    // the block's 256 parameters lie in one segment of the parameter vector
    // (all segment boundaries are multiples of 256): where their partials
    // are contiguous (all but W5's transpose), one thread brings the jobs'
    // rows of 1 KB into shared memory with bulk copies
    const uint32_t i0 = blockIdx.x * blockDim.x;
    uint32_t j0, nj, src0, d0, d1, src1;
    mlp_dw_source(i0, jobs, &j0, &nj, &src0);
    mlp_dw_source(i0 + 1, jobs, &d0, &d1, &src1);
    const bool bulk = part && blockDim.x == 256 && src1 == src0 + 1 && nj <= max_rows;
    const uint32_t b_addr = tc::smem_addr(&bar);
    if (threadIdx.x == 0) {
        a = table[step];
        if (bulk) {
            tc::mbar_init(b_addr, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0 && bulk) {
        tc::mbar_expect_tx(b_addr, nj * 1024u);
        for (uint32_t k = 0; k < nj; ++k)
            tc::bulk_g2s(tc::smem_addr(rows + k * 256), part + size_t(j0 + k) * MLP_DW_PART + src0, 1024u, b_addr);
    }
    __syncthreads();
    bool landed = false;
    if (bulk)
        for (uint32_t it = 0; it < tc::SLEEP_LIMIT && !landed; ++it) landed = tc::mbar_try_sleep(b_addr, 0, 1000000u);
    if (i < n) {
        float gs;
        if (part) {
            uint32_t pj0, pnj, src;
            mlp_dw_source(uint32_t(i), jobs, &pj0, &pnj, &src);
            gs = 0.f;
            if (landed) {
                for (uint32_t k = 0; k < pnj; ++k) gs += rows[k * 256 + threadIdx.x];
            } else {
#pragma unroll 8
                for (uint32_t k = 0; k < pnj; ++k) gs += part[size_t(pj0 + k) * MLP_DW_PART + src];
            }
        } else {
            gs = grad[i];
        }
        const float gi = gs * a.gscale;
        const float mi = a.b1 * m_old + (1.f - a.b1) * gi;
        const float vi = a.b2 * v_old + (1.f - a.b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p_old - a.lr * (mi * a.c1) / (sqrtf(vi * a.c2) + a.eps);
        p[i] = pi;
        const __nv_bfloat16 h = __float2bfloat16_rn(pi);
        if (bf16_copy) bf16_copy[i] = h;
        if (img) {
            uint32_t f, t;
            bool halved;
            mlp_image_offsets(uint32_t(i), &f, &t, &halved);
            const __nv_bfloat16 w = halved ? __hmul(h, __float2bfloat16(0.5f)) : h;
            if (f != ~0u) img[f / 2] = w;
            if (img_t && t != ~0u) img_t[t / 2] = w;
        }
    }
    // no copy may still be landing in this block's shared memory when it exits
    if (bulk && !landed && threadIdx.x == 0)
        for (uint32_t it = 0; it < tc::SLEEP_LIMIT && !tc::mbar_try_sleep(b_addr, 0, 1000000u); ++it) {}
    __syncthreads();
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctr->done, 1u) == gridDim.x - 1) {
            ctr->done = 0u;
            ctr->step = step + 1u;
            ctr->batch += 1u;
            __threadfence();
        }
    }
}

cudaError_t launch_adam_counted(float* p, const float* g, const float* part, const DwJobs& jobs, float* m, float* v,
                                __nv_bfloat16* copy, void* img, void* img_t, int n, const AdamStep* table,
                                TrainCounters* ctr, cudaStream_t st, bool pdl) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    // room for the partial rows of the largest job kind (at most
    // MGK_ADAM_BULK_ROWS rows of 1 KB; 0: every partial read directly)
    const uint32_t max_rows =
        part ? std::min<uint32_t>(MGK_ADAM_BULK_ROWS, std::max(jobs.heavy, std::max(jobs.l0, jobs.l4))) : 0u;
    cfg.gridDim = dim3((n + 255) / 256, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = max_rows * 1024u;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_adam_counted, p, g, part, jobs, max_rows, m, v, copy,
                                       static_cast<__nv_bfloat16*>(img), static_cast<__nv_bfloat16*>(img_t), n,
                                       table, ctr);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// Batch assembly: rows perm[b0 + i] of the sample set.
__global__ void k_gather(const float* __restrict__ feat, const SampleLabel* __restrict__ lab,
                         const uint32_t* __restrict__ perm, int b0, int B, __nv_bfloat16* __restrict__ x0,
                         SampleLabel* __restrict__ blab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const uint32_t s = perm[b0 + i];
    for (int k = 0; k < MLP_IN_PAD; ++k)
        x0[size_t(i) * MLP_IN_PAD + k] = __float2bfloat16_rn(k < MLP_IN ? feat[size_t(s) * MLP_IN + k] : 0.f);
    blab[i] = lab[s];
}

cudaError_t launch_gather(const float* feat, const SampleLabel* lab, const uint32_t* perm, int b0, int B,
                          __nv_bfloat16* x0, SampleLabel* blab, cudaStream_t st) {
    k_gather<<<(B + 255) / 256, 256, 0, st>>>(feat, lab, perm, b0, B, x0, blab);
    return cudaGetLastError();
}

// The sample-set order of one epoch: perm[i] = P(i) for a keyed
// pseudo-random permutation P of [0, n).  P is a 4-round balanced Feistel
// network on the smallest even number of bits that covers n (a bijection of
// that domain), its round function the MurmurHash3 finalizer (A. Appleby)
// of the right half xor the round key; values outside [0, n) are walked on
// through P until they fall inside ("cycle walking": the orbit of i under P
// returns to i < n, so the walk ends, after fewer than 4 steps on average).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint32_t feistel_index(uint32_t i, uint32_t n, uint32_t half_bits, uint4 key) {
    const uint32_t mask = half_bits >= 32 ? 0xFFFFFFFFu : (1u << half_bits) - 1u;
    const uint32_t k[4] = {key.x, key.y, key.z, key.w};
    uint32_t x = i;
    do {
        uint32_t L = x >> half_bits, R = x & mask;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t t = L ^ (fmix32(R ^ k[r]) & mask);
            L = R;
            R = t;
        }
        x = (L << half_bits) | R;
    } while (x >= n);
    return x;
}
__global__ void k_epoch_perm(uint32_t* __restrict__ perm, uint32_t n, uint32_t half_bits, uint4 key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = feistel_index(i, n, half_bits, key);
}

__global__ void k_epoch_begin(TrainCounters* ctr) {
    ctr->batch = 0u;
    ctr->epoch += 1u;
}
__global__ void k_epoch_perm_counted(uint32_t* __restrict__ perm, uint32_t n, uint32_t half_bits,
                                     const uint4* __restrict__ keys, const TrainCounters* ctr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = feistel_index(i, n, half_bits, keys[ctr->epoch - 1u]);
}

cudaError_t launch_epoch_begin(uint32_t* perm, uint32_t n, const uint4* keys, TrainCounters* ctr, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_epoch_begin<<<1, 1, 0, st>>>(ctr);
    uint32_t bits = 2;
    while (bits < 32 && (uint64_t(1) << bits) < n) ++bits;
    bits += bits & 1u;
    k_epoch_perm_counted<<<(n + 255) / 256, 256, 0, st>>>(perm, n, bits / 2, keys, ctr);
    return cudaGetLastError();
}

cudaError_t launch_epoch_perm(uint32_t* perm, uint32_t n, const uint32_t key[4], cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t bits = 2;
    while (bits < 32 && (uint64_t(1) << bits) < n) ++bits;
    bits += bits & 1u;
    k_epoch_perm<<<(n + 255) / 256, 256, 0, st>>>(perm, n, bits / 2, make_uint4(key[0], key[1], key[2], key[3]));
    return cudaGetLastError();
}

// Inference input: n FP32 feature rows (7 floats) to BF16 rows of 16, rows
// [n, rows) zero.
__global__ void k_features_bf16(const float* __restrict__ feat, uint32_t n, uint32_t rows,
                                __nv_bfloat16* __restrict__ x0) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    __nv_bfloat162 v[MLP_IN_PAD / 2];
#pragma unroll
    for (int k = 0; k < MLP_IN_PAD / 2; ++k) {
        const float a = (i < n && 2 * k < MLP_IN) ? feat[size_t(i) * MLP_IN + 2 * k] : 0.f;
        const float b = (i < n && 2 * k + 1 < MLP_IN) ? feat[size_t(i) * MLP_IN + 2 * k + 1] : 0.f;
        v[k] = __floats2bfloat162_rn(a, b);
    }
    uint4* dst = reinterpret_cast<uint4*>(x0 + size_t(i) * MLP_IN_PAD);
    dst[0] = *reinterpret_cast<const uint4*>(&v[0]);
    dst[1] = *reinterpret_cast<const uint4*>(&v[4]);
}

cudaError_t launch_features_bf16(const float* feat, uint32_t n, uint32_t rows, __nv_bfloat16* x0, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    k_features_bf16<<<(rows + 255) / 256, 256, 0, st>>>(feat, n, rows, x0);
    return cudaGetLastError();
}

}  // namespace mgk
