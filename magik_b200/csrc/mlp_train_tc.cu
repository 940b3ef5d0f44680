// Training kernels of the deflection surrogate on the 5th-generation tensor
// cores (tcgen05.mma, accumulators in tensor memory, operands brought in by
// bulk copies), for one batch of B rows (a multiple of 128):
//
//  k_mlp_chain_tc<FWD>  forward with stash: all five layers of a 128-row
//                       tile in one CTA (the structure of the fused
//                       inference kernel), writing the pre-activations Z_l
//                       of layers 1-4 (the activations H_l = silu(Z_l) are
//                       recomputed where the weight gradients need them),
//                       then the loss of each row (mlp_loss.cuh) and the
//                       BF16 output gradient dOut.  The FP32 outputs are
//                       written only where asked for.
//  k_mlp_chain_tc<BWD>  the input gradients of a tile through the layers:
//                       dZ4 = (dOut W5) * silu'(Z4), dZ3 = (dZ4 W4) * silu'(Z3),
//                       ... dZ1, the weights read as the transposes of the
//                       forward's weight image (N-major operands).
//  k_mlp_dw_tc          weight gradients dW_l = dZ_l^T H_{l-1} (and
//                       dW5^T = H4^T dOut) over a range of batch tiles per
//                       CTA (split K), both operands M/N-major views of the
//                       stashed tiles, the partial in tensor memory, written
//                       once per CTA.  The CTA's other warps turn each staged
//                       Z_{l-1} into H_{l-1} = silu(Z_{l-1}) in shared memory
//                       before its MMAs and sum the columns of dZ_l (dOut for
//                       layer 5) for the bias gradients.
//  k_mlp_dw_reduce      sums the CTAs' partials into the gradient vector (no
//                       atomics: the gradient does not depend on the order in
//                       which CTAs finish).
//
// Activation layout in global memory ("tiled"): the rows of a matrix with C
// columns (C = 16 or 256) in tiles of 128; tile t at t * 128 * C * 2 bytes;
// inside a tile, element (row, col) at kmaj(row, col, 16 C) (tc_sm100.cuh),
// the K-major operand layout of the tensor cores.  A tile is thus one
// contiguous bulk copy and serves as the K-major A operand of the next layer
// and, read with SBO = 128 and LBO = 16 C, as the M- or N-major operand of
// the weight gradients.  The weight image (mlp_tc.cu) serves the forward as
// K-major B operand and the backward as N-major B operand the same way.
//
// SiLU and its derivative come from tanh.approx.f32:
//   silu(z) = u + u tanh(u) and sigmoid(z) = (1 + tanh(u)) / 2, u = z / 2;
//   silu'(z) = s (1 + z (1 - s)).
// The results are rounded to BF16 where the network stores them (Z, H, dZ),
// so the approximation's 2^-11 relative error is below their resolution.
//
// Every mbarrier wait is bounded (tc::mbar_wait); a timeout sets bit 1 of
// *status, the other roles leave their loops, the CTA drains its copies and
// MMAs and frees its tensor memory.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.h"
#include "mlp_loss.cuh"
#include "tc_sm100.cuh"

namespace mgk {
namespace {

using namespace tc;

constexpr int TM = 128;
constexpr uint32_t A_BYTES = TM * MLP_HID * 2;  // 64 KB activation tile
constexpr uint32_t A_SBO = 4096;                // 8-row group stride of a 256-column tile
constexpr uint32_t X_SBO = 256;                 // ... of a 16-column tile
constexpr uint32_t X_TILE = TM * MLP_IN_PAD * 2;  // 4 KB

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
__device__ __forceinline__ float2 unpack_bf16(uint32_t v) {
    return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xFFFF0000u));
}
// silu of both BF16 halves of a word, rounded back to BF16
__device__ __forceinline__ uint32_t silu_bf16x2(uint32_t v) {
    const float2 z = unpack_bf16(v);
    return pack_bf16(silu_f(z.x), silu_f(z.y));
}
__device__ __forceinline__ void add_bf16x2(float& a, float& b, uint32_t v) {
    const float2 f = unpack_bf16(v);
    a += f.x;
    b += f.y;
}

// ============================================================ chain kernel
constexpr int N_SLOT = 2;
constexpr uint32_t SLOT_BYTES = 32768;
constexpr int EPI_WARPS = 16;
constexpr int CH_THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t CH_TMEM = 512;
constexpr uint32_t OFF_A = 0;
constexpr uint32_t OFF_W = OFF_A + 2 * A_BYTES;
constexpr uint32_t OFF_BIAS = OFF_W + N_SLOT * SLOT_BYTES;
constexpr uint32_t N_BIAS = 4 * MLP_HID + MLP_OUT_PAD;
constexpr uint32_t OFF_BAR = OFF_BIAS + N_BIAS * 4;
constexpr uint32_t OFF_MISC = OFF_BAR + 16 * 8;
constexpr uint32_t CH_SMEM = OFF_MISC + 16 + 128;
static_assert(CH_SMEM <= 232448, "shared memory");

enum { FWD = 0, BWD = 1 };

// Step `l` of a tile: its weight chunks and the shape of their MMAs.
struct Step {
    int c0, nc;         // first chunk of the weight image, number of chunks
    int ksteps;         // K steps of 16 per chunk
    uint32_t n;         // MMA N
    uint32_t b_lbo, b_sbo, b_kstep;  // B descriptor and its advance per K step
    bool b_mn;          // B read N-major (the transposed weights)
    bool a_reset;       // the A operand's K restarts at 0 in every chunk (N-sliced chunks)
    uint32_t d_col;     // TMEM column advance per chunk
};
template <int DIR> __device__ __forceinline__ Step step_of(int l) {
    if constexpr (DIR == FWD) {
        if (l == 0) return Step{0, 1, 1, 256u, 128u, 256u, 256u, false, false, 0u};
        if (l == 4) return Step{13, 1, 16, 16u, 128u, 4096u, 256u, false, false, 0u};
        return Step{1 + 4 * (l - 1), 4, 4, 256u, 128u, 1024u, 256u, false, false, 0u};
    } else {
        // W5^T: one chunk, K = 16 (the outputs), N = 256; then W4^T, W3^T,
        // W2^T: four chunks of 64 output columns, K = 256 each
        if (l == 0) return Step{13, 1, 1, 256u, 4096u, 128u, 8192u, true, false, 0u};
        const int layer = 4 - l;  // 3, 2, 1: W4, W3, W2
        return Step{1 + 4 * (layer - 1), 4, 16, 64u, 1024u, 128u, 2048u, true, true, 64u};
    }
}

struct ChainArgs {
    const unsigned char* img;  // weight image (layers 1-4 stored halved)
    const float* params;       // FP32 parameters (biases)
    const unsigned char* in;   // FWD: X0 tiles (16 columns); BWD: dOut tiles (16 columns)
    unsigned char* z[4];       // Z_1..Z_4 tiles (FWD writes, BWD reads)
    unsigned char* dz[4];      // BWD: dZ_1..dZ_4 tiles (written)
    float* out;                // FWD: outputs [rows][16] FP32, or null
    const SampleLabel* lab;    // FWD: the batch's labels for the fused loss
    unsigned char* dout;       // FWD: dOut tiles (16 columns), d(loss)/d(out) / B in BF16
    float* loss_acc;           // FWD: += the batch's mean loss
    LossWeights w;
    uint32_t n_tiles;
    uint32_t* status;
};

template <int DIR>
__global__ void __launch_bounds__(CH_THREADS, 1) k_mlp_chain_tc(ChainArgs g) {
    constexpr int S = DIR == FWD ? MLP_LAYERS : MLP_LAYERS - 1;  // steps per tile
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t sbase = smem_addr(smem);
    const uint32_t bar_full = sbase + OFF_BAR, bar_empty = bar_full + N_SLOT * 8;
    const uint32_t bar_d = bar_full + 2 * N_SLOT * 8, bar_a = bar_d + 2 * 8, bar_drain = bar_a + 2 * 8;
    float* bias = reinterpret_cast<float*>(smem + OFF_BIAS);
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(smem + OFF_MISC);
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + OFF_MISC + 4);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_tiles = g.n_tiles;
    const uint32_t my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t my_pairs = (my_tiles + 1) / 2;  // an odd count ends with an empty tile in buffer 1

    if constexpr (DIR == FWD) {
        for (uint32_t i = threadIdx.x; i < N_BIAS; i += CH_THREADS) {
            const int l = i < 4 * MLP_HID ? int(i / MLP_HID) : 4;
            const uint32_t k = i < 4 * MLP_HID ? i % MLP_HID : i - 4 * MLP_HID;
            bias[i] = g.params[mlp_b_off(l) + k];
        }
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < N_SLOT; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bar_d + 8 * b, 1);
            mbar_init(bar_a + 8 * b, 32 * EPI_WARPS / 2);
        }
        mbar_init(bar_drain, 1);
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + OFF_MISC),
                     "r"(CH_TMEM)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t j = 0;
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l)
                    for (int b = 0; b < 2 && ok; ++b) {
                        const Step st = step_of<DIR>(l);
                        if constexpr (DIR == BWD) {
                            // the Z tiles the epilogue reads for silu', one step ahead, into L2
                            const uint32_t tile = blockIdx.x + (2 * p + uint32_t(b)) * gridDim.x;
                            if (tile < n_tiles) {
                                if (l == 0) bulk_prefetch_l2(g.z[3] + size_t(tile) * A_BYTES, A_BYTES);
                                const unsigned char* zn = l == 0 ? g.z[2] : (l == 1 ? g.z[1] : g.z[0]);
                                if (l + 1 < S) bulk_prefetch_l2(zn + size_t(tile) * A_BYTES, A_BYTES);
                            }
                        }
                        for (int ci = 0; ci < st.nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (use > 0 && !mbar_wait(bar_empty + 8 * s, (use - 1) & 1u, abort_flag)) {
                                ok = false;
                                break;
                            }
                            const int c = st.c0 + ci;
                            mbar_expect_tx(bar_full + 8 * s, mlp_chunk_bytes(c));
                            bulk_g2s(sbase + OFF_W + s * SLOT_BYTES, g.img + mlp_chunk_offset(c), mlp_chunk_bytes(c),
                                     bar_full + 8 * s);
                        }
                    }
            const uint32_t first = j > N_SLOT ? j - N_SLOT : 0;
            for (uint32_t k = first; k < j; ++k) {
                const uint32_t s = k % N_SLOT, use = k / N_SLOT;
                for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_full + 8 * s, use & 1u); ++it) {}
            }
        }
    } else if (warp == 1) {
        // ----------------------------------------------------------------- MMA
        if (lane == 0) {
            uint32_t j = 0, ar[2] = {0u, 0u};
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l)
                    for (uint32_t b = 0; b < 2 && ok; ++b) {
                        if (!mbar_wait(bar_a + 8 * b, ar[b] & 1u, abort_flag)) { ok = false; break; }
                        ++ar[b];
                        tc_fence_after();
                        const Step st = step_of<DIR>(l);
                        const uint32_t idesc = idesc_bf16_major(TM, st.n, false, st.b_mn);
                        const uint32_t a_base = sbase + OFF_A + b * A_BYTES;
                        for (int ci = 0; ci < st.nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                            tc_fence_after();
                            const uint32_t wslot = sbase + OFF_W + s * SLOT_BYTES;
                            const uint32_t d = tmem + b * 256u + uint32_t(ci) * st.d_col;
                            for (int ks = 0; ks < st.ksteps; ++ks) {
                                const uint32_t kk = st.a_reset ? uint32_t(ks) : uint32_t(ci * st.ksteps + ks);
                                const uint64_t a = smem_desc(a_base + kk * 256u, 128u, A_SBO);
                                const uint64_t bd = smem_desc(wslot + uint32_t(ks) * st.b_kstep, st.b_lbo, st.b_sbo);
                                mma_bf16_ss(d, a, bd, idesc, kk > 0 ? 1u : 0u);
                            }
                            mma_commit(bar_empty + 8 * s);
                        }
                        if (ok) mma_commit(bar_d + 8 * b);
                    }
            mma_commit(bar_drain);
            for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_drain, 0); ++it) {}
        }
    } else {
        // ------------------------------------------------------------ epilogue
        // a warp reads the TMEM lanes of its place in its warpgroup, 32 (warp
        // % 4) ..; the first four warps of a buffer take columns 0-127, the
        // other four 128-255
        const uint32_t buf = (warp - 2) >> 3, q = warp & 3u, half = ((warp - 2) >> 2) & 1u;
        const uint32_t row = q * 32 + lane;
        const uint32_t t_lane = tmem + ((q * 32u) << 16) + buf * 256u;
        unsigned char* A = smem + OFF_A + buf * A_BYTES;
        const uint32_t bar_db = bar_d + 8 * buf, bar_ab = bar_a + 8 * buf;
        uint32_t dr = 0;
        bool ok = true;
        float loss = 0.f;  // FWD: this thread's rows' loss
        for (uint32_t t = buf; t < 2 * my_pairs && ok; t += 2) {
            const uint32_t tile = blockIdx.x + t * gridDim.x;  // >= n_tiles for the empty tile
            const bool valid = tile < n_tiles;
            // the tile's 16-column input (X0, or dOut) into the A buffer
            if (half == 0) {
                uint4 c0 = uint4{0u, 0u, 0u, 0u}, c1 = c0;
                if (valid) {
                    const unsigned char* src = g.in + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                    c0 = *reinterpret_cast<const uint4*>(src);
                    c1 = *reinterpret_cast<const uint4*>(src + 128);
                }
                *reinterpret_cast<uint4*>(A + kmaj(row, 0, A_SBO)) = c0;
                *reinterpret_cast<uint4*>(A + kmaj(row, 8, A_SBO)) = c1;
            }
            fence_proxy_async();
            mbar_arrive(bar_ab);
            const size_t tile_off = size_t(tile) * A_BYTES;
            for (int l = 0; l < S; ++l) {
                const int li = DIR == FWD ? l : 3 - l;  // the Z (dZ) index this step writes (reads)
                unsigned char* const zl = li == 0 ? g.z[0] : (li == 1 ? g.z[1] : (li == 2 ? g.z[2] : g.z[3]));
                unsigned char* const dzl = li == 0 ? g.dz[0] : (li == 1 ? g.dz[1] : (li == 2 ? g.dz[2] : g.dz[3]));
                // BWD: the first block's Z, loaded while the MMAs run
                uint4 zn[4];
                if constexpr (DIR == BWD) {
#pragma unroll
                    for (int gq = 0; gq < 4; ++gq)
                        zn[gq] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off +
                                                                          kmaj(row, half * 128 + 8 * gq, A_SBO))
                                       : uint4{0u, 0u, 0u, 0u};
                }
                if (!mbar_wait(bar_db, dr & 1u, abort_flag)) { ok = false; break; }
                ++dr;
                tc_fence_after();
                if (DIR == FWD && l == 4) {
                    if (half == 0) {
                        uint32_t v[16];
                        tmem_ld16(t_lane, v);
                        tmem_wait_ld(v);
                        tc_fence_before();
                        if (valid) {
                            const float* b5 = bias + 4 * MLP_HID;
                            float o[MLP_OUT_PAD];
#pragma unroll
                            for (int k = 0; k < MLP_OUT_PAD; ++k) o[k] = __uint_as_float(v[k]) + b5[k];
                            const uint32_t r = tile * TM + row;
                            if (g.out) {
                                float4* op = reinterpret_cast<float4*>(g.out + size_t(r) * MLP_OUT_PAD);
#pragma unroll
                                for (int k = 0; k < 4; ++k)
                                    op[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
                            }
                            if (g.lab) {
                                float d[MLP_OUT_PAD];
                                loss += mlp_row_loss(o, g.lab[r], g.w, d);
                                const float inv_b = 1.0f / float(n_tiles * TM);
                                uint32_t dv[8];
#pragma unroll
                                for (int k = 0; k < 8; ++k) dv[k] = pack_bf16(d[2 * k] * inv_b, d[2 * k + 1] * inv_b);
                                unsigned char* dst = g.dout + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                                *reinterpret_cast<uint4*>(dst) = uint4{dv[0], dv[1], dv[2], dv[3]};
                                *reinterpret_cast<uint4*>(dst + 128) = uint4{dv[4], dv[5], dv[6], dv[7]};
                            }
                        }
                    }
                    continue;
                }
                // 4 blocks of 32 columns of this warp's half
                const float scale = (DIR == FWD || l > 0) ? 2.0f : 1.0f;  // layers 1-4 are stored halved
                for (int blk = 0; blk < 4; ++blk) {
                    const uint32_t col = half * 128 + uint32_t(blk) * 32;
                    uint32_t v[32];
                    tmem_ld32(t_lane + col, v);
                    tmem_wait_ld(v);
#pragma unroll
                    for (int gq = 0; gq < 4; ++gq) {
                        const uint32_t off = kmaj(row, col + 8 * gq, A_SBO);
                        uint32_t hv[4], zv[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int c = gq * 8 + 2 * e;
                            const float a0 = scale * __uint_as_float(v[c]), a1 = scale * __uint_as_float(v[c + 1]);
                            if constexpr (DIR == FWD) {
                                const float z0 = a0 + bias[l * MLP_HID + col + c];
                                const float z1 = a1 + bias[l * MLP_HID + col + c + 1];
                                zv[e] = pack_bf16(z0, z1);
                                hv[e] = pack_bf16(silu_f(z0), silu_f(z1));
                            } else {
                                const uint32_t zw = e == 0 ? zn[gq].x : (e == 1 ? zn[gq].y : (e == 2 ? zn[gq].z : zn[gq].w));
                                const float2 zf = unpack_bf16(zw);
                                hv[e] = pack_bf16(a0 * silu_grad_f(zf.x), a1 * silu_grad_f(zf.y));
                                zv[e] = 0u;
                            }
                        }
                        // FWD: H into the next layer's operand, Z to the stash;
                        // BWD: dZ into the next step's operand and to global memory
                        const uint4 h4 = uint4{hv[0], hv[1], hv[2], hv[3]};
                        if (l < S - 1) *reinterpret_cast<uint4*>(A + off) = h4;
                        if (valid) {
                            if constexpr (DIR == FWD)
                                *reinterpret_cast<uint4*>(zl + tile_off + off) = uint4{zv[0], zv[1], zv[2], zv[3]};
                            else
                                *reinterpret_cast<uint4*>(dzl + tile_off + off) = h4;
                        }
                    }
                    if constexpr (DIR == BWD) {
                        // the next block's Z, loaded while this block's results drain
                        if (blk < 3) {
#pragma unroll
                            for (int gq = 0; gq < 4; ++gq)
                                zn[gq] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off +
                                                                                  kmaj(row, col + 32 + 8 * gq, A_SBO))
                                               : uint4{0u, 0u, 0u, 0u};
                        }
                    }
                }
                tc_fence_before();
                if (l < S - 1) {
                    fence_proxy_async();
                    mbar_arrive(bar_ab);
                }
            }
        }
        if constexpr (DIR == FWD) {
            if (half == 0 && g.loss_acc) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
                if (lane == 0) atomicAdd(g.loss_acc, loss / float(n_tiles * TM));
            }
        }
    }
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(g.status, 2u);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CH_TMEM) : "memory");
    }
}

// ========================================================= weight gradients
// Job j of the grid: layer L and a contiguous range of batch tiles.
//   L = 0:    dW1 = dZ1^T X0      M = 256 (dZ1 columns), N = 16
//   L = 1..3: dW_{L+1} = dZ_{L+1}^T H_L   M = 256, N = 256
//   L = 4:    dW5^T = H4^T dOut   M = 256 (H4 columns), N = 16
// Stages of 64 batch rows: half a tile of the A matrix (32 KB) and of the B
// matrix (32 KB, or 2 KB for 16 columns); the M = 256 rows of the result in
// two MMA halves of 128.  H_L comes in as Z_L and is made in place.  A stage
// passes full (the bulk copies landed) -> conv (the epilogue warps made H and
// took the column sums) -> the MMAs -> empty (their commit).
constexpr int DW_STAGES = 3;
constexpr uint32_t DW_A_BYTES = 32768, DW_B_BYTES = 32768;
constexpr uint32_t DW_STAGE = DW_A_BYTES + DW_B_BYTES;
constexpr int DW_EPI_WARPS = 8;
constexpr int DW_THREADS = 32 * (2 + DW_EPI_WARPS);
constexpr uint32_t DW_OFF_BAR = DW_STAGES * DW_STAGE;
constexpr uint32_t DW_OFF_MISC = DW_OFF_BAR + 16 * 8;
constexpr uint32_t DW_OFF_RED = DW_OFF_MISC + 16;             // [8 warps][16] output-bias sums
constexpr uint32_t DW_SMEM = DW_OFF_RED + DW_EPI_WARPS * 16 * 4 + 128;
static_assert(DW_SMEM <= 232448, "shared memory");
constexpr uint32_t DW_PART = MLP_HID * MLP_HID + MLP_HID;  // floats per job: the partial dW and bias sums

struct DwArgs {
    const unsigned char* dz[4];  // dZ1..dZ4 tiles
    const unsigned char* z[4];   // Z1..Z4 tiles (H = silu(Z) is made in shared memory)
    const unsigned char* x0;     // X0 tiles (16 columns)
    const unsigned char* dout;   // dOut tiles (16 columns)
    float* part;                 // [jobs][DW_PART]
    uint32_t n_tiles;
    uint32_t jobs_heavy;         // jobs per layer of L = 1..3
    uint32_t jobs_light;         // jobs per layer of L = 0 and 4
    uint32_t* status;
};

__device__ __forceinline__ void dw_job(const DwArgs& g, uint32_t j, int& L, uint32_t& t0, uint32_t& t1) {
    uint32_t per, k;
    if (j < 3 * g.jobs_heavy) {
        L = 1 + int(j / g.jobs_heavy);
        per = g.jobs_heavy;
        k = j % g.jobs_heavy;
    } else {
        const uint32_t jl = j - 3 * g.jobs_heavy;
        L = jl < g.jobs_light ? 0 : 4;
        per = g.jobs_light;
        k = jl % g.jobs_light;
    }
    t0 = uint32_t(uint64_t(g.n_tiles) * k / per);
    t1 = uint32_t(uint64_t(g.n_tiles) * (k + 1) / per);
}

__global__ void __launch_bounds__(DW_THREADS, 1) k_mlp_dw_tc(DwArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t sbase = smem_addr(smem);
    const uint32_t bar_full = sbase + DW_OFF_BAR, bar_empty = bar_full + DW_STAGES * 8;
    const uint32_t bar_conv = bar_empty + DW_STAGES * 8;
    const uint32_t bar_done = bar_conv + DW_STAGES * 8, bar_drain = bar_done + 8;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(smem + DW_OFF_MISC);
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + DW_OFF_MISC + 4);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int L;
    uint32_t t0, t1;
    dw_job(g, blockIdx.x, L, t0, t1);
    const bool wide = L >= 1 && L <= 3;     // N = 256
    const uint32_t n = wide ? 256u : 16u;
    const uint32_t tmem_cols = wide ? 512u : 32u;
    // the bias gradient: the column sums of A = dZ_L (L <= 3) or of B = dOut (L = 4)
    const unsigned char* Am = L == 4 ? g.z[3] : (L == 0 ? g.dz[0] : (L == 1 ? g.dz[1] : (L == 2 ? g.dz[2] : g.dz[3])));
    const unsigned char* Bm = L == 0 ? g.x0 : (L == 1 ? g.z[0] : (L == 2 ? g.z[1] : (L == 3 ? g.z[2] : g.dout)));
    const uint32_t a_tile = A_BYTES, b_tile = wide ? A_BYTES : X_TILE;
    const uint32_t b_half = b_tile / 2, b_lbo = wide ? A_SBO : X_SBO;
    const uint32_t n_stages = 2 * (t1 - t0);  // half tiles

    if (threadIdx.x == 0) {
        for (int s = 0; s < DW_STAGES; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_conv + 8 * s, 32 * DW_EPI_WARPS);  // every epilogue thread
            mbar_init(bar_empty + 8 * s, 1);                 // the MMA commit
        }
        mbar_init(bar_done, 1);
        mbar_init(bar_drain, 1);
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + DW_OFF_MISC),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            bool ok = true;
            uint32_t j = 0;
            for (; j < n_stages && ok; ++j) {
                const uint32_t s = j % DW_STAGES, use = j / DW_STAGES;
                if (use > 0 && !mbar_wait(bar_empty + 8 * s, (use - 1) & 1u, abort_flag)) { ok = false; break; }
                const uint32_t tile = t0 + j / 2, hf = j & 1u;
                const uint32_t dst = sbase + s * DW_STAGE;
                mbar_expect_tx(bar_full + 8 * s, DW_A_BYTES + b_half);
                bulk_g2s(dst, Am + size_t(tile) * a_tile + hf * DW_A_BYTES, DW_A_BYTES, bar_full + 8 * s);
                bulk_g2s(dst + DW_A_BYTES, Bm + size_t(tile) * b_tile + hf * b_half, b_half, bar_full + 8 * s);
            }
            const uint32_t first = j > DW_STAGES ? j - DW_STAGES : 0;
            for (uint32_t k = first; k < j; ++k) {
                const uint32_t s = k % DW_STAGES, use = k / DW_STAGES;
                for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_full + 8 * s, use & 1u); ++it) {}
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = true;
            const uint32_t idesc = idesc_bf16_major(TM, n, true, true);
            for (uint32_t j = 0; j < n_stages && ok; ++j) {
                const uint32_t s = j % DW_STAGES, use = j / DW_STAGES;
                if (!mbar_wait(bar_conv + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t sa = sbase + s * DW_STAGE, sb = sa + DW_A_BYTES;
                // 64 rows of K: 4 steps of 16 rows, two 8-row groups each
                for (uint32_t ks = 0; ks < 4; ++ks)
                    for (uint32_t mh = 0; mh < 2; ++mh) {
                        // A: M-major, the M half starts 16 column groups (2 KB) in
                        const uint64_t a = smem_desc(sa + mh * 2048u + ks * 2u * A_SBO, A_SBO, 128u);
                        const uint64_t b = smem_desc(sb + ks * 2u * b_lbo, b_lbo, 128u);
                        mma_bf16_ss(tmem + mh * n, a, b, idesc, (j > 0 || ks > 0) ? 1u : 0u);
                    }
                mma_commit(bar_empty + 8 * s);
            }
            if (ok) mma_commit(bar_done);
            mma_commit(bar_drain);
            for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_drain, 0); ++it) {}
        }
    } else {
        // per stage: H = silu(Z) in place of the staged Z half tile, the
        // column sums for the bias gradient; then the partial out of TMEM
        const uint32_t ew = warp - 2;  // 0..7
        const uint32_t et = threadIdx.x - 64;
        // column sums: L <= 3, warp ew sums the 8-column groups 4 ew .. 4 ew + 3
        // of A (lane: group 4 ew + lane % 4, row lane / 4 of each 8-row group);
        // L = 4, warp ew the 8-row group ew of B (lanes 0-15: group lane / 8,
        // row lane % 8)
        float csum[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) csum[e] = 0.f;
        bool ok = true;
        for (uint32_t j = 0; j < n_stages && ok; ++j) {
            const uint32_t s = j % DW_STAGES, use = j / DW_STAGES;
            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
            unsigned char* sa = smem + s * DW_STAGE;
            unsigned char* sb = sa + DW_A_BYTES;
            if (L >= 1) {
                // the 32 KB half tile of Z (B for L = 1..3, A for L = 4) -> H
                uint4* zt = reinterpret_cast<uint4*>(L == 4 ? sa : sb);
#pragma unroll 2
                for (uint32_t k = 0; k < DW_A_BYTES / 16 / (32 * DW_EPI_WARPS); ++k) {
                    const uint4 v = zt[et + k * 32 * DW_EPI_WARPS];
                    zt[et + k * 32 * DW_EPI_WARPS] =
                        uint4{silu_bf16x2(v.x), silu_bf16x2(v.y), silu_bf16x2(v.z), silu_bf16x2(v.w)};
                }
            }
            if (L <= 3) {
                const unsigned char* a = sa + (4 * ew + (lane & 3u)) * 128u + (lane >> 2) * 16u;
#pragma unroll
                for (uint32_t rg = 0; rg < 8; ++rg) {
                    const uint4 v = *reinterpret_cast<const uint4*>(a + rg * A_SBO);
                    add_bf16x2(csum[0], csum[1], v.x);
                    add_bf16x2(csum[2], csum[3], v.y);
                    add_bf16x2(csum[4], csum[5], v.z);
                    add_bf16x2(csum[6], csum[7], v.w);
                }
            } else if (lane < 16) {
                const uint4 v = *reinterpret_cast<const uint4*>(sb + ew * X_SBO + (lane >> 3) * 128u + (lane & 7u) * 16u);
                add_bf16x2(csum[0], csum[1], v.x);
                add_bf16x2(csum[2], csum[3], v.y);
                add_bf16x2(csum[4], csum[5], v.z);
                add_bf16x2(csum[6], csum[7], v.w);
            }
            fence_proxy_async();
            mbar_arrive(bar_conv + 8 * s);
        }
        float* part = g.part + size_t(blockIdx.x) * DW_PART;
        if (L <= 3) {
            // sum over the 8 rows of a group (lanes of equal lane % 4)
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 4);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 8);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 16);
            }
            if (lane < 4) {
                float* dst = part + MLP_HID * MLP_HID + (4 * ew + lane) * 8;
#pragma unroll
                for (int e = 0; e < 8; ++e) dst[e] = csum[e];
            }
        } else {
            // over the rows of the group (lane % 8), then over the warps in order
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 1);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 2);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 4);
            }
            float* red = reinterpret_cast<float*>(smem + DW_OFF_RED);
            if (lane == 0 || lane == 8) {
#pragma unroll
                for (int e = 0; e < 8; ++e) red[ew * 16 + (lane >> 3) * 8 + e] = csum[e];
            }
            asm volatile("bar.sync 1, %0;" ::"n"(32 * DW_EPI_WARPS) : "memory");
            if (ew == 0 && lane < 16) {
                float t = 0.f;
                for (int k = 0; k < DW_EPI_WARPS; ++k) t += red[k * 16 + lane];
                part[MLP_HID * MLP_HID + lane] = t;
            }
        }
        if (ok && mbar_wait(bar_done, 0, abort_flag)) {
            tc_fence_after();
            // a warp reads the TMEM lanes of its place in its warpgroup,
            // 32 (warp % 4) ..; warps 2-5 take M half 0, warps 6-9 half 1
            const uint32_t q = warp & 3u, mh = ew >> 2;
            const uint32_t m = mh * 128 + q * 32 + lane;  // result row
            const uint32_t base = tmem + ((q * 32u) << 16) + mh * n;
            float* dst = part + size_t(m) * n;
            for (uint32_t c = 0; c < n; c += 16) {
                uint32_t v[16];
                tmem_ld16(base + c, v);
                tmem_wait_ld(v);
#pragma unroll
                for (int k = 0; k < 16; k += 4)
                    *reinterpret_cast<float4*>(dst + c + k) =
                        make_float4(__uint_as_float(v[k]), __uint_as_float(v[k + 1]), __uint_as_float(v[k + 2]),
                                    __uint_as_float(v[k + 3]));
            }
            tc_fence_before();
        }
    }
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(g.status, 2u);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

// grad = the sum of the jobs' partials: W1..W5 (W5 from its transpose) and
// b1..b5; one thread per gradient element, the jobs summed in order.
__global__ void __launch_bounds__(256) k_mlp_dw_reduce(const float* __restrict__ part, uint32_t jobs_heavy,
                                                       uint32_t jobs_light, float* __restrict__ grad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // element i of [W2 | W3 | W4 | W1 | W5 | b1 | b2 | b3 | b4 | b5]
    constexpr uint32_t NW = MLP_HID * MLP_HID, NS = MLP_HID * MLP_IN_PAD;
    uint32_t j0, nj, src, dst;
    if (i < 3 * NW) {
        const uint32_t L = 1 + i / NW, e = i % NW;
        j0 = (L - 1) * jobs_heavy; nj = jobs_heavy; src = e; dst = mlp_w_off(int(L)) + e;
    } else if (i < 3 * NW + NS) {
        const uint32_t e = i - 3 * NW;  // dW1 [256][16]
        j0 = 3 * jobs_heavy; nj = jobs_light; src = e; dst = mlp_w_off(0) + e;
    } else if (i < 3 * NW + 2 * NS) {
        const uint32_t e = i - 3 * NW - NS;  // dW5 [16][256] from dW5^T [256][16]
        const uint32_t o = e / MLP_HID, in = e % MLP_HID;
        j0 = 3 * jobs_heavy + jobs_light; nj = jobs_light; src = in * MLP_OUT_PAD + o; dst = mlp_w_off(4) + e;
    } else if (i < 3 * NW + 2 * NS + 4 * MLP_HID) {
        const uint32_t e = i - 3 * NW - 2 * NS, L = e / MLP_HID, c = e % MLP_HID;
        j0 = L == 0 ? 3 * jobs_heavy : (L - 1) * jobs_heavy;
        nj = L == 0 ? jobs_light : jobs_heavy;
        src = NW + c; dst = mlp_b_off(int(L)) + c;
    } else if (i < 3 * NW + 2 * NS + 4 * MLP_HID + MLP_OUT_PAD) {
        const uint32_t c = i - 3 * NW - 2 * NS - 4 * MLP_HID;  // b5 from the dOut column sums
        j0 = 3 * jobs_heavy + jobs_light; nj = jobs_light; src = NW + c; dst = mlp_b_off(4) + c;
    } else {
        return;
    }
    float s = 0.f;
#pragma unroll 4
    for (uint32_t k = 0; k < nj; ++k) s += part[size_t(j0 + k) * DW_PART + src];
    grad[dst] = s;
}

}  // namespace

// ------------------------------------------------------------ launchers
size_t mlp_dw_partial_floats(uint32_t jobs) { return size_t(jobs) * DW_PART; }

cudaError_t launch_mlp_fwd_stash_tc(const void* img, const float* params, const void* x0_tiles, void* const* z,
                                    float* out, const SampleLabel* lab, const LossWeights& w, void* dout_tiles,
                                    float* loss_acc, uint32_t n_tiles, uint32_t* status, int sm_count,
                                    cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_chain_tc<FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             CH_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img);
    a.params = params;
    a.in = static_cast<const unsigned char*>(x0_tiles);
    for (int l = 0; l < 4; ++l) a.z[l] = static_cast<unsigned char*>(z[l]);
    a.out = out;
    a.lab = lab;
    a.w = w;
    a.dout = static_cast<unsigned char*>(dout_tiles);
    a.loss_acc = loss_acc;
    a.n_tiles = n_tiles;
    a.status = status;
    if (lab && !dout_tiles) return cudaErrorInvalidValue;
    const uint32_t grid = n_tiles < uint32_t(sm_count) ? n_tiles : uint32_t(sm_count);
    if (grid == 0) return cudaSuccess;
    k_mlp_chain_tc<FWD><<<grid, CH_THREADS, CH_SMEM, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_mlp_bwd_dx_tc(const void* img, const void* dout_tiles, void* const* z, void* const* dz,
                                 uint32_t n_tiles, uint32_t* status, int sm_count, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_chain_tc<BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             CH_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img);
    a.in = static_cast<const unsigned char*>(dout_tiles);
    for (int l = 0; l < 4; ++l) {
        a.z[l] = static_cast<unsigned char*>(z[l]);
        a.dz[l] = static_cast<unsigned char*>(dz[l]);
    }
    a.n_tiles = n_tiles;
    a.status = status;
    const uint32_t grid = n_tiles < uint32_t(sm_count) ? n_tiles : uint32_t(sm_count);
    if (grid == 0) return cudaSuccess;
    k_mlp_chain_tc<BWD><<<grid, CH_THREADS, CH_SMEM, st>>>(a);
    return cudaGetLastError();
}

void mlp_dw_jobs(uint32_t n_tiles, int sm_count, uint32_t* heavy, uint32_t* light) {
    // per tile a dW job of the 256-column layers moves 128 KB and does
    // 16.8 MFLOP, a 16-column one 68 KB and 1 MFLOP: about 3 : 1 in CTAs
    uint32_t sms = uint32_t(sm_count > 8 ? sm_count : 8);
    uint32_t l = sms / 8, h = (sms - 2 * l) / 3;
    if (h > n_tiles) h = n_tiles;
    if (l > n_tiles) l = n_tiles;
    *heavy = h ? h : 1;
    *light = l ? l : 1;
}

cudaError_t launch_mlp_dw_tc(void* const* dz, void* const* z, const void* x0_tiles, const void* dout_tiles,
                             float* part, float* grad, uint32_t n_tiles, uint32_t jobs_heavy, uint32_t jobs_light,
                             uint32_t* status, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, DW_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    DwArgs a{};
    for (int l = 0; l < 4; ++l) {
        a.dz[l] = static_cast<const unsigned char*>(dz[l]);
        a.z[l] = static_cast<const unsigned char*>(z[l]);
    }
    a.x0 = static_cast<const unsigned char*>(x0_tiles);
    a.dout = static_cast<const unsigned char*>(dout_tiles);
    a.part = part;
    a.n_tiles = n_tiles;
    a.jobs_heavy = jobs_heavy;
    a.jobs_light = jobs_light;
    a.status = status;
    if (n_tiles == 0) return cudaSuccess;
    const uint32_t jobs = 3 * jobs_heavy + 2 * jobs_light;
    k_mlp_dw_tc<<<jobs, DW_THREADS, DW_SMEM, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint32_t n_out = 3 * MLP_HID * MLP_HID + 2 * MLP_HID * MLP_IN_PAD + 4 * MLP_HID + MLP_OUT_PAD;
    k_mlp_dw_reduce<<<(n_out + 255) / 256, 256, 0, st>>>(part, jobs_heavy, jobs_light, grad);
    return cudaGetLastError();
}

}  // namespace mgk
