// Fused inference of the deflection surrogate on the 5th-generation tensor
// cores: all five layers of a tile of 128 rows run in one CTA, accumulators
// in tensor memory, activations resident in shared memory between layers.
// Each CTA keeps two tiles in flight (buffers 0 and 1, two 256-column TMEM
// accumulators) so that the epilogue of one tile overlaps the MMAs of the
// other.
//
//  warp 0      producer: streams the weight image in chunks of at most 32 KB
//              into a 2-slot shared-memory ring (cp.async.bulk + mbarrier
//              transaction counts), in the order the MMA warp consumes them.
//  warp 1      allocates 512 TMEM columns; lane 0 issues tcgen05.mma
//              (M = 128, K = 16 per instruction, N = 256 or 16), layer by
//              layer alternating between the two tiles, and commits each
//              chunk to its slot's "empty" barrier and each layer to the
//              tile's "d_ready" barrier.
//  warps 2..9  epilogue of buffer 0, warps 10..17 of buffer 1: tcgen05.ld
//              of the accumulator (warp w reads TMEM lanes 32 (w % 4) ..;
//              the first four warps of a buffer columns 0-127, the other four
//              128-255), bias + SiLU, BF16 back into the tile's activations,
//              or the 16 FP32 outputs of the last layer to global memory.
//
// SiLU is evaluated as u (1 + tanh u) with u = z / 2, on pairs of values in
// BF16x2 (one tanh.approx.bf16x2 and one fma.rn.bf16x2 per pair, u rounded
// to BF16 first: about one BF16 ulp of extra error on the activations).  The image holds the weights of the four SiLU layers halved (exact
// in BF16) and the biases are staged halved, so u = accumulator + bias.
//
// Operand layout in shared memory (both operands K-major, no swizzle): the
// canonical 8 x 16-byte core matrices, element (row, k) of a tile at
//   (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// so a K step of 16 advances the descriptor start by 256 bytes.  The weight
// image in global memory is stored chunk by chunk in exactly this layout, so
// each chunk is one contiguous bulk copy.
//
// Every wait on an mbarrier is bounded; on a timeout the kernel sets bit 1 of
// *status, lets the other roles leave their loops, waits (bounded) for its
// own bulk copies and MMAs, frees its TMEM and returns.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.h"
#include "tc_sm100.cuh"

namespace mgk {
namespace {

using namespace tc;

constexpr int TM = 128;                   // rows per tile
// A bulk copy costs about the same time whatever its size up to 32 KB, so the
// ring uses few large slots rather than many small ones.
constexpr int N_SLOT = 2;
constexpr uint32_t SLOT_BYTES = 32768;
constexpr uint32_t A_BYTES = TM * MLP_HID * 2;  // 64 KB activation tile
constexpr uint32_t A_SBO = 4096;                // 8-row group stride of the activation tile
constexpr int N_CHUNKS = MLP_IMAGE_CHUNKS;      // W1, W2 x4, W3 x4, W4 x4, W5
constexpr int EPI_WARPS = 16;                   // 8 per buffer
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t TMEM_COLS = 512;             // two 256-column accumulators

// Shared-memory map (dynamic, offsets from a 128-byte aligned base).
constexpr uint32_t OFF_A = 0;                                // two activation tiles
constexpr uint32_t OFF_W = OFF_A + 2 * A_BYTES;              // weight ring
constexpr uint32_t OFF_BIAS = OFF_W + N_SLOT * SLOT_BYTES;   // b1..b4 halved, b5
constexpr uint32_t N_BIAS = 4 * MLP_HID + MLP_OUT_PAD;
constexpr uint32_t OFF_BAR = OFF_BIAS + N_BIAS * 4;          // full[2], empty[2], d_ready[2], a_ready[2], drain
constexpr uint32_t OFF_MISC = OFF_BAR + 16 * 8;              // tmem base, abort flag
static_assert(2 * N_SLOT + 5 <= 16, "barrier area");
constexpr uint32_t SMEM_BYTES = OFF_MISC + 16 + 128;         // + alignment slack
static_assert(SMEM_BYTES <= 232448, "shared memory");

// Chunk c of the weight image (mlp.h): byte offset and size.
__host__ __device__ constexpr uint32_t chunk_offset(int c) { return mlp_chunk_offset(c); }
__host__ __device__ constexpr uint32_t chunk_bytes(int c) { return mlp_chunk_bytes(c); }
constexpr uint32_t IMAGE_BYTES = MLP_IMAGE_BYTES;

// silu of a pair with u = z / 2:  z sigmoid(z) = u (1 + tanh u), in BF16x2.
__device__ __forceinline__ uint32_t silu_half_pair(float u0, float u1) {
    const uint32_t u = pack_bf16(u0, u1);
    uint32_t t, h;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(u));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(u), "r"(t));
    return h;
}

// Bias + SiLU of 32 accumulator columns of one row into the activation tile.
__device__ __forceinline__ void epilogue_block(const uint32_t (&v)[32], const float* hb, unsigned char* dst0) {
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        uint32_t pk[4];
#pragma unroll
        for (int e = 0; e < 4; e += 2) {
            const int c = g * 8 + 2 * e;
            const float4 bb = *reinterpret_cast<const float4*>(hb + c);
            pk[e] = silu_half_pair(__uint_as_float(v[c]) + bb.x, __uint_as_float(v[c + 1]) + bb.y);
            pk[e + 1] = silu_half_pair(__uint_as_float(v[c + 2]) + bb.z, __uint_as_float(v[c + 3]) + bb.w);
        }
        *reinterpret_cast<uint4*>(dst0 + g * 128) = uint4{pk[0], pk[1], pk[2], pk[3]};
    }
}


}  // namespace

// Weight image for the fused kernel from the BF16 parameter copy (offsets of
// the flat parameter vector, weights [out][in]).
__global__ void k_weight_image(const __nv_bfloat16* __restrict__ wb, unsigned char* __restrict__ img) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // one BF16 element of the image
    if (i >= IMAGE_BYTES / 2) return;
    const uint32_t byte = i * 2;
    int c = 0;
    while (c < N_CHUNKS - 1 && byte >= chunk_offset(c + 1)) ++c;
    const uint32_t o = byte - chunk_offset(c);
    // invert kmaj for the chunk's shape
    uint32_t sbo, layer, k_base;
    if (c == 0) { sbo = 256; layer = 0; k_base = 0; }
    else if (c == 13) { sbo = 4096; layer = 4; k_base = 0; }
    else { sbo = 1024; layer = 1 + (c - 1) / 4; k_base = 64 * ((c - 1) % 4); }
    const uint32_t grp = o / sbo, rem = o % sbo;
    const uint32_t kc = rem / 128, r2 = rem % 128;
    const uint32_t row = grp * 8 + r2 / 16, k = kc * 8 + (r2 % 16) / 2;
    const uint32_t in_dim = layer == 0 ? MLP_IN_PAD : MLP_HID;
    const __nv_bfloat16 w = wb[mlp_w_off(int(layer)) + size_t(row) * in_dim + k_base + k];
    // layers followed by SiLU are stored halved (exact: a power-of-two scale)
    reinterpret_cast<__nv_bfloat16*>(img)[i] = layer < 4 ? __hmul(w, __float2bfloat16(0.5f)) : w;
}

__global__ void __launch_bounds__(THREADS, 1)
    k_mlp_infer_tc(const float* __restrict__ feat, uint32_t n, const unsigned char* __restrict__ img,
                   const float* __restrict__ params, float* __restrict__ out, uint32_t* status) {
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
    const uint32_t n_tiles = (n + TM - 1) / TM;
    const uint32_t my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t my_pairs = (my_tiles + 1) / 2;  // an odd count ends with an empty tile in buffer 1

    for (uint32_t i = threadIdx.x; i < N_BIAS; i += THREADS) {
        const int l = i < 4 * MLP_HID ? int(i / MLP_HID) : 4;
        const uint32_t k = i < 4 * MLP_HID ? i % MLP_HID : i - 4 * MLP_HID;
        bias[i] = l < 4 ? 0.5f * params[mlp_b_off(l) + k] : params[mlp_b_off(l) + k];
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
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        // chunk order: per tile pair, per layer, per buffer, the layer's chunks
        if (lane == 0) {
            uint32_t j = 0;
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < MLP_LAYERS && ok; ++l)
                    for (int b = 0; b < 2 && ok; ++b) {
                        const int c0 = l == 0 ? 0 : (l == 4 ? 13 : 1 + 4 * (l - 1));
                        const int nc = (l == 0 || l == 4) ? 1 : 4;
                        for (int ci = 0; ci < nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (use > 0 && !mbar_wait(bar_empty + 8 * s, (use - 1) & 1u, abort_flag)) {
                                ok = false;
                                break;
                            }
                            const int c = c0 + ci;
                            mbar_expect_tx(bar_full + 8 * s, chunk_bytes(c));
                            bulk_g2s(sbase + OFF_W + s * SLOT_BYTES, img + chunk_offset(c), chunk_bytes(c),
                                     bar_full + 8 * s);
                        }
                    }
            // drain: every issued copy has landed before the CTA may exit
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
                for (int l = 0; l < MLP_LAYERS && ok; ++l)
                    for (uint32_t b = 0; b < 2 && ok; ++b) {
                        if (!mbar_wait(bar_a + 8 * b, ar[b] & 1u, abort_flag)) { ok = false; break; }
                        ++ar[b];
                        tc_fence_after();
                        const int nc = (l == 0 || l == 4) ? 1 : 4;
                        const uint32_t idesc = idesc_bf16(TM, l == 4 ? MLP_OUT_PAD : MLP_HID);
                        const uint32_t b_sbo = l == 0 ? 256u : (l == 4 ? 4096u : 1024u);
                        const int ksteps = l == 0 ? 1 : (l == 4 ? 16 : 4);
                        const uint32_t a_base = sbase + OFF_A + b * A_BYTES;
                        const uint32_t d = tmem + b * 256u;
                        for (int ci = 0; ci < nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                            tc_fence_after();
                            const uint32_t wslot = sbase + OFF_W + s * SLOT_BYTES;
                            for (int ks = 0; ks < ksteps; ++ks) {
                                const uint32_t kk = uint32_t(ci * ksteps + ks);  // K step within the layer
                                const uint64_t a = smem_desc(a_base + kk * 256u, 128u, A_SBO);
                                const uint64_t bd = smem_desc(wslot + uint32_t(ks) * 256u, 128u, b_sbo);
                                mma_bf16_ss(d, a, bd, idesc, kk > 0 ? 1u : 0u);
                            }
                            mma_commit(bar_empty + 8 * s);
                        }
                        if (ok) mma_commit(bar_d + 8 * b);
                    }
            // all MMAs issued by this thread are complete before TMEM is freed
            mma_commit(bar_drain);
            for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_drain, 0); ++it) {}
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const uint32_t buf = (warp - 2) >> 3, q = warp & 3u, half = ((warp - 2) >> 2) & 1u;
        const uint32_t row = q * 32 + lane;
        const uint32_t t_lane = tmem + ((q * 32u) << 16) + buf * 256u;
        unsigned char* A = smem + OFF_A + buf * A_BYTES;
        const uint32_t bar_db = bar_d + 8 * buf, bar_ab = bar_a + 8 * buf;
        uint32_t dr = 0;
        bool ok = true;
        for (uint32_t t = buf; t < 2 * my_pairs && ok; t += 2) {
            const uint32_t tile = blockIdx.x + t * gridDim.x;  // >= n_tiles for the empty tile
            const uint32_t g_row = tile * TM + row;
            const bool valid = tile < n_tiles && g_row < n;
            // layer-1 input: features -> BF16, K padded to 16
            if (half == 0) {
                float f[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) f[k] = (valid && k < MLP_IN) ? feat[size_t(g_row) * MLP_IN + k] : 0.f;
                *reinterpret_cast<uint4*>(A + kmaj(row, 0, A_SBO)) =
                    uint4{pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7])};
                *reinterpret_cast<uint4*>(A + kmaj(row, 8, A_SBO)) = uint4{0u, 0u, 0u, 0u};
            }
            fence_proxy_async();
            mbar_arrive(bar_ab);
            for (int l = 0; l < MLP_LAYERS; ++l) {
                if (!mbar_wait(bar_db, dr & 1u, abort_flag)) { ok = false; break; }
                ++dr;
                tc_fence_after();
                if (l < 4) {
                    // 4 blocks of 32 columns, TMEM loads double-buffered
                    const float* hb = bias + l * MLP_HID + half * 128;
                    const uint32_t tc = t_lane + half * 128;
                    unsigned char* dst = A + kmaj(row, half * 128, A_SBO);
                    uint32_t va[32], vb[32];
                    tmem_ld32(tc, va);
                    tmem_wait_ld(va);
                    tmem_ld32(tc + 32, vb);
                    epilogue_block(va, hb, dst);
                    tmem_wait_ld(vb);
                    tmem_ld32(tc + 64, va);
                    epilogue_block(vb, hb + 32, dst + 4 * 128);
                    tmem_wait_ld(va);
                    tmem_ld32(tc + 96, vb);
                    epilogue_block(va, hb + 64, dst + 8 * 128);
                    tmem_wait_ld(vb);
                    epilogue_block(vb, hb + 96, dst + 12 * 128);
                    tc_fence_before();
                    fence_proxy_async();
                    mbar_arrive(bar_ab);
                } else if (half == 0) {
                    uint32_t v[16];
                    tmem_ld16(t_lane, v);
                    tmem_wait_ld(v);
                    tc_fence_before();
                    if (valid) {
                        const float* b5 = bias + 4 * MLP_HID;
                        float4* o = reinterpret_cast<float4*>(out + size_t(g_row) * MLP_OUT_PAD);
#pragma unroll
                        for (int g = 0; g < 4; ++g)
                            o[g] = make_float4(__uint_as_float(v[4 * g]) + b5[4 * g],
                                               __uint_as_float(v[4 * g + 1]) + b5[4 * g + 1],
                                               __uint_as_float(v[4 * g + 2]) + b5[4 * g + 2],
                                               __uint_as_float(v[4 * g + 3]) + b5[4 * g + 3]);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicOr(status, 2u);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

size_t mlp_image_bytes() { return IMAGE_BYTES; }

cudaError_t launch_weight_image(const __nv_bfloat16* wb, void* img, cudaStream_t st) {
    const uint32_t n = IMAGE_BYTES / 2;
    k_weight_image<<<(n + 255) / 256, 256, 0, st>>>(wb, static_cast<unsigned char*>(img));
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer_tc(const float* feat, uint32_t n, const void* img, const float* params, float* out,
                                uint32_t* status, int sm_count, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const uint32_t tiles = (n + TM - 1) / TM;
    const uint32_t grid = tiles < uint32_t(sm_count) ? tiles : uint32_t(sm_count);
    k_mlp_infer_tc<<<grid, THREADS, SMEM_BYTES, st>>>(feat, n, static_cast<const unsigned char*>(img), params, out,
                                                       status);
    return cudaGetLastError();
}

}  // namespace mgk
