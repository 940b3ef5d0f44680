// Weight gradients of the deflection surrogate's training on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory,
// operands brought in by bulk copies), for one batch of B rows (a multiple
// of 128).  The forward with stash and the input-gradient chain are the
// FWD and BWD chains of mlp_tc.cu.
//
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
// the weight gradients.
//
// H is rounded to BF16 as the forward rounds it, from the BF16 Z: silu of
// the rounded z, which differs from the forward's silu(z) by at most about
// one BF16 ulp.
//
// Every mbarrier wait is bounded (tc::mbar_wait); a timeout sets bit 1 of
// *status, the other roles leave their loops, the CTA drains its copies and
// MMAs and frees its tensor memory.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.h"
#include "mlp_act.cuh"
#include "tc_sm100.cuh"

namespace mgk {
namespace {

using namespace tc;
using namespace act;

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
// The ring: 3 stages of 64 KB for a 256-column layer, 5 of 36 KB for W1 and
// W5 (whose B half tile is 2 KB), in the same 192 KB.
constexpr uint32_t DW_A_BYTES = 32768, DW_B_BYTES = 32768;
constexpr uint32_t DW_RING = 3 * (DW_A_BYTES + DW_B_BYTES);
constexpr int DW_MAX_SLOTS = 5;
constexpr uint32_t DW_LIGHT_STAGE = DW_A_BYTES + 4096;
static_assert(DW_MAX_SLOTS * DW_LIGHT_STAGE <= DW_RING, "light ring");
constexpr int DW_EPI_WARPS = 16;
constexpr int DW_THREADS = 32 * (2 + DW_EPI_WARPS);
constexpr uint32_t DW_OFF_BAR = DW_RING;  // full, empty, conv per slot; done; drain
constexpr uint32_t DW_OFF_MISC = DW_OFF_BAR + 32 * 8;
constexpr uint32_t DW_OFF_RED = DW_OFF_MISC + 16;             // [8 row groups][16] output-bias sums
constexpr uint32_t DW_SMEM = DW_OFF_RED + 8 * 16 * 4 + 128;
static_assert(DW_SMEM <= 232448, "shared memory");
constexpr uint32_t DW_PART = MLP_DW_PART;  // floats per job: the partial dW and bias sums

struct DwArgs {
    const unsigned char* dz[4];  // dZ1..dZ4 tiles
    const unsigned char* z[4];   // Z1..Z4 tiles (H = silu(Z) is made in shared memory)
    const unsigned char* x0;     // X0 tiles (16 columns)
    const unsigned char* dout;   // dOut tiles (16 columns)
    float* part;                 // [jobs][DW_PART]
    uint32_t n_tiles;
    DwJobs jobs;
    uint32_t* status;
};

__device__ __forceinline__ void dw_job(const DwArgs& g, uint32_t j, int& L, uint32_t& t0, uint32_t& t1) {
    uint32_t per, k;
    if (j < 3 * g.jobs.heavy) {
        L = 1 + int(j / g.jobs.heavy);
        per = g.jobs.heavy;
        k = j % g.jobs.heavy;
    } else if (j < 3 * g.jobs.heavy + g.jobs.l0) {
        L = 0;
        per = g.jobs.l0;
        k = j - 3 * g.jobs.heavy;
    } else {
        L = 4;
        per = g.jobs.l4;
        k = j - 3 * g.jobs.heavy - g.jobs.l0;
    }
    t0 = uint32_t(uint64_t(g.n_tiles) * k / per);
    t1 = uint32_t(uint64_t(g.n_tiles) * (k + 1) / per);
}

__global__ void __launch_bounds__(DW_THREADS, 1) k_mlp_dw_tc(DwArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t sbase = smem_addr(smem);
    const uint32_t bar_full = sbase + DW_OFF_BAR, bar_empty = bar_full + DW_MAX_SLOTS * 8;
    const uint32_t bar_conv = bar_empty + DW_MAX_SLOTS * 8;
    const uint32_t bar_done = bar_conv + DW_MAX_SLOTS * 8, bar_drain = bar_done + 8;
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
    const uint32_t n_slot = wide ? 3u : uint32_t(DW_MAX_SLOTS);
    const uint32_t stage = wide ? DW_A_BYTES + DW_B_BYTES : DW_LIGHT_STAGE;

    if (threadIdx.x == 0) {
        for (int s = 0; s < DW_MAX_SLOTS; ++s) {
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
    // everything above overlaps the previous kernel's tail when launched as its dependent
    grid_dependency_wait();

    if (warp == 0) {
        if (lane == 0) {
            bool ok = true;
            uint32_t j = 0;
            for (; j < n_stages && ok; ++j) {
                const uint32_t s = j % n_slot, use = j / n_slot;
                if (use > 0 && !mbar_wait(bar_empty + 8 * s, (use - 1) & 1u, abort_flag)) { ok = false; break; }
                const uint32_t tile = t0 + j / 2, hf = j & 1u;
                const uint32_t dst = sbase + s * stage;
                mbar_expect_tx(bar_full + 8 * s, DW_A_BYTES + b_half);
                bulk_g2s(dst, Am + size_t(tile) * a_tile + hf * DW_A_BYTES, DW_A_BYTES, bar_full + 8 * s);
                bulk_g2s(dst + DW_A_BYTES, Bm + size_t(tile) * b_tile + hf * b_half, b_half, bar_full + 8 * s);
            }
            const uint32_t first = j > n_slot ? j - n_slot : 0;
            for (uint32_t k = first; k < j; ++k) {
                const uint32_t s = k % n_slot, use = k / n_slot;
                for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_full + 8 * s, use & 1u); ++it) {}
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = true;
            const uint32_t idesc = idesc_bf16_major(TM, n, true, true);
            for (uint32_t j = 0; j < n_stages && ok; ++j) {
                const uint32_t s = j % n_slot, use = j / n_slot;
                if (!mbar_wait(bar_conv + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t sa = sbase + s * stage, sb = sa + DW_A_BYTES;
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
        const uint32_t ew = warp - 2;  // 0..15
        const uint32_t et = threadIdx.x - 64;
        // column sums: L <= 3, warp ew sums the 8-column groups 2 ew, 2 ew + 1
        // of A (lane: group 2 ew + lane % 2, row (lane / 2) % 8 of the 8-row
        // groups 4 (lane / 16) .. + 3); L = 4, warp ew < 8 the 8-row group ew
        // of B (lanes 0-15: group lane / 8, row lane % 8)
        float csum[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) csum[e] = 0.f;
        bool ok = true;
        for (uint32_t j = 0; j < n_stages && ok; ++j) {
            const uint32_t s = j % n_slot, use = j / n_slot;
            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
            unsigned char* sa = smem + s * stage;
            unsigned char* sb = sa + DW_A_BYTES;
            if (L >= 1) {
                // the 32 KB half tile of Z (B for L = 1..3, A for L = 4) -> H
                uint4* zt = reinterpret_cast<uint4*>(L == 4 ? sa : sb);
#pragma unroll
                for (uint32_t k = 0; k < DW_A_BYTES / 16 / (32 * DW_EPI_WARPS); ++k) {
                    const uint4 v = zt[et + k * 32 * DW_EPI_WARPS];
                    zt[et + k * 32 * DW_EPI_WARPS] =
                        uint4{silu_bf16x2(v.x), silu_bf16x2(v.y), silu_bf16x2(v.z), silu_bf16x2(v.w)};
                }
            }
            if (L <= 3) {
                const unsigned char* a =
                    sa + (2 * ew + (lane & 1u)) * 128u + ((lane >> 1) & 7u) * 16u + (lane >> 4) * 4u * A_SBO;
#pragma unroll
                for (uint32_t rg = 0; rg < 4; ++rg) {
                    const uint4 v = *reinterpret_cast<const uint4*>(a + rg * A_SBO);
                    add_bf16x2(csum[0], csum[1], v.x);
                    add_bf16x2(csum[2], csum[3], v.y);
                    add_bf16x2(csum[4], csum[5], v.z);
                    add_bf16x2(csum[6], csum[7], v.w);
                }
            } else if (ew < 8 && lane < 16) {
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
            // sum over the rows (lanes of equal lane % 2)
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 2);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 4);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 8);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 16);
            }
            if (lane < 2) {
                float* dst = part + MLP_HID * MLP_HID + (2 * ew + lane) * 8;
#pragma unroll
                for (int e = 0; e < 8; ++e) dst[e] = csum[e];
            }
        } else {
            // over the rows of the group (lane % 8), then over the row groups in order
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 1);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 2);
                csum[e] += __shfl_xor_sync(0xFFFFFFFFu, csum[e], 4);
            }
            float* red = reinterpret_cast<float*>(smem + DW_OFF_RED);
            if (ew < 8 && (lane == 0 || lane == 8)) {
#pragma unroll
                for (int e = 0; e < 8; ++e) red[ew * 16 + (lane >> 3) * 8 + e] = csum[e];
            }
            asm volatile("bar.sync 1, %0;" ::"n"(32 * DW_EPI_WARPS) : "memory");
            if (ew == 0 && lane < 16) {
                float t = 0.f;
                for (int k = 0; k < 8; ++k) t += red[k * 16 + lane];
                part[MLP_HID * MLP_HID + lane] = t;
            }
        }
        if (ok && mbar_wait(bar_done, 0, abort_flag)) {
            tc_fence_after();
            // a warp reads the TMEM lanes of its place in its warpgroup,
            // 32 (warp % 4) ..: M half (ew / 4) % 2, column half ew / 8 (for
            // N = 16 only the first)
            const uint32_t q = warp & 3u, mh = (ew >> 2) & 1u, ch = ew >> 3;
            const uint32_t m = mh * 128 + q * 32 + lane;  // result row
            const uint32_t base = tmem + ((q * 32u) << 16) + mh * n;
            float* dst = part + size_t(m) * n;
            const uint32_t c0 = n == 256u ? ch * 128u : 0u, c1 = n == 256u ? c0 + 128u : (ch == 0 ? n : 0u);
            for (uint32_t c = c0; c < c1; c += 16) {
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
    grid_dependents_go();
    if (*abort_flag && threadIdx.x == 0) atomicOr(g.status, 2u);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

// grad = the sum of the jobs' partials, one thread per parameter, the jobs
// summed in order (mlp_dw_source).
__global__ void __launch_bounds__(256) k_mlp_dw_reduce(const float* __restrict__ part, DwJobs jobs,
                                                       float* __restrict__ grad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PARAMS) return;
    uint32_t j0, nj, src;
    mlp_dw_source(i, jobs, &j0, &nj, &src);
    float s = 0.f;
#pragma unroll 4
    for (uint32_t k = 0; k < nj; ++k) s += part[size_t(j0 + k) * DW_PART + src];
    grad[i] = s;
}

}  // namespace

// ------------------------------------------------------------ launchers
size_t mlp_dw_partial_floats(uint32_t jobs) { return size_t(jobs) * DW_PART; }

DwJobs mlp_dw_jobs(uint32_t n_tiles, int sm_count) {
    // CTAs in proportion to a tile's cost in each kind of job (measured on
    // B200 from the spans of the jobs: 2.95, 1.55 and 1.90 us per tile for a
    // 256-column layer, W1 and W5), so that the jobs end together
    const uint32_t sms = uint32_t(sm_count > 8 ? sm_count : 8);
    const double unit = double(sms) / (3 * 2.95 + 1.55 + 1.90);
    uint32_t l4 = uint32_t(unit * 1.90 + 0.5), l0 = uint32_t(unit * 1.55 + 0.5);
    uint32_t h = (sms - l0 - l4) / 3;
    DwJobs j;
    j.heavy = h < 1 ? 1 : (h > n_tiles ? n_tiles : h);
    j.l0 = l0 < 1 ? 1 : (l0 > n_tiles ? n_tiles : l0);
    j.l4 = l4 < 1 ? 1 : (l4 > n_tiles ? n_tiles : l4);
    return j;
}

cudaError_t launch_mlp_dw_tc(void* const* dz, void* const* z, const void* x0_tiles, const void* dout_tiles,
                             float* part, float* grad, uint32_t n_tiles, const DwJobs& jobs, uint32_t* status,
                             cudaStream_t st, bool reduce, bool pdl) {
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
    a.jobs = jobs;
    a.status = status;
    if (n_tiles == 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3(jobs.total(), 1, 1);
    cfg.blockDim = dim3(DW_THREADS, 1, 1);
    cfg.dynamicSmemBytes = DW_SMEM;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_mlp_dw_tc, a);
    if (e != cudaSuccess) return e;
    if (!reduce) return cudaSuccess;
    k_mlp_dw_reduce<<<(MLP_PARAMS + 255) / 256, 256, 0, st>>>(part, jobs, grad);
    return cudaGetLastError();
}

}  // namespace mgk
