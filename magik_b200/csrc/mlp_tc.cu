// The layer chains of the deflection surrogate on the 5th-generation tensor
// cores: all layers of a 128-row tile run in one CTA, accumulators in tensor
// memory, activations resident in shared memory between layers.  One kernel
// template, three chains:
//
//  INFER  inference: features (FP32) in, the 16 FP32 outputs out.
//  FWD    training forward: the batch's rows gathered from the sample set
//         through the epoch's order (X0 also to global memory for the weight
//         gradients); the pre-activations Z_1..Z_4 to the stash, then each
//         row's loss (mlp_loss.cuh) and the BF16 output gradient dOut / B;
//         the FP32 outputs only where asked for.
//  BWD    training input gradients: dOut tiles in;
//         dZ4 = (dOut W5) * silu'(Z4), dZ3 = (dZ4 W4) * silu'(Z3), ... dZ1.
//
// Each CTA is persistent (at most one per SM) and keeps two tiles in flight
// (buffers 0 and 1, two 256-column TMEM accumulators), so the epilogue of one
// overlaps the MMAs of the other.
//
// PAIR (opt-in, MGK_SURROGATE_PAIRS=1): clusters of two CTAs run
// cta_group::2 MMAs of M = 256 issued by the even CTA; each CTA holds its 128
// rows of the activation tile and half of every weight chunk (N rows
// 128 rank ..), its accumulator rows in its own tensor memory.  The odd CTA
// forwards the landing of its chunk halves and the writing of its activation
// rows to the even CTA's peer_full / peer_a barriers (remote mbarrier
// arrivals at cluster scope); the MMA commits arrive on the barriers of both
// CTAs (multicast); both CTAs meet at a cluster barrier after setting up
// their barriers and before freeing their memory.
//
//  warp 0       producer: streams the weight image in chunks of at most
//               32 KB into a 3-slot shared-memory ring (cp.async.bulk +
//               mbarrier transaction counts), in the order the MMA warp
//               consumes them.  BWD: it also prefetches each step's Z tile
//               into L2 a step ahead.
//  warp 1       allocates 512 TMEM columns; lane 0 issues tcgen05.mma
//               (M = 128, K = 16 per instruction, N = 256 or 16), step by
//               step alternating between the two tiles, and commits each
//               chunk to its slot's "empty" barrier and each step to the
//               tile's "d_ready" barrier.
//  warps 2..17  epilogue: all 16 warps take every step, in the MMA's order.
//               Warp w reads TMEM lanes 32 (w % 4) .. (the rows of its lane
//               quarter) and 64 of the 256 columns ((w - 2) / 4); the output
//               layer's 16 columns go to the first four warps, and the next
//               tile's input is loaded by the second four meanwhile.
//
// Weights: the image (mlp_chunk_offset, mlp.h) holds W1..W5 K-major for the
// forward; the transposed image holds W5^T, W4^T, W3^T, W2^T K-major for the
// backward, so both chains issue the same N = 256 MMAs.  Layers followed by
// SiLU are stored halved (exact in BF16): the accumulator is z / 2 - b / 2.
//
// SiLU: INFER evaluates u (1 + tanh u), u = z / 2, in BF16x2 (one
// tanh.approx.bf16x2 and one fma.rn.bf16x2 per pair, u rounded to BF16
// first: about one BF16 ulp of extra error on the activations); FWD and BWD
// in FP32 with tanh.approx.f32 (mlp_act.cuh), rounded to BF16 where stored.
//
// Operand layout in shared memory (both operands K-major, no swizzle): the
// canonical 8 x 16-byte core matrices, element (row, k) of a tile at
//   (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// so a K step of 16 advances the descriptor start by 256 bytes.  The weight
// images and the activation tiles in global memory are stored in exactly
// this layout, so each chunk or tile is one contiguous bulk copy.
//
// Every wait on an mbarrier is bounded; on a timeout the kernel sets bit 1 of
// *status, lets the other roles leave their loops, waits (bounded) for its
// own bulk copies and MMAs, frees its TMEM and returns.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.h"
#include "mlp_act.cuh"
#include "mlp_loss.cuh"
#include "tc_sm100.cuh"

namespace mgk {
namespace {

using namespace tc;
using namespace act;

constexpr int EPI_WARPS = 16;
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr uint32_t TMEM_COLS = 512;             // two 256-column accumulators
constexpr uint32_t IMAGE_BYTES = MLP_IMAGE_BYTES;
constexpr uint32_t T_IMAGE_BYTES = 8192u + 12u * 32768u;  // W5^T, then W4^T, W3^T, W2^T in 64-column slices

// The weight ring and the shared-memory map (dynamic, offsets from a
// 128-byte aligned base) of a single CTA (PAIR = false: whole chunks, 3
// slots of 32 KB) and of a CTA of a pair (its half of each chunk, 6 slots of
// 16 KB).  Barriers: full[slots], empty[slots], d_ready[2], a_ready[2],
// drain; for a pair also peer_full[slots] and peer_a[2] (the other CTA's
// chunk halves landed, its activation rows written).
template <bool PAIR> struct Layout {
    static constexpr int slots = PAIR ? 6 : 3;
    static constexpr uint32_t slot_bytes = PAIR ? 16384u : 32768u;
    static constexpr uint32_t off_a = 0;                                  // two activation tiles
    static constexpr uint32_t off_w = off_a + 2 * A_BYTES;                // weight ring
    static constexpr uint32_t off_bar = off_w + slots * slot_bytes;
    static constexpr uint32_t n_bar = (PAIR ? 3 : 2) * slots + (PAIR ? 7 : 5);
    static constexpr uint32_t off_misc = off_bar + ((n_bar * 8 + 127) / 128) * 128;  // tmem base, abort flag
    static constexpr uint32_t smem_bytes = off_misc + 16 + 128;          // + alignment slack
    static_assert(smem_bytes <= 232448, "shared memory");
};

enum { INFER = 0, FWD = 1, BWD = 2, FB = 3 };  // FB: forward then backward, per tile

}  // namespace

// The two weight images from the BF16 parameter copy (weights [out][in]):
// element i < IMAGE_BYTES / 2 of the forward image, the rest of the
// transposed image (img_t may be null: then only the forward image).
__global__ void k_weight_image(const __nv_bfloat16* __restrict__ wb, unsigned char* __restrict__ img,
                               unsigned char* __restrict__ img_t) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // one BF16 element of an image
    const bool tr = i >= IMAGE_BYTES / 2;
    if (tr) {
        i -= IMAGE_BYTES / 2;
        if (img_t == nullptr || i >= T_IMAGE_BYTES / 2) return;
    }
    const uint32_t byte = i * 2;
    int c = 0;
    while (c < MLP_IMAGE_CHUNKS - 1 && byte >= mlp_chunk_offset(c + 1)) ++c;
    const uint32_t o = byte - mlp_chunk_offset(c);
    // invert kmaj for the chunk's shape: (row, k) of a K-major chunk
    uint32_t sbo, layer, k_base;
    if (!tr) {
        if (c == 0) { sbo = 256; layer = 0; k_base = 0; }
        else if (c == 13) { sbo = 4096; layer = 4; k_base = 0; }
        else { sbo = 1024; layer = 1 + (c - 1) / 4; k_base = 64 * ((c - 1) % 4); }
    } else {
        if (c == 0) { sbo = 256; layer = 4; k_base = 0; }
        else { sbo = 1024; layer = 3 - (c - 1) / 4; k_base = 64 * ((c - 1) % 4); }
    }
    const uint32_t grp = o / sbo, rem = o % sbo;
    const uint32_t kc = rem / 128, r2 = rem % 128;
    const uint32_t row = grp * 8 + r2 / 16, k = kc * 8 + (r2 % 16) / 2;
    const uint32_t in_dim = layer == 0 ? MLP_IN_PAD : MLP_HID;
    // forward: row = output, k = input; transposed: row = input, k = output
    const size_t e = tr ? size_t(k_base + k) * in_dim + row : size_t(row) * in_dim + k_base + k;
    const __nv_bfloat16 w = wb[mlp_w_off(int(layer)) + e];
    // layers followed by SiLU are stored halved (exact: a power-of-two scale)
    const __nv_bfloat16 v = layer < 4 ? __hmul(w, __float2bfloat16(0.5f)) : w;
    reinterpret_cast<__nv_bfloat16*>(tr ? img_t : img)[i] = v;
}

namespace {

struct ChainArgs {
    const unsigned char* img;    // weight image (BWD: the transposed image)
    const unsigned char* img_t;  // FB: the transposed image of the backward steps
    const float* params;       // FP32 parameters (biases)
    const float* feat;         // INFER: features [n_rows][7]; FWD: the sample set's features
    const uint32_t* perm;      // FWD: the batch is rows perm[b0 ..] of the sample set
    uint32_t b0;
    unsigned char* x0;         // FWD: the batch's X0 tiles (16 columns, BF16), written
    const unsigned char* in;   // BWD: dOut tiles (16 columns)
    unsigned char* z[4];       // Z_1..Z_4 tiles (FWD writes, BWD reads)
    unsigned char* dz[4];      // BWD: dZ_1..dZ_4 tiles (written)
    float* out;                // INFER, FWD: outputs [rows][16] FP32 (FWD: may be null)
    const SampleLabel* lab;    // FWD: the sample set's labels for the fused loss (may be null)
    unsigned char* dout;       // FWD: dOut tiles, d(loss)/d(out) / B in BF16
    float* loss_acc;           // FWD: += the batch's mean loss
    const TrainCounters* ctr;  // FWD, counted run: the batch is batch ctr->batch (b0 added), the loss
                               // goes to loss_acc[ctr->epoch - 1]
    LossWeights w;
    uint32_t n_rows;
    uint32_t n_tiles;
    uint32_t* status;
};

// Step l of a tile: its weight chunks and the shape of their MMAs.  The
// backward's steps (W5^T, W4^T, W3^T, W2^T of the transposed image) have the
// forward's first four shapes.
struct Step {
    int c0, nc;      // first chunk, number of chunks
    int ksteps;      // K steps of 16 per chunk
    uint32_t n;      // MMA N
    uint32_t b_sbo;  // 8-row stride of the chunk
};
__device__ __forceinline__ Step step_of(int l) {
    if (l == 0) return Step{0, 1, 1, 256u, 256u};
    if (l == 4) return Step{13, 1, 16, 16u, 4096u};
    return Step{1 + 4 * (l - 1), 4, 4, 256u, 1024u};
}

// Epilogue of 16 accumulator columns of one row of a hidden layer (INFER,
// FWD): bias and SiLU into the next step's operand (8-column groups 128 bytes
// apart from `a`); FWD: Z to the stash at `zs` (null for the empty tile).
// Pairs of columns in FP32x2 arithmetic; z = 2 acc + b and u = acc + b / 2
// are single roundings (the scalings by 2 and 1/2 are exact).
template <int DIR>
__device__ __forceinline__ void hidden16(const uint32_t (&v)[16], const float* bl, unsigned char* a,
                                         unsigned char* zs) {
    const float2 half2 = make_float2(0.5f, 0.5f), two2 = make_float2(2.0f, 2.0f);
#pragma unroll
    for (int gq = 0; gq < 2; ++gq) {
        const float4 b0 = __ldg(reinterpret_cast<const float4*>(bl + gq * 8));
        const float4 b1 = __ldg(reinterpret_cast<const float4*>(bl + gq * 8 + 4));
        const float2 bp[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                              make_float2(b1.z, b1.w)};
        uint32_t hv[4], zv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c = gq * 8 + 2 * e;
            const float2 acc = make_float2(__uint_as_float(v[c]), __uint_as_float(v[c + 1]));
            if constexpr (DIR == INFER) {
                const float2 u = __ffma2_rn(half2, bp[e], acc);
                hv[e] = silu_half_pair(u.x, u.y);
                zv[e] = 0u;
            } else {
                const float2 z = __ffma2_rn(two2, acc, bp[e]);
                zv[e] = pack_bf16(z.x, z.y);
                const float2 u = __fmul2_rn(half2, z);
                const float2 h = __ffma2_rn(u, make_float2(tanh_approx(u.x), tanh_approx(u.y)), u);
                hv[e] = pack_bf16(h.x, h.y);
            }
        }
        *reinterpret_cast<uint4*>(a + gq * 128) = uint4{hv[0], hv[1], hv[2], hv[3]};
        if constexpr (DIR == FWD) {
            if (zs) *reinterpret_cast<uint4*>(zs + gq * 128) = uint4{zv[0], zv[1], zv[2], zv[3]};
        }
    }
}

// Epilogue of 16 accumulator columns of one row of the backward:
// dZ = scale acc * silu'(Z) for the BF16 Z of `z` (2 x 8 columns), into the
// next step's operand at `a` (null at the last step) and to global memory at
// `dz` (null for the empty tile).  silu'(z) = s (1 + z (1 - s)),
// s = (1 + tanh(z / 2)) / 2, in FP32x2.
__device__ __forceinline__ void backward16(const uint32_t (&v)[16], const uint4 (&z)[2], float scale,
                                           unsigned char* a, unsigned char* dz) {
    const float2 half2 = make_float2(0.5f, 0.5f), one2 = make_float2(1.0f, 1.0f), sc2 = make_float2(scale, scale);
#pragma unroll
    for (int gq = 0; gq < 2; ++gq) {
        const uint32_t zw[4] = {z[gq].x, z[gq].y, z[gq].z, z[gq].w};
        uint32_t hv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c = gq * 8 + 2 * e;
            const float2 zf = unpack_bf16(zw[e]);
            const float2 u = __fmul2_rn(half2, zf);
            const float2 s = __ffma2_rn(half2, make_float2(tanh_approx(u.x), tanh_approx(u.y)), half2);
            const float2 g = __fmul2_rn(s, __ffma2_rn(zf, __fadd2_rn(one2, make_float2(-s.x, -s.y)), one2));
            const float2 acc = make_float2(__uint_as_float(v[c]), __uint_as_float(v[c + 1]));
            const float2 d = __fmul2_rn(__fmul2_rn(sc2, acc), g);
            hv[e] = pack_bf16(d.x, d.y);
        }
        const uint4 h4 = uint4{hv[0], hv[1], hv[2], hv[3]};
        if (a) *reinterpret_cast<uint4*>(a + gq * 128) = h4;
        if (dz) *reinterpret_cast<uint4*>(dz + gq * 128) = h4;
    }
}

template <int DIR, bool PAIR>
__global__ void __launch_bounds__(THREADS, 1) k_mlp_chain_tc(ChainArgs g) {
    // steps per tile: FB runs the forward's five, then the backward's four
    constexpr int S = DIR == BWD ? MLP_LAYERS - 1 : (DIR == FB ? 2 * MLP_LAYERS - 1 : MLP_LAYERS);
    constexpr bool FWDLIKE = DIR == FWD || DIR == FB;  // gathers its input, stashes Z, takes the loss
    static_assert(!(PAIR && DIR == FB), "the forward-and-backward chain runs as single CTAs");
    // step l of a tile: a backward step?  Its index within its chain
    auto bwd_step = [](int l) { return DIR == BWD || (DIR == FB && l >= MLP_LAYERS); };
    auto step_in = [](int l) { return DIR == FB && l >= MLP_LAYERS ? l - MLP_LAYERS : l; };
    using LY = Layout<PAIR>;
    constexpr int N_SLOT = LY::slots;
    constexpr uint32_t SLOT_BYTES = LY::slot_bytes, OFF_A = LY::off_a, OFF_W = LY::off_w, OFF_MISC = LY::off_misc;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t sbase = smem_addr(smem);
    const uint32_t bar_full = sbase + LY::off_bar, bar_empty = bar_full + N_SLOT * 8;
    const uint32_t bar_d = bar_empty + N_SLOT * 8, bar_a = bar_d + 2 * 8, bar_drain = bar_a + 2 * 8;
    const uint32_t bar_pfull = bar_drain + 8, bar_pa = bar_pfull + N_SLOT * 8;  // PAIR only
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(smem + OFF_MISC);
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + OFF_MISC + 4);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_tiles = g.n_tiles;
    // work units: 128-row tiles, or for a pair 256-row tiles whose rows
    // 0-127 belong to the even CTA (rank 0, which issues the MMAs) and
    // 128-255 to the odd one
    const uint32_t rank = PAIR ? cluster_ctarank() : 0u;
    const uint32_t unit = PAIR ? blockIdx.x >> 1 : blockIdx.x, n_units = PAIR ? gridDim.x >> 1 : gridDim.x;
    const uint32_t units = PAIR ? (n_tiles + 1) / 2 : n_tiles;
    const uint32_t my_units = unit < units ? (units - 1 - unit) / n_units + 1 : 0;
    const uint32_t my_pairs = (my_units + 1) / 2;  // an odd count ends with an empty unit in buffer 1
    // the 128-row tile of this CTA in buffer b of pair p
    auto tile_of = [&](uint32_t p, uint32_t b) {
        const uint32_t u = unit + (2 * p + b) * n_units;
        return PAIR ? 2 * u + rank : u;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < N_SLOT; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bar_d + 8 * b, 1);
            mbar_init(bar_a + 8 * b, 32 * EPI_WARPS);
        }
        mbar_init(bar_drain, 1);
        if constexpr (PAIR) {
            for (int s = 0; s < N_SLOT; ++s) mbar_init(bar_pfull + 8 * s, 1);
            for (int b = 0; b < 2; ++b) mbar_init(bar_pa + 8 * b, EPI_WARPS);
        }
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // a pair: both CTAs' barriers are initialised before either signals the other's
    if constexpr (PAIR) cluster_sync();
    if (warp == 1) {
        if constexpr (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + OFF_MISC),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + OFF_MISC),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // everything above overlaps the previous kernel's tail when launched as its dependent
    grid_dependency_wait();
    // FWD: the batch's first row in the order, and where its loss goes
    const uint32_t b0 = g.b0 + (FWDLIKE && g.ctr ? g.ctr->batch * g.n_rows : 0u);
    float* const loss_dst = FWDLIKE && g.loss_acc ? g.loss_acc + (g.ctr ? g.ctr->epoch - 1u : 0u) : nullptr;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        // chunk order: per tile pair, per step, per buffer, the step's chunks
        if (lane == 0) {
            uint32_t j = 0;
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l)
                    for (uint32_t b = 0; b < 2 && ok; ++b) {
                        const Step st = step_of(step_in(l));
                        if constexpr (DIR == BWD) {
                            // the Z tiles the epilogue reads for silu', one step ahead, into L2
                            const uint32_t tile = tile_of(p, b);
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
                            // a pair: this CTA's half of the chunk, the N rows (B columns) 128 rank ..
                            const int c = st.c0 + ci;
                            const uint32_t bytes = PAIR ? mlp_chunk_bytes(c) / 2 : mlp_chunk_bytes(c);
                            mbar_expect_tx(bar_full + 8 * s, bytes);
                            const unsigned char* img = DIR == FB && bwd_step(l) ? g.img_t : g.img;
                            bulk_g2s(sbase + OFF_W + s * SLOT_BYTES, img + mlp_chunk_offset(c) + rank * bytes, bytes,
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
        if (lane == 0 && rank == 0) {
            uint32_t j = 0, ar[2] = {0u, 0u};
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l)
                    for (uint32_t b = 0; b < 2 && ok; ++b) {
                        if (!mbar_wait(bar_a + 8 * b, ar[b] & 1u, abort_flag)) { ok = false; break; }
                        if (PAIR && !mbar_wait_cluster(bar_pa + 8 * b, ar[b] & 1u, abort_flag)) { ok = false; break; }
                        ++ar[b];
                        tc_fence_after();
                        const Step st = step_of(step_in(l));
                        const uint32_t idesc = idesc_bf16(PAIR ? 2 * TM : TM, st.n);
                        const uint32_t a_base = sbase + OFF_A + b * A_BYTES;
                        const uint32_t d = tmem + b * 256u;
                        for (int ci = 0; ci < st.nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                            if (PAIR && !mbar_wait_cluster(bar_pfull + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                            tc_fence_after();
                            const uint32_t wslot = sbase + OFF_W + s * SLOT_BYTES;
                            for (int ks = 0; ks < st.ksteps; ++ks) {
                                const uint32_t kk = uint32_t(ci * st.ksteps + ks);  // K step within the layer
                                const uint64_t a = smem_desc(a_base + kk * 256u, 128u, A_SBO);
                                const uint64_t bd = smem_desc(wslot + uint32_t(ks) * 256u, 128u, st.b_sbo);
                                if constexpr (PAIR) mma_bf16_ss_pair(d, a, bd, idesc, kk > 0 ? 1u : 0u);
                                else mma_bf16_ss(d, a, bd, idesc, kk > 0 ? 1u : 0u);
                            }
                            if constexpr (PAIR) mma_commit_pair(bar_empty + 8 * s);
                            else mma_commit(bar_empty + 8 * s);
                        }
                        if (ok) {
                            if constexpr (PAIR) mma_commit_pair(bar_d + 8 * b);
                            else mma_commit(bar_d + 8 * b);
                        }
                    }
            // all MMAs issued by this thread are complete before TMEM is freed
            if constexpr (PAIR) mma_commit_pair(bar_drain);
            else mma_commit(bar_drain);
            for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_drain, 0); ++it) {}
        } else if (PAIR && lane == 0) {
            // the odd CTA of a pair: each of its chunk halves, once landed, to
            // the even CTA's peer_full; at the end the even CTA's last commit
            // (drain: no MMA reads this CTA's memory any more)
            uint32_t j = 0;
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l)
                    for (uint32_t b = 0; b < 2 && ok; ++b) {
                        const Step st = step_of(step_in(l));
                        for (int ci = 0; ci < st.nc; ++ci, ++j) {
                            const uint32_t s = j % N_SLOT, use = j / N_SLOT;
                            if (!mbar_wait(bar_full + 8 * s, use & 1u, abort_flag)) { ok = false; break; }
                            mbar_arrive_remote(mapa_shared(bar_pfull + 8 * s, 0));
                        }
                    }
            for (uint32_t it = 0; it < SLEEP_LIMIT && !mbar_try_sleep(bar_drain, 0, 1000000u); ++it) {}
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const uint32_t ew = warp - 2, q = warp & 3u, cq = ew >> 2;  // lane quarter, column quarter
        const uint32_t row = q * 32 + lane;
        const uint32_t t_q = tmem + ((q * 32u) << 16);
        // the 16-column input of the tile of pair p, buffer b into buffer b's
        // activation tile, by the warps of column quarter 1 (one row each)
        auto load_input = [&](uint32_t p, uint32_t b) {
            if (cq != 1) return;
            const uint32_t tile = tile_of(p, b);
            unsigned char* A = smem + OFF_A + b * A_BYTES;
            uint4 c0 = uint4{0u, 0u, 0u, 0u}, c1 = c0;
            if constexpr (DIR != BWD) {
                const uint32_t r = tile * TM + row;
                if (tile < n_tiles && r < g.n_rows) {
                    const size_t src = FWDLIKE ? size_t(g.perm[b0 + r]) : size_t(r);
                    float f[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) f[k] = k < MLP_IN ? g.feat[src * MLP_IN + k] : 0.f;
                    c0 = uint4{pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]),
                               pack_bf16(f[6], f[7])};
                    if constexpr (FWDLIKE) {
                        unsigned char* dst = g.x0 + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                        *reinterpret_cast<uint4*>(dst) = c0;
                        *reinterpret_cast<uint4*>(dst + 128) = c1;
                    }
                }
            } else if (tile < n_tiles) {
                const unsigned char* src = g.in + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                c0 = *reinterpret_cast<const uint4*>(src);
                c1 = *reinterpret_cast<const uint4*>(src + 128);
            }
            *reinterpret_cast<uint4*>(A + kmaj(row, 0, A_SBO)) = c0;
            *reinterpret_cast<uint4*>(A + kmaj(row, 8, A_SBO)) = c1;
        };
        // buffer b's activation rows of this CTA are written: a single CTA
        // (or the even CTA of a pair) arrives on its a_ready, each warp of
        // the odd CTA once on the even CTA's peer_a
        auto arrive_a = [&](uint32_t b) {
            if constexpr (PAIR) {
                if (rank != 0) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive_remote(mapa_shared(bar_pa + 8 * b, 0));
                    return;
                }
            }
            mbar_arrive(bar_a + 8 * b);
        };
        uint32_t dr[2] = {0u, 0u};
        bool ok = true;
        float loss = 0.f;  // FWD: the loss of this thread's rows
        if (my_pairs > 0) {
            load_input(0, 0);
            load_input(0, 1);
            fence_proxy_async();
            arrive_a(0);
            arrive_a(1);
        }
        for (uint32_t p = 0; p < my_pairs && ok; ++p)
            for (int l = 0; l < S && ok; ++l)
                for (uint32_t b = 0; b < 2 && ok; ++b) {
                    const uint32_t tile = tile_of(p, b);
                    const bool valid = tile < n_tiles;  // false for the empty tile
                    const size_t tile_off = size_t(tile) * A_BYTES;
                    unsigned char* const A = smem + OFF_A + b * A_BYTES;
                    const uint32_t tb = t_q + b * 256u;
                    const bool bw = bwd_step(l);
                    const int sl = step_in(l);
                    const int li = bw ? 3 - sl : sl;  // the Z (and dZ) of this step
                    unsigned char* const zl = li == 0 ? g.z[0] : (li == 1 ? g.z[1] : (li == 2 ? g.z[2] : g.z[3]));
                    // BWD: the first 32 of this warp's 64 columns of Z, loaded while the MMAs run
                    uint4 zs[4];
                    if (bw) {
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            zs[k] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off +
                                                                            kmaj(row, cq * 64 + 8 * k, A_SBO))
                                          : uint4{0u, 0u, 0u, 0u};
                    }
                    if (!mbar_wait(bar_d + 8 * b, dr[b] & 1u, abort_flag)) { ok = false; break; }
                    ++dr[b];
                    tc_fence_after();
                    if (bw) {
                        // dZ_{li} = scale acc * silu'(Z_{li}); W5 is stored whole, W4..W2 halved;
                        // 4 blocks of 16 columns
                        const float scale = sl > 0 ? 2.0f : 1.0f;
                        unsigned char* const dzl =
                            li == 0 ? g.dz[0] : (li == 1 ? g.dz[1] : (li == 2 ? g.dz[2] : g.dz[3]));
                        const uint32_t c0 = cq * 64;
                        unsigned char* const an = sl < MLP_LAYERS - 2 ? A + kmaj(row, c0, A_SBO) : nullptr;
                        unsigned char* const dn = valid ? dzl + tile_off + kmaj(row, c0, A_SBO) : nullptr;
                        const uint4 z0[2] = {zs[0], zs[1]}, z1[2] = {zs[2], zs[3]};
                        uint32_t v[16];
                        tmem_ld16(tb + c0, v);
                        tmem_wait_ld(v);
                        backward16(v, z0, scale, an, dn);
                        // the last 32 columns' Z, while the second block runs
                        uint4 z2[2], z3[2];
#pragma unroll
                        for (int k = 0; k < 2; ++k) {
                            z2[k] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off + kmaj(row, c0 + 32 + 8 * k, A_SBO))
                                          : uint4{0u, 0u, 0u, 0u};
                            z3[k] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off + kmaj(row, c0 + 48 + 8 * k, A_SBO))
                                          : uint4{0u, 0u, 0u, 0u};
                        }
                        tmem_ld16(tb + c0 + 16, v);
                        tmem_wait_ld(v);
                        backward16(v, z1, scale, an ? an + 256 : nullptr, dn ? dn + 256 : nullptr);
                        tmem_ld16(tb + c0 + 32, v);
                        tmem_wait_ld(v);
                        backward16(v, z2, scale, an ? an + 512 : nullptr, dn ? dn + 512 : nullptr);
                        tmem_ld16(tb + c0 + 48, v);
                        tmem_wait_ld(v);
                        backward16(v, z3, scale, an ? an + 768 : nullptr, dn ? dn + 768 : nullptr);
                    } else if (sl == 4) {
                        // the outputs: bias; FWD: the loss and dOut
                        if (cq == 0) {
                            uint32_t v[16];
                            tmem_ld16(tb, v);
                            tmem_wait_ld(v);
                            const uint32_t r = tile * TM + row;
                            if (valid && r < g.n_rows) {
                                const float4* b5 = reinterpret_cast<const float4*>(g.params + mlp_b_off(4));
                                float o[MLP_OUT_PAD];
#pragma unroll
                                for (int k = 0; k < 4; ++k) {
                                    const float4 bb = __ldg(b5 + k);
                                    o[4 * k] = __uint_as_float(v[4 * k]) + bb.x;
                                    o[4 * k + 1] = __uint_as_float(v[4 * k + 1]) + bb.y;
                                    o[4 * k + 2] = __uint_as_float(v[4 * k + 2]) + bb.z;
                                    o[4 * k + 3] = __uint_as_float(v[4 * k + 3]) + bb.w;
                                }
                                if (g.out) {
                                    float4* op = reinterpret_cast<float4*>(g.out + size_t(r) * MLP_OUT_PAD);
#pragma unroll
                                    for (int k = 0; k < 4; ++k)
                                        op[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
                                }
                                if constexpr (FWDLIKE) {
                                    if (g.lab) {
                                        float d[MLP_OUT_PAD];
                                        loss += mlp_row_loss(o, g.lab[g.perm[b0 + r]], g.w, d);
                                        const float inv_b = 1.0f / float(g.n_rows);
                                        uint32_t dv[8];
#pragma unroll
                                        for (int k = 0; k < 8; ++k)
                                            dv[k] = pack_bf16(d[2 * k] * inv_b, d[2 * k + 1] * inv_b);
                                        unsigned char* dst = g.dout + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                                        *reinterpret_cast<uint4*>(dst) = uint4{dv[0], dv[1], dv[2], dv[3]};
                                        *reinterpret_cast<uint4*>(dst + 128) = uint4{dv[4], dv[5], dv[6], dv[7]};
                                        if constexpr (DIR == FB) {
                                            // dOut is also the backward's first input
                                            *reinterpret_cast<uint4*>(A + kmaj(row, 0, A_SBO)) = uint4{dv[0], dv[1], dv[2], dv[3]};
                                            *reinterpret_cast<uint4*>(A + kmaj(row, 8, A_SBO)) = uint4{dv[4], dv[5], dv[6], dv[7]};
                                        }
                                    }
                                }
                            }
                        }
                    } else {
                        // hidden layer: z = 2 acc + b (INFER: u = z / 2 = acc + b / 2), H = silu(z)
                        // into the next step's operand; FWD: Z to the stash
                        const float* bl = g.params + mlp_b_off(sl) + cq * 64;
                        // 4 blocks of 16 columns, the TMEM load of the next block in flight
                        // while a block is processed
                        const uint32_t c0 = cq * 64;
                        unsigned char* const an = A + kmaj(row, c0, A_SBO);
                        unsigned char* const zn = (FWDLIKE && valid) ? zl + tile_off + kmaj(row, c0, A_SBO) : nullptr;
                        uint32_t va[16], vb[16];
                        tmem_ld16(tb + c0, va);
                        tmem_wait_ld(va);
                        tmem_ld16(tb + c0 + 16, vb);
                        hidden16<DIR == FB ? FWD : DIR>(va, bl, an, zn);
                        tmem_wait_ld(vb);
                        tmem_ld16(tb + c0 + 32, va);
                        hidden16<DIR == FB ? FWD : DIR>(vb, bl + 16, an + 256, zn ? zn + 256 : nullptr);
                        tmem_wait_ld(va);
                        tmem_ld16(tb + c0 + 48, vb);
                        hidden16<DIR == FB ? FWD : DIR>(va, bl + 32, an + 512, zn ? zn + 512 : nullptr);
                        tmem_wait_ld(vb);
                        hidden16<DIR == FB ? FWD : DIR>(vb, bl + 48, an + 768, zn ? zn + 768 : nullptr);
                    }
                    tc_fence_before();
                    const bool last = l == S - 1, more = p + 1 < my_pairs;
                    if (last && more) load_input(p + 1, b);
                    if (!last || more) {
                        fence_proxy_async();
                        arrive_a(b);
                    }
                }
        if constexpr (FWDLIKE) {
            if (cq == 0 && loss_dst) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
                if (lane == 0) atomicAdd(loss_dst, loss / float(g.n_rows));
            }
        }
    }
    __syncthreads();
    grid_dependents_go();
    // a pair: neither CTA leaves (freeing the shared memory the other
    // signals) before both are done
    if constexpr (PAIR) cluster_sync();
    if (*abort_flag && threadIdx.x == 0) atomicOr(g.status, 2u);
    if (warp == 1) {
        tc_fence_after();
        if constexpr (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ------------------------------------------------------------------------
// The chains with the activations in tensor memory (opt-in,
// MGK_SURROGATE_CHAIN=tmem; measured slower than the shared-memory kernel).
//
// Each tile's layer input is the MMA's A operand in tensor memory (A[m][k]
// at lane m, column k / 2), its accumulator an N-half of 128 columns: per
// buffer b, columns 256 b .. + 127 hold the accumulator and 256 b + 128 ..
// + 255 the 256 BF16 activations of the tile's rows.  A hidden layer runs
// as two MMA groups per tile (output columns 0-127, then 128-255), in the
// order (half 0: tile 0, tile 1), (half 1: tile 0, tile 1), so the MMAs of
// one group overlap the epilogue of the one before; each weight chunk stays
// in shared memory for all four groups of its layer (half the weight stream
// of the shared-memory kernel per tile), and the tensor core reads only the
// weights from shared memory.  The epilogue of half 0 keeps its 32 columns
// of BF16 results per row in registers until half 1 is done, then writes
// the whole layer output into the tile's A columns with tcgen05.st.  Warps
// 2-9 take tile 0's groups and warps 10-17 tile 1's, so the two tiles'
// epilogues run side by side.
//
// Barriers: full / empty per weight slot; d_ready[b] (a group's MMAs are
// complete), acc_free[b] (the epilogue has loaded the accumulator),
// a_ready[b] (the tile's A columns hold the layer input), drain.
namespace ta {
constexpr int SLOTS = 6;
constexpr uint32_t SLOT_BYTES = 32768;
constexpr uint32_t OFF_W = 0;
constexpr uint32_t OFF_BAR = OFF_W + SLOTS * SLOT_BYTES;
constexpr uint32_t N_BAR = 2 * SLOTS + 7;
constexpr uint32_t OFF_MISC = OFF_BAR + ((N_BAR * 8 + 127) / 128) * 128;
constexpr uint32_t SMEM_BYTES = OFF_MISC + 16 + 128;
static_assert(SMEM_BYTES <= 232448, "shared memory");
}  // namespace ta

// 16 accumulator columns of one row of a hidden layer (INFER, FWD) to 8
// BF16x2 words of H (bias and SiLU as hidden16); FWD: Z to the stash at zs
// (null for the empty tile).
template <int DIR>
__device__ __forceinline__ void hidden16_words(const uint32_t (&v)[16], const float* bl, unsigned char* zs,
                                               uint32_t (&w)[8]) {
    const float2 half2 = make_float2(0.5f, 0.5f), two2 = make_float2(2.0f, 2.0f);
#pragma unroll
    for (int gq = 0; gq < 2; ++gq) {
        const float4 b0 = __ldg(reinterpret_cast<const float4*>(bl + gq * 8));
        const float4 b1 = __ldg(reinterpret_cast<const float4*>(bl + gq * 8 + 4));
        const float2 bp[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                              make_float2(b1.z, b1.w)};
        uint32_t zv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c = gq * 8 + 2 * e;
            const float2 acc = make_float2(__uint_as_float(v[c]), __uint_as_float(v[c + 1]));
            if constexpr (DIR == INFER) {
                const float2 u = __ffma2_rn(half2, bp[e], acc);
                w[gq * 4 + e] = silu_half_pair(u.x, u.y);
                zv[e] = 0u;
            } else {
                const float2 z = __ffma2_rn(two2, acc, bp[e]);
                zv[e] = pack_bf16(z.x, z.y);
                const float2 u = __fmul2_rn(half2, z);
                const float2 h = __ffma2_rn(u, make_float2(tanh_approx(u.x), tanh_approx(u.y)), u);
                w[gq * 4 + e] = pack_bf16(h.x, h.y);
            }
        }
        if constexpr (DIR == FWD) {
            if (zs) *reinterpret_cast<uint4*>(zs + gq * 128) = uint4{zv[0], zv[1], zv[2], zv[3]};
        }
    }
}

// 16 accumulator columns of one row of the backward to 8 BF16x2 words of
// dZ = scale acc * silu'(Z) (as backward16), also to global memory at dz
// (null for the empty tile).
__device__ __forceinline__ void backward16_words(const uint32_t (&v)[16], const uint4 (&z)[2], float scale,
                                                 unsigned char* dz, uint32_t (&w)[8]) {
    const float2 half2 = make_float2(0.5f, 0.5f), one2 = make_float2(1.0f, 1.0f), sc2 = make_float2(scale, scale);
#pragma unroll
    for (int gq = 0; gq < 2; ++gq) {
        const uint32_t zw[4] = {z[gq].x, z[gq].y, z[gq].z, z[gq].w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c = gq * 8 + 2 * e;
            const float2 zf = unpack_bf16(zw[e]);
            const float2 u = __fmul2_rn(half2, zf);
            const float2 s = __ffma2_rn(half2, make_float2(tanh_approx(u.x), tanh_approx(u.y)), half2);
            const float2 gr = __fmul2_rn(s, __ffma2_rn(zf, __fadd2_rn(one2, make_float2(-s.x, -s.y)), one2));
            const float2 acc = make_float2(__uint_as_float(v[c]), __uint_as_float(v[c + 1]));
            const float2 d = __fmul2_rn(__fmul2_rn(sc2, acc), gr);
            w[gq * 4 + e] = pack_bf16(d.x, d.y);
        }
        if (dz)
            *reinterpret_cast<uint4*>(dz + gq * 128) = uint4{w[gq * 4], w[gq * 4 + 1], w[gq * 4 + 2], w[gq * 4 + 3]};
    }
}

template <int DIR>
__global__ void __launch_bounds__(THREADS, 1) k_mlp_chain_ta(ChainArgs g) {
    constexpr int S = DIR == BWD ? MLP_LAYERS - 1 : MLP_LAYERS;  // steps per tile
    constexpr int NS = ta::SLOTS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t sbase = smem_addr(smem);
    const uint32_t bar_full = sbase + ta::OFF_BAR, bar_empty = bar_full + NS * 8;
    const uint32_t bar_d = bar_empty + NS * 8, bar_accf = bar_d + 16, bar_ardy = bar_accf + 16;
    const uint32_t bar_drain = bar_ardy + 16;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(smem + ta::OFF_MISC);
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + ta::OFF_MISC + 4);

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_tiles = g.n_tiles;
    const uint32_t my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t my_pairs = (my_tiles + 1) / 2;  // an odd count ends with an empty tile in buffer 1
    auto tile_of = [&](uint32_t p, uint32_t b) { return blockIdx.x + (2 * p + b) * gridDim.x; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bar_d + 8 * b, 1);
            mbar_init(bar_accf + 8 * b, 32 * EPI_WARPS / 2);  // the buffer's 8 epilogue warps
            mbar_init(bar_ardy + 8 * b, 32 * EPI_WARPS / 2);
        }
        mbar_init(bar_drain, 1);
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + ta::OFF_MISC),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // everything above overlaps the previous kernel's tail when launched as its dependent
    grid_dependency_wait();
    const uint32_t b0 = g.b0 + (DIR == FWD && g.ctr ? g.ctr->batch * g.n_rows : 0u);
    float* const loss_dst = DIR == FWD && g.loss_acc ? g.loss_acc + (g.ctr ? g.ctr->epoch - 1u : 0u) : nullptr;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        // each chunk once per tile pair and layer, in the MMA's order
        if (lane == 0) {
            uint32_t j = 0;
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l) {
                    const Step st = step_of(l);
                    if constexpr (DIR == BWD) {
                        // the Z tiles the epilogue reads for silu', a step ahead, into L2
                        for (uint32_t b = 0; b < 2; ++b) {
                            const uint32_t tile = tile_of(p, b);
                            if (tile < n_tiles) {
                                if (l == 0) bulk_prefetch_l2(g.z[3] + size_t(tile) * A_BYTES, A_BYTES);
                                const unsigned char* zn = l == 0 ? g.z[2] : (l == 1 ? g.z[1] : g.z[0]);
                                if (l + 1 < S) bulk_prefetch_l2(zn + size_t(tile) * A_BYTES, A_BYTES);
                            }
                        }
                    }
                    for (int ci = 0; ci < st.nc; ++ci, ++j) {
                        const uint32_t s = j % NS, use = j / NS;
                        if (use > 0 && !mbar_wait(bar_empty + 8 * s, (use - 1) & 1u, abort_flag)) {
                            ok = false;
                            break;
                        }
                        const int c = st.c0 + ci;
                        mbar_expect_tx(bar_full + 8 * s, mlp_chunk_bytes(c));
                        bulk_g2s(sbase + ta::OFF_W + s * ta::SLOT_BYTES, g.img + mlp_chunk_offset(c), mlp_chunk_bytes(c),
                                 bar_full + 8 * s);
                    }
                }
            // drain: every issued copy has landed before the CTA may exit
            const uint32_t first = j > NS ? j - NS : 0;
            for (uint32_t k = first; k < j; ++k) {
                const uint32_t s = k % NS, use = k / NS;
                for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_full + 8 * s, use & 1u); ++it) {}
            }
        }
    } else if (warp == 1) {
        // ----------------------------------------------------------------- MMA
        if (lane == 0) {
            uint32_t j0 = 0, uses[2] = {0u, 0u}, ar[2] = {0u, 0u};
            bool ok = true;
            for (uint32_t p = 0; p < my_pairs && ok; ++p)
                for (int l = 0; l < S && ok; ++l) {
                    const Step st = step_of(l);
                    const int nh = st.n == 16u ? 1 : 2;      // N halves of 128 (one group of 16 for W5)
                    const uint32_t nn = st.n == 16u ? 16u : 128u;
                    const uint32_t idesc = idesc_bf16(TM, nn);
                    for (int h = 0; h < nh && ok; ++h)
                        for (uint32_t b = 0; b < 2 && ok; ++b) {
                            if (uses[b] > 0 && !mbar_wait(bar_accf + 8 * b, (uses[b] - 1) & 1u, abort_flag)) {
                                ok = false;
                                break;
                            }
                            ++uses[b];
                            if (h == 0) {
                                if (!mbar_wait(bar_ardy + 8 * b, ar[b] & 1u, abort_flag)) { ok = false; break; }
                                ++ar[b];
                            }
                            tc_fence_after();
                            const uint32_t d = tmem + b * 256u, a_col = tmem + b * 256u + 128u;
                            for (int ci = 0; ci < st.nc; ++ci) {
                                const uint32_t jj = j0 + uint32_t(ci), s = jj % NS;
                                if (h == 0 && b == 0) {
                                    if (!mbar_wait(bar_full + 8 * s, (jj / NS) & 1u, abort_flag)) { ok = false; break; }
                                    tc_fence_after();
                                }
                                // this half's N rows of the chunk: 16 8-row groups in
                                const uint32_t wslot = sbase + ta::OFF_W + s * ta::SLOT_BYTES + uint32_t(h) * 16u * st.b_sbo;
                                for (int ks = 0; ks < st.ksteps; ++ks) {
                                    const uint32_t kk = uint32_t(ci * st.ksteps + ks);  // K step within the layer
                                    const uint64_t bd = smem_desc(wslot + uint32_t(ks) * 256u, 128u, st.b_sbo);
                                    mma_bf16_ts(d, a_col + kk * 8u, bd, idesc, kk > 0 ? 1u : 0u);
                                }
                            }
                            if (ok) mma_commit(bar_d + 8 * b);
                        }
                    // the layer's chunks are free once its four groups are done
                    for (int ci = 0; ci < st.nc && ok; ++ci) mma_commit(bar_empty + 8 * ((j0 + uint32_t(ci)) % NS));
                    j0 += uint32_t(st.nc);
                }
            // all MMAs issued by this thread are complete before TMEM is freed
            mma_commit(bar_drain);
            for (uint32_t it = 0; it < WAIT_LIMIT && !mbar_try(bar_drain, 0); ++it) {}
        }
    } else {
        // ------------------------------------------------------------ epilogue
        // warps 2-9 take buffer 0, warps 10-17 buffer 1, so the two tiles'
        // epilogues run side by side; warp w: TMEM lanes 32 (w % 4) .. (its
        // rows) and 64 of the 128 columns of each group
        const uint32_t ew = warp - 2, b = ew >> 3, q = warp & 3u, cq = (ew >> 2) & 1u;
        const uint32_t row = q * 32 + lane;
        const uint32_t t_q = tmem + ((q * 32u) << 16);
        const uint32_t acc = t_q + b * 256u, a_col = acc + 128u;
        // the 16-column input of the tile of pair p into this buffer's A
        // columns, by the warps of column half 1 (one row each)
        auto load_input = [&](uint32_t p) {
            if (cq != 1) return;
            const uint32_t tile = tile_of(p, b);
            uint4 c0 = uint4{0u, 0u, 0u, 0u}, c1 = c0;
            if constexpr (DIR != BWD) {
                const uint32_t r = tile * TM + row;
                if (tile < n_tiles && r < g.n_rows) {
                    const size_t src = DIR == FWD ? size_t(g.perm[b0 + r]) : size_t(r);
                    float f[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) f[k] = k < MLP_IN ? g.feat[src * MLP_IN + k] : 0.f;
                    c0 = uint4{pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]),
                               pack_bf16(f[6], f[7])};
                    if constexpr (DIR == FWD) {
                        unsigned char* dst = g.x0 + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                        *reinterpret_cast<uint4*>(dst) = c0;
                        *reinterpret_cast<uint4*>(dst + 128) = c1;
                    }
                }
            } else if (tile < n_tiles) {
                const unsigned char* src = g.in + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                c0 = *reinterpret_cast<const uint4*>(src);
                c1 = *reinterpret_cast<const uint4*>(src + 128);
            }
            const uint32_t w8[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            tmem_st8(a_col, w8);
            tmem_wait_st();
        };
        auto arrive = [&](uint32_t bar) {
            tc_fence_before();
            mbar_arrive(bar);
        };
        uint32_t dr = 0;
        uint32_t hold[32];  // half 0 of the layer output, until half 1 is done
        bool ok = true;
        float loss = 0.f;  // FWD: the loss of this thread's rows
        if (my_pairs > 0) {
            load_input(0);
            arrive(bar_ardy + 8 * b);
        }
        for (uint32_t p = 0; p < my_pairs && ok; ++p)
            for (int l = 0; l < S && ok; ++l) {
                const Step st = step_of(l);
                const int nh = st.n == 16u ? 1 : 2;
                const int li = DIR == BWD ? 3 - l : l;  // the Z (and dZ) of this step
                unsigned char* const zl = li == 0 ? g.z[0] : (li == 1 ? g.z[1] : (li == 2 ? g.z[2] : g.z[3]));
                unsigned char* const dzl = li == 0 ? g.dz[0] : (li == 1 ? g.dz[1] : (li == 2 ? g.dz[2] : g.dz[3]));
                const uint32_t tile = tile_of(p, b);
                const bool valid = tile < n_tiles;  // false for the empty tile
                const size_t tile_off = size_t(tile) * A_BYTES;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (h >= nh || !ok) break;
                    const uint32_t col = uint32_t(h) * 128u + cq * 64u;  // this warp's first output column
                    // BWD: the first block's Z, loaded while the MMAs run
                    uint4 zs[2];
                    if constexpr (DIR == BWD) {
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                            zs[k] = valid ? *reinterpret_cast<const uint4*>(zl + tile_off + kmaj(row, col + 8 * k, A_SBO))
                                          : uint4{0u, 0u, 0u, 0u};
                    }
                    if (!mbar_wait(bar_d + 8 * b, dr & 1u, abort_flag)) { ok = false; break; }
                    ++dr;
                    tc_fence_after();
                    if (DIR != BWD && l == 4) {
                        // the outputs: bias; FWD: the loss and dOut
                        if (cq == 0) {
                            uint32_t v[16];
                            tmem_ld16(acc, v);
                            tmem_wait_ld(v);
                            const uint32_t r = tile * TM + row;
                            if (valid && r < g.n_rows) {
                                const float4* b5 = reinterpret_cast<const float4*>(g.params + mlp_b_off(4));
                                float o[MLP_OUT_PAD];
#pragma unroll
                                for (int k = 0; k < 4; ++k) {
                                    const float4 bb = __ldg(b5 + k);
                                    o[4 * k] = __uint_as_float(v[4 * k]) + bb.x;
                                    o[4 * k + 1] = __uint_as_float(v[4 * k + 1]) + bb.y;
                                    o[4 * k + 2] = __uint_as_float(v[4 * k + 2]) + bb.z;
                                    o[4 * k + 3] = __uint_as_float(v[4 * k + 3]) + bb.w;
                                }
                                if (g.out) {
                                    float4* op = reinterpret_cast<float4*>(g.out + size_t(r) * MLP_OUT_PAD);
#pragma unroll
                                    for (int k = 0; k < 4; ++k)
                                        op[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
                                }
                                if constexpr (DIR == FWD) {
                                    if (g.lab) {
                                        float dd[MLP_OUT_PAD];
                                        loss += mlp_row_loss(o, g.lab[g.perm[b0 + r]], g.w, dd);
                                        const float inv_b = 1.0f / float(g.n_rows);
                                        uint32_t dv[8];
#pragma unroll
                                        for (int k = 0; k < 8; ++k)
                                            dv[k] = pack_bf16(dd[2 * k] * inv_b, dd[2 * k + 1] * inv_b);
                                        unsigned char* dst = g.dout + size_t(tile) * X_TILE + kmaj(row, 0, X_SBO);
                                        *reinterpret_cast<uint4*>(dst) = uint4{dv[0], dv[1], dv[2], dv[3]};
                                        *reinterpret_cast<uint4*>(dst + 128) = uint4{dv[4], dv[5], dv[6], dv[7]};
                                    }
                                }
                            }
                        }
                        arrive(bar_accf + 8 * b);
                    } else {
                        // 64 columns in four blocks of 16
                        const float scale = l > 0 ? 2.0f : 1.0f;  // BWD: W5 whole, W4..W2 halved
                        unsigned char* const zt = (DIR == FWD && valid) ? zl + tile_off : nullptr;
                        unsigned char* const dt = (DIR == BWD && valid) ? dzl + tile_off : nullptr;
                        const bool write_a = h == 1 && l < S - 1;
                        if (write_a) {
                            // half 0 of the layer output into the tile's A columns (K = col -> column
                            // col / 2); BWD reads it back from the dZ it wrote
                            uint32_t h0[16];
#pragma unroll
                            for (int part = 0; part < 2; ++part) {
                                if constexpr (DIR == BWD) {
#pragma unroll
                                    for (int k = 0; k < 4; ++k) {
                                        const uint4 u = valid ? *reinterpret_cast<const uint4*>(
                                                                    dzl + tile_off +
                                                                    kmaj(row, cq * 64u + uint32_t(part) * 32u + 8u * k, A_SBO))
                                                              : uint4{0u, 0u, 0u, 0u};
                                        h0[4 * k] = u.x; h0[4 * k + 1] = u.y; h0[4 * k + 2] = u.z; h0[4 * k + 3] = u.w;
                                    }
                                } else {
#pragma unroll
                                    for (int k = 0; k < 16; ++k) h0[k] = hold[part * 16 + k];
                                }
                                tmem_st16(a_col + cq * 32u + uint32_t(part) * 16u, h0);
                            }
                        }
#pragma unroll
                        for (int blk = 0; blk < 4; ++blk) {
                            uint32_t v[16];
                            tmem_ld16(acc + cq * 64u + uint32_t(blk) * 16u, v);
                            tmem_wait_ld(v);
                            // the accumulator may be overwritten once all blocks are loaded
                            if (blk == 3) arrive(bar_accf + 8 * b);
                            const uint32_t c = col + uint32_t(blk) * 16u;
                            uint32_t w8[8];
                            if constexpr (DIR == BWD) {
                                const uint4 z2[2] = {zs[0], zs[1]};
                                if (blk < 3) {
                                    // the next block's Z, while this one is processed
#pragma unroll
                                    for (int k = 0; k < 2; ++k)
                                        zs[k] = valid ? *reinterpret_cast<const uint4*>(
                                                            zl + tile_off + kmaj(row, c + 16 + 8 * k, A_SBO))
                                                      : uint4{0u, 0u, 0u, 0u};
                                }
                                backward16_words(v, z2, scale, dt ? dt + kmaj(row, c, A_SBO) : nullptr, w8);
                            } else {
                                hidden16_words<DIR>(v, g.params + mlp_b_off(l) + c,
                                                    zt ? zt + kmaj(row, c, A_SBO) : nullptr, w8);
                            }
                            if (h == 0) {
                                if constexpr (DIR != BWD) {
#pragma unroll
                                    for (int k = 0; k < 8; ++k) hold[blk * 8 + k] = w8[k];
                                }
                            } else if (write_a) {
                                tmem_st8(a_col + 64u + cq * 32u + uint32_t(blk) * 8u, w8);
                            }
                        }
                        if (write_a) tmem_wait_st();
                    }
                    // after the layer's last group: the tile's A columns are ready
                    if (h == nh - 1) {
                        const bool last = l == S - 1, more = p + 1 < my_pairs;
                        if (last && more) load_input(p + 1);
                        if (!last || more) arrive(bar_ardy + 8 * b);
                    }
                }
            }
        if constexpr (DIR == FWD) {
            if (cq == 0 && loss_dst) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
                if (lane == 0) atomicAdd(loss_dst, loss / float(g.n_rows));
            }
        }
    }
    __syncthreads();
    grid_dependents_go();
    if (*abort_flag && threadIdx.x == 0) atomicOr(g.status, 2u);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// The chains run as single CTAs (cta_group::1) unless MGK_SURROGATE_PAIRS=1
// selects CTA pairs (cta_group::2: each SM streams half of every weight
// chunk).  Both give the same bits; on B200 the pairs measured slower (the
// even CTA's bulk copies landed 5-7 thousand cycles after issue against
// 1.5-2 thousand in the odd CTA, and its MMA thread waited on them).
bool use_pairs() {
    const char* v = std::getenv("MGK_SURROGATE_PAIRS");
    return v && v[0] == '1';
}

// pdl: launched as a programmatic dependent of the previous kernel in the
// stream (its set-up overlaps that kernel's tail).
// The TMEM kernel (activations in tensor memory) instead of the
// shared-memory one: MGK_SURROGATE_CHAIN=tmem.  Same bits; on B200 it
// measured slower (inference 594 against 814-833 TFLOP/s, training chains
// 68 + 77 against 60 + 63 us per step).
bool use_tmem_chain() {
    const char* v = std::getenv("MGK_SURROGATE_CHAIN");
    return v && std::strcmp(v, "tmem") == 0;
}

// The grid of the single-CTA chains, which take their tiles in pairs: the
// fewest CTAs that leave the busiest one no more pairs than one CTA per SM
// would (512 tiles on 148 SMs: 128 CTAs of two full pairs, not 148 of which
// 80 stream the weights for an empty tile).  MGK_CHAIN_GRID=n asks for n
// CTAs (at most one per SM and per tile).
uint32_t chain_grid(uint32_t n_tiles, int sm_count) {
    const uint32_t sms = uint32_t(sm_count > 0 ? sm_count : 1);
    uint32_t grid = n_tiles < sms ? n_tiles : sms;
    const uint32_t pairs = (n_tiles + 2 * grid - 1) / (2 * grid);  // of the busiest CTA
    const uint32_t fewest = (n_tiles + 2 * pairs - 1) / (2 * pairs);
    if (fewest < grid) grid = fewest;
    if (const char* e = std::getenv("MGK_CHAIN_GRID")) {
        const unsigned long v = std::strtoul(e, nullptr, 10);
        if (v >= 1 && v <= sms) grid = v < n_tiles ? uint32_t(v) : n_tiles;
    }
    return grid;
}

template <int DIR>
cudaError_t launch_chain(const ChainArgs& a, int sm_count, cudaStream_t st, bool pdl = false) {
    if (a.n_tiles == 0) return cudaSuccess;
    // the forward-and-backward chain exists only as single CTAs in shared memory
    constexpr bool ONLY_SMEM = DIR == FB;
    if constexpr (!ONLY_SMEM) {
    if (!use_pairs() && use_tmem_chain()) {
        static bool attr = false;
        if (!attr) {
            cudaError_t e = cudaFuncSetAttribute(k_mlp_chain_ta<DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 ta::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        const uint32_t grid = a.n_tiles < uint32_t(sm_count) ? a.n_tiles : uint32_t(sm_count);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.gridDim = dim3(grid, 1, 1);
        cfg.blockDim = dim3(THREADS, 1, 1);
        cfg.dynamicSmemBytes = ta::SMEM_BYTES;
        cfg.stream = st;
        cfg.attrs = at;
        cfg.numAttrs = pdl ? 1 : 0;
        return cudaLaunchKernelEx(&cfg, k_mlp_chain_ta<DIR>, a);
    }
    }
    if (ONLY_SMEM || !use_pairs()) {
        static bool attr = false;
        if (!attr) {
            cudaError_t e = cudaFuncSetAttribute(k_mlp_chain_tc<DIR, false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, Layout<false>::smem_bytes);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        const uint32_t grid = chain_grid(a.n_tiles, sm_count);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.gridDim = dim3(grid, 1, 1);
        cfg.blockDim = dim3(THREADS, 1, 1);
        cfg.dynamicSmemBytes = Layout<false>::smem_bytes;
        cfg.stream = st;
        cfg.attrs = at;
        cfg.numAttrs = pdl ? 1 : 0;
        return cudaLaunchKernelEx(&cfg, k_mlp_chain_tc<DIR, false>, a);
    }
    if constexpr (!ONLY_SMEM) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = Layout<true>::smem_bytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // as many pairs as fit on the device at once (one CTA per SM)
    static int max_pairs = 0;
    if (max_pairs == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_chain_tc<DIR, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             Layout<true>::smem_bytes);
        if (e != cudaSuccess) return e;
        cfg.gridDim = dim3(2 * uint32_t(sm_count / 2), 1, 1);
        int n = 0;
        e = cudaOccupancyMaxActiveClusters(&n, k_mlp_chain_tc<DIR, true>, &cfg);
        if (e != cudaSuccess) return e;
        if (n < 1) return cudaErrorInvalidConfiguration;
        max_pairs = n;
    }
    const uint32_t units = (a.n_tiles + 1) / 2;
    const uint32_t pairs = units < uint32_t(max_pairs) ? units : uint32_t(max_pairs);
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    return cudaLaunchKernelEx(&cfg, k_mlp_chain_tc<DIR, true>, a);
    }
    return cudaSuccess;
}

}  // namespace

size_t mlp_image_bytes() { return IMAGE_BYTES; }
size_t mlp_t_image_bytes() { return T_IMAGE_BYTES; }

cudaError_t launch_weight_image(const __nv_bfloat16* wb, void* img, void* img_t, cudaStream_t st) {
    const uint32_t n = (IMAGE_BYTES + (img_t ? T_IMAGE_BYTES : 0u)) / 2;
    k_weight_image<<<(n + 255) / 256, 256, 0, st>>>(wb, static_cast<unsigned char*>(img),
                                                     static_cast<unsigned char*>(img_t));
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer_tc(const float* feat, uint32_t n, const void* img, const float* params, float* out,
                                uint32_t* status, int sm_count, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img);
    a.params = params;
    a.feat = feat;
    a.out = out;
    a.n_rows = n;
    a.n_tiles = (n + TM - 1) / TM;
    a.status = status;
    return launch_chain<INFER>(a, sm_count, st);
}

cudaError_t launch_mlp_fwd_stash_tc(const void* img, const float* params, const float* feat, const uint32_t* perm,
                                    uint32_t b0, void* x0_tiles, void* const* z, float* out, const SampleLabel* lab,
                                    const LossWeights& w, void* dout_tiles, float* loss_acc, uint32_t n_tiles,
                                    const TrainCounters* ctr, uint32_t* status, int sm_count, cudaStream_t st,
                                    bool pdl) {
    if (lab && !dout_tiles) return cudaErrorInvalidValue;
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img);
    a.params = params;
    a.feat = feat;
    a.perm = perm;
    a.b0 = b0;
    a.x0 = static_cast<unsigned char*>(x0_tiles);
    for (int l = 0; l < 4; ++l) a.z[l] = static_cast<unsigned char*>(z[l]);
    a.out = out;
    a.lab = lab;
    a.w = w;
    a.dout = static_cast<unsigned char*>(dout_tiles);
    a.loss_acc = loss_acc;
    a.ctr = ctr;
    a.n_rows = n_tiles * TM;
    a.n_tiles = n_tiles;
    a.status = status;
    return launch_chain<FWD>(a, sm_count, st, pdl);
}

cudaError_t launch_mlp_fwd_bwd_tc(const void* img, const void* img_t, const float* params, const float* feat,
                                  const uint32_t* perm, uint32_t b0, void* x0_tiles, void* const* z, void* const* dz,
                                  const SampleLabel* lab, const LossWeights& w, void* dout_tiles, float* loss_acc,
                                  uint32_t n_tiles, const TrainCounters* ctr, uint32_t* status, int sm_count,
                                  cudaStream_t st, bool pdl) {
    if (!lab || !dout_tiles) return cudaErrorInvalidValue;
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img);
    a.img_t = static_cast<const unsigned char*>(img_t);
    a.params = params;
    a.feat = feat;
    a.perm = perm;
    a.b0 = b0;
    a.x0 = static_cast<unsigned char*>(x0_tiles);
    for (int l = 0; l < 4; ++l) {
        a.z[l] = static_cast<unsigned char*>(z[l]);
        a.dz[l] = static_cast<unsigned char*>(dz[l]);
    }
    a.lab = lab;
    a.w = w;
    a.dout = static_cast<unsigned char*>(dout_tiles);
    a.loss_acc = loss_acc;
    a.ctr = ctr;
    a.n_rows = n_tiles * TM;
    a.n_tiles = n_tiles;
    a.status = status;
    return launch_chain<FB>(a, sm_count, st, pdl);
}

cudaError_t launch_mlp_bwd_dx_tc(const void* img_t, const void* dout_tiles, void* const* z, void* const* dz,
                                 uint32_t n_tiles, uint32_t* status, int sm_count, cudaStream_t st, bool pdl) {
    ChainArgs a{};
    a.img = static_cast<const unsigned char*>(img_t);
    a.in = static_cast<const unsigned char*>(dout_tiles);
    for (int l = 0; l < 4; ++l) {
        a.z[l] = static_cast<unsigned char*>(z[l]);
        a.dz[l] = static_cast<unsigned char*>(dz[l]);
    }
    a.n_rows = n_tiles * TM;
    a.n_tiles = n_tiles;
    a.status = status;
    return launch_chain<BWD>(a, sm_count, st, pdl);
}

}  // namespace mgk
