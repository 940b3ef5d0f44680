// Driver of the deflection surrogate: parameters, sample generation,
// training (forward, loss, backward, Adam on the library's tensor-core
// kernels), inference and the routed render.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "dev_scene.cuh"
#include "internal.h"
#include "mlp.h"

using namespace mgk;

namespace {

// Offsets (in floats) of the layers in the flat parameter vector; weights are
// stored [out][in] (the K-major B operand of the forward GEMMs).
struct Layout {
    size_t w[MLP_LAYERS], b[MLP_LAYERS], total;
    int in[MLP_LAYERS], out[MLP_LAYERS];
};
Layout param_layout() {
    Layout L{};
    const int ins[MLP_LAYERS] = {MLP_IN_PAD, MLP_HID, MLP_HID, MLP_HID, MLP_HID};
    const int outs[MLP_LAYERS] = {MLP_HID, MLP_HID, MLP_HID, MLP_HID, MLP_OUT_PAD};
    size_t o = 0;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        L.in[l] = ins[l];
        L.out[l] = outs[l];
        L.w[l] = o;
        o += size_t(ins[l]) * outs[l];
        L.b[l] = o;
        o += outs[l];
    }
    L.total = o;
    return L;
}

}  // namespace

struct mgk_surrogate {
    mgk_context* ctx = nullptr;
    int device = 0;
    Layout L{};
    float* p = nullptr;        // FP32 master parameters
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    __nv_bfloat16* wb = nullptr;  // BF16 copies (same offsets)
    uint64_t step = 0;
    // training buffers for batch `tb`
    int tb = 0;
    // the tensor-core training path (mlp_train_tc.cu): tiled activations and
    // the weight-gradient partials; off (the mma.sync GEMMs of mlp.cu) when
    // MGK_SURROGATE_TRAIN=mma was set at creation
    bool train_tc = true;
    void *tx0 = nullptr, *tZ[4] = {}, *tdZ[4] = {}, *tdout = nullptr;
    float* dw_part = nullptr;
    DwJobs dw_jobs{};
    __nv_bfloat16 *x0 = nullptr, *Z[4] = {}, *H[4] = {}, *dza = nullptr, *dzb = nullptr, *dout = nullptr;
    float *out = nullptr, *dout32 = nullptr, *loss = nullptr;
    mgk_sample_label* blab = nullptr;
    uint32_t* perm = nullptr;
    uint32_t perm_n = 0;
    uint32_t order_n = 0;  // length of the latest mgk_surrogate_shuffle order (rows gradient_step may take)
    // inference buffers for batch `ib`
    int ib = 0;
    __nv_bfloat16 *ix0 = nullptr, *iha = nullptr, *ihb = nullptr;
    float* iout = nullptr;
    // fused tensor-core inference: weight image (rebuilt after each update)
    void* img = nullptr;
    void* img_t = nullptr;  // the transposed image of the training backward (tcgen05 path)
    bool img_valid = false;
    uint32_t* status = nullptr;  // bit 1: a bounded wait of the fused kernel gave up
    int sm_count = 0;
    std::vector<void*> owned;
    // mgk_surrogate_train on the tensor-core path: the run's position on the
    // device, its tables (Adam constants per step, order keys per epoch), the
    // epoch losses, and the CUDA graph of one epoch with the key it was
    // captured for
    TrainCounters* ctr = nullptr;
    AdamStep* adam_table = nullptr;
    uint4* keys = nullptr;
    float* epoch_loss = nullptr;
    uint32_t table_cap = 0, epoch_cap = 0;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t epoch_graph = nullptr;
    struct GraphKey {
        const void *feat, *lab;
        uint32_t n, B;
        LossWeights w;
        const void *table, *keys, *loss;
        char env[96];  // the values of the switches that change which kernels an epoch launches
    } graph_key{};
};

namespace {

template <class P> cudaError_t dalloc(mgk_surrogate* s, P** ptr, size_t bytes) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return e;
    s->owned.push_back(q);
    *ptr = static_cast<P*>(q);
    return cudaSuccess;
}

#define TRY(call)                                          \
    do {                                                   \
        cudaError_t _e = (call);                           \
        if (_e != cudaSuccess) {                           \
            cudaGetLastError();                            \
            return MGK_ERROR_CUDA;                         \
        }                                                  \
    } while (0)

mgk_result ensure_train_buffers(mgk_surrogate* s, int B) {
    if (s->tb >= B) return MGK_SUCCESS;
    if (s->tb) return MGK_ERROR_INVALID_ARGUMENT;  // one batch size per network
    const size_t act = size_t(B) * MLP_HID * sizeof(__nv_bfloat16);
    TRY(dalloc(s, &s->x0, size_t(B) * MLP_IN_PAD * 2));
    for (int l = 0; l < 4; ++l) {
        TRY(dalloc(s, &s->Z[l], act));
        TRY(dalloc(s, &s->H[l], act));
    }
    TRY(dalloc(s, &s->dza, act));
    TRY(dalloc(s, &s->dzb, act));
    TRY(dalloc(s, &s->dout, size_t(B) * MLP_OUT_PAD * 2));
    TRY(dalloc(s, &s->out, size_t(B) * MLP_OUT_PAD * 4));
    TRY(dalloc(s, &s->dout32, size_t(B) * MLP_OUT_PAD * 4));
    TRY(dalloc(s, &s->loss, 64));
    TRY(dalloc(s, &s->blab, size_t(B) * sizeof(mgk_sample_label)));
    if (s->train_tc) {
        if (B % 128) return MGK_ERROR_INVALID_ARGUMENT;
        TRY(dalloc(s, &s->tx0, size_t(B) * MLP_IN_PAD * 2));
        for (int l = 0; l < 4; ++l) {
            TRY(dalloc(s, &s->tZ[l], act));
            TRY(dalloc(s, &s->tdZ[l], act));
        }
        TRY(dalloc(s, &s->tdout, size_t(B) * MLP_OUT_PAD * 2));
        TRY(dalloc(s, &s->img_t, mlp_t_image_bytes()));
        s->img_valid = false;  // both images are built from now on
        // the weight gradients on 7/8 of the SMs (129 of 148): on B200, 128
        // CTAs took 197.8 us per training step against 201.3 with 148, 198.6
        // with 112 and 202.6 with 96 (fewer CTAs contending for DRAM, fewer
        // partials for Adam); MGK_DW_CTAS=n asks for n
        int ctas = s->sm_count * 7 / 8;
        if (const char* e = std::getenv("MGK_DW_CTAS")) {
            const int v = std::atoi(e);
            if (v > 0 && v <= s->sm_count) ctas = v;
        }
        s->dw_jobs = mlp_dw_jobs(uint32_t(B) / 128u, ctas);
        // MGK_DW_JOBS=h,l0,l4: the jobs per 256-column layer, for W1 and for
        // W5 (each at most one per tile, together at most one CTA per SM)
        if (const char* e = std::getenv("MGK_DW_JOBS")) {
            unsigned h = 0, l0 = 0, l4 = 0;
            const uint32_t tiles = uint32_t(B) / 128u;
            if (std::sscanf(e, "%u,%u,%u", &h, &l0, &l4) == 3 && h >= 1 && l0 >= 1 && l4 >= 1 && h <= tiles &&
                l0 <= tiles && l4 <= tiles && 3 * h + l0 + l4 <= unsigned(s->sm_count)) {
                s->dw_jobs.heavy = h;
                s->dw_jobs.l0 = l0;
                s->dw_jobs.l4 = l4;
            }
        }
        TRY(dalloc(s, &s->dw_part, mlp_dw_partial_floats(s->dw_jobs.total()) * sizeof(float)));
    }
    s->tb = B;
    return MGK_SUCCESS;
}

mgk_result ensure_infer_buffers(mgk_surrogate* s, int B) {
    if (s->ib >= B) return MGK_SUCCESS;
    if (s->ib) return MGK_ERROR_INVALID_ARGUMENT;
    TRY(dalloc(s, &s->ix0, size_t(B) * MLP_IN_PAD * 2));
    TRY(dalloc(s, &s->iha, size_t(B) * MLP_HID * 2));
    TRY(dalloc(s, &s->ihb, size_t(B) * MLP_HID * 2));
    TRY(dalloc(s, &s->iout, size_t(B) * MLP_OUT_PAD * 4));
    s->ib = B;
    return MGK_SUCCESS;
}

// Permutation buffer of the sample set (grown by reallocation).
mgk_result ensure_perm(mgk_surrogate* s, uint32_t n) {
    if (s->perm_n >= n) return MGK_SUCCESS;
    if (s->perm) {
        for (auto& q : s->owned)
            if (q == s->perm) q = nullptr;
        cudaFree(s->perm);
        s->perm = nullptr;
        s->perm_n = 0;
    }
    TRY(dalloc(s, &s->perm, size_t(n) * 4));
    s->perm_n = n;
    return MGK_SUCCESS;
}

GemmArgs gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, int lda, int ldb, int ldc) {
    GemmArgs g{};
    g.A = A; g.B = B; g.M = M; g.N = N; g.K = K; g.lda = lda; g.ldb = ldb; g.ldc = ldc; g.k_split = K;
    return g;
}

// Forward pass of a batch of B rows from x0; with Z == nullptr (inference)
// only the activations are written, ping-ponging between ha and hb.
cudaError_t forward(mgk_surrogate* s, const __nv_bfloat16* x0, int B, __nv_bfloat16* const* Z,
                    __nv_bfloat16* const* H, float* out, cudaStream_t st) {
    const Layout& L = s->L;
    GemmArgs g = gemm(x0, s->wb + L.w[0], B, MLP_HID, MLP_IN_PAD, MLP_IN_PAD, MLP_IN_PAD, MLP_HID);
    g.bias = s->p + L.b[0];
    g.Z = Z ? Z[0] : nullptr;
    g.H = H[0];
    cudaError_t e = launch_gemm(GEMM_FWD_FIRST, g, st);
    for (int l = 1; l < 4 && e == cudaSuccess; ++l) {
        g = gemm(H[l - 1], s->wb + L.w[l], B, MLP_HID, MLP_HID, MLP_HID, MLP_HID, MLP_HID);
        g.bias = s->p + L.b[l];
        g.Z = Z ? Z[l] : nullptr;
        g.H = H[l];
        e = launch_gemm(GEMM_FWD_HIDDEN, g, st);
    }
    if (e != cudaSuccess) return e;
    g = gemm(H[3], s->wb + L.w[4], B, MLP_OUT_PAD, MLP_HID, MLP_HID, MLP_HID, MLP_OUT_PAD);
    g.bias = s->p + L.b[4];
    g.out = out;
    return launch_gemm(GEMM_FWD_OUT, g, st);
}

// One gradient of the batch rows perm[b0 .. b0 + B) on the tensor-core
// path: forward (gathering the rows) with stash and loss, input gradients,
// weight gradients (all of grad is written); the batch mean loss is added to
// *loss_acc.
// The forward and backward chains as one kernel (each tile's backward right
// after its forward: 6 us per step of 65,536 rows less than two kernels on
// B200) unless MGK_SURROGATE_FUSED=0, or a chain variant other than the
// shared-memory one is asked for.
bool fused_chains() {
    const char* f = std::getenv("MGK_SURROGATE_FUSED");
    const char* p = std::getenv("MGK_SURROGATE_PAIRS");
    const char* c = std::getenv("MGK_SURROGATE_CHAIN");
    return !(f && f[0] == '0') && !(p && p[0] == '1') && !(c && std::strcmp(c, "tmem") == 0);
}

// The values of the environment switches that choose the training kernels,
// each followed by ';' (a captured epoch is replayed only under the same).
void switch_values(char (&out)[96]) {
    static const char* const names[] = {"MGK_SURROGATE_FUSED", "MGK_SURROGATE_PDL", "MGK_SURROGATE_PAIRS",
                                        "MGK_SURROGATE_CHAIN"};
    size_t k = 0;
    for (const char* n : names) {
        if (const char* v = std::getenv(n))
            for (; *v && k + 2 < sizeof(out); ++v) out[k++] = *v;
        if (k + 1 < sizeof(out)) out[k++] = ';';
    }
}

cudaError_t gradient_tc(mgk_surrogate* s, const float* feat, const mgk_sample_label* lab, int b0, int B,
                        const LossWeights& w, float* loss_acc, cudaStream_t st, const TrainCounters* ctr = nullptr,
                        bool reduce = true, bool pdl = false) {
    const uint32_t tiles = uint32_t(B) / 128u;
    cudaError_t e = cudaSuccess;
    if (!s->img_valid) {
        e = launch_weight_image(s->wb, s->img, s->img_t, st);
        s->img_valid = e == cudaSuccess;
    }
    if (fused_chains()) {
        if (e == cudaSuccess)
            e = launch_mlp_fwd_bwd_tc(s->img, s->img_t, s->p, feat, s->perm, uint32_t(b0), s->tx0, s->tZ, s->tdZ, lab,
                                      w, s->tdout, loss_acc, tiles, ctr, s->status, s->sm_count, st, pdl);
    } else {
        if (e == cudaSuccess)
            e = launch_mlp_fwd_stash_tc(s->img, s->p, feat, s->perm, uint32_t(b0), s->tx0, s->tZ, nullptr, lab, w,
                                        s->tdout, loss_acc, tiles, ctr, s->status, s->sm_count, st, pdl);
        if (e == cudaSuccess)
            e = launch_mlp_bwd_dx_tc(s->img_t, s->tdout, s->tZ, s->tdZ, tiles, s->status, s->sm_count, st, pdl);
    }
    if (e == cudaSuccess)
        e = launch_mlp_dw_tc(s->tdZ, s->tZ, s->tx0, s->tdout, s->dw_part, s->grad, tiles, s->dw_jobs, s->status, st,
                             reduce, pdl);
    return e;
}

// One gradient on the mma.sync path (mlp.cu): gather, forward, backward.
cudaError_t backward(mgk_surrogate* s, int B, const LossWeights& w, float* loss_acc, cudaStream_t st);
cudaError_t gradient_mma(mgk_surrogate* s, const float* feat, const mgk_sample_label* lab, int b0, int B,
                         const LossWeights& w, float* loss_acc, cudaStream_t st) {
    cudaError_t e = launch_gather(feat, lab, s->perm, b0, B, s->x0, s->blab, st);
    if (e == cudaSuccess) e = forward(s, s->x0, B, s->Z, s->H, s->out, st);
    if (e == cudaSuccess) e = backward(s, B, w, loss_acc, st);
    return e;
}

cudaError_t gradient(mgk_surrogate* s, const float* feat, const mgk_sample_label* lab, int b0, int B,
                     const LossWeights& w, float* loss_acc, cudaStream_t st) {
    return s->train_tc ? gradient_tc(s, feat, lab, b0, B, w, loss_acc, st)
                       : gradient_mma(s, feat, lab, b0, B, w, loss_acc, st);
}

// Loss, backward pass and gradient accumulation of the batch in the training
// buffers (grad is zeroed first); the batch mean loss is added to *loss_acc.
cudaError_t backward(mgk_surrogate* s, int B, const LossWeights& w, float* loss_acc, cudaStream_t st) {
    const Layout& L = s->L;
    cudaError_t e = cudaMemsetAsync(s->grad, 0, L.total * sizeof(float), st);
    if (e == cudaSuccess) e = launch_loss(s->out, s->blab, B, w, s->dout, s->dout32, loss_acc, st);
    if (e != cudaSuccess) return e;
    const int ks = B >= 1024 && B % 1024 == 0 ? 1024 : B;
    // output layer
    GemmArgs g = gemm(s->dout, s->H[3], MLP_OUT_PAD, MLP_HID, B, MLP_OUT_PAD, MLP_HID, MLP_HID);
    g.k_split = ks;
    g.out = s->grad + L.w[4];
    if ((e = launch_gemm(GEMM_DW_OUT, g, st)) != cudaSuccess) return e;
    if ((e = launch_colsum_f32(s->dout32, B, MLP_OUT_PAD, s->grad + L.b[4], st)) != cudaSuccess) return e;
    g = gemm(s->dout, s->wb + L.w[4], B, MLP_HID, MLP_OUT_PAD, MLP_OUT_PAD, MLP_HID, MLP_HID);
    g.Zp = s->Z[3];
    g.H = s->dza;
    if ((e = launch_gemm(GEMM_DX_FROM_OUT, g, st)) != cudaSuccess) return e;
    // hidden layers 4, 3, 2 (index l = 3, 2, 1): dz of layer l is in `cur`
    __nv_bfloat16* cur = s->dza;
    __nv_bfloat16* nxt = s->dzb;
    for (int l = 3; l >= 1; --l) {
        g = gemm(cur, s->H[l - 1], MLP_HID, MLP_HID, B, MLP_HID, MLP_HID, MLP_HID);
        g.k_split = ks;
        g.out = s->grad + L.w[l];
        if ((e = launch_gemm(GEMM_DW_HIDDEN, g, st)) != cudaSuccess) return e;
        if ((e = launch_colsum(cur, B, MLP_HID, MLP_HID, s->grad + L.b[l], st)) != cudaSuccess) return e;
        g = gemm(cur, s->wb + L.w[l], B, MLP_HID, MLP_HID, MLP_HID, MLP_HID, MLP_HID);
        g.Zp = s->Z[l - 1];
        g.H = nxt;
        if ((e = launch_gemm(GEMM_DX_HIDDEN, g, st)) != cudaSuccess) return e;
        __nv_bfloat16* t = cur;
        cur = nxt;
        nxt = t;
    }
    // first layer
    g = gemm(cur, s->x0, MLP_HID, MLP_IN_PAD, B, MLP_HID, MLP_IN_PAD, MLP_IN_PAD);
    g.k_split = ks;
    g.out = s->grad + L.w[0];
    if ((e = launch_gemm(GEMM_DW_FIRST, g, st)) != cudaSuccess) return e;
    return launch_colsum(cur, B, MLP_HID, MLP_HID, s->grad + L.b[0], st);
}

}  // namespace

namespace mgk {

// Inference: the fused tensor-core kernel over all n rows.
cudaError_t surrogate_infer(mgk_surrogate* s, const float* feat, uint32_t n, float* out, cudaStream_t st) {
    if (!s->img_valid) {
        cudaError_t e = launch_weight_image(s->wb, s->img, s->img_t, st);
        if (e != cudaSuccess) return e;
        s->img_valid = true;
    }
    return launch_mlp_infer_tc(feat, n, s->img, s->p, out, s->status, s->sm_count, st);
}

// Status word of the fused kernel (0: no wait gave up); synchronous.
uint32_t surrogate_status(mgk_surrogate* s) {
    uint32_t h = 0;
    if (cudaMemcpy(&h, s->status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return ~0u;
    return h;
}

// Inference with the tiled GEMM kernels of the training path, in sub-batches
// of the network's inference buffers (used to compare the two paths).
cudaError_t surrogate_infer_tiled(mgk_surrogate* s, const float* feat, uint32_t n, float* out, cudaStream_t st) {
    constexpr uint32_t IB = 1u << 20;
    if (ensure_infer_buffers(s, int(IB)) != MGK_SUCCESS) return cudaErrorMemoryAllocation;
    for (uint32_t b0 = 0; b0 < n; b0 += IB) {
        const uint32_t cnt = std::min<uint32_t>(IB, n - b0);
        const uint32_t padded = (cnt + 127) / 128 * 128;
        float* dst = out + size_t(b0) * MLP_OUT_PAD;
        cudaError_t e = launch_features_bf16(feat + size_t(b0) * MLP_IN, cnt, padded, s->ix0, st);
        if (e != cudaSuccess) return e;
        __nv_bfloat16* H[4] = {s->iha, s->ihb, s->iha, s->ihb};
        e = forward(s, s->ix0, int(padded), nullptr, H, padded == cnt ? dst : s->iout, st);
        if (e != cudaSuccess) return e;
        if (padded != cnt) {
            e = cudaMemcpyAsync(dst, s->iout, size_t(cnt) * MLP_OUT_PAD * 4, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace mgk

namespace {

LossWeights loss_weights(const mgk_train_config& c) {
    return LossWeights{c.w_cls, c.w_r, c.w_g, c.w_dir, c.w_conf, c.tol_r, c.tol_g, c.tol_dir};
}

// The sample-set order of one epoch into s->perm, on the device: the keyed
// permutation of launch_epoch_perm with round keys from the counter-based
// hash of (seed, epoch).
cudaError_t epoch_order(mgk_surrogate* s, uint32_t n, uint64_t seed, uint32_t epoch, cudaStream_t st) {
    uint32_t key[4];
    for (uint32_t r = 0; r < 4; ++r) key[r] = rng_u32(seed, 0x7E11u, epoch, r);
    return launch_epoch_perm(s->perm, n, key, st);
}

// Step size of step `k` of `total` (cosine decay from lr to lr_final) and the
// Adam constants after the network's step counter advanced to it.
AdamStep adam_constants(const mgk_train_config& c, double prog, uint64_t step, float gscale) {
    const float lr = float(double(c.lr_final) +
                           0.5 * double(c.lr - c.lr_final) * (1.0 + std::cos(3.14159265358979323846 * prog)));
    return AdamStep{lr, c.beta1, c.beta2, c.eps,
                    float(1.0 / (1.0 - std::pow(double(c.beta1), double(step)))),
                    float(1.0 / (1.0 - std::pow(double(c.beta2), double(step)))), gscale};
}

// Programmatic dependent launches in the counted run unless MGK_SURROGATE_PDL=0.
bool pdl_on() {
    const char* v = std::getenv("MGK_SURROGATE_PDL");
    return !(v && v[0] == '0');
}

// Training on the tensor-core path as a counted run: the tables of the run
// go to the device, epoch 0 runs as ordinary launches (which also set up the
// kernels' attributes), the later epochs replay a CUDA graph of one epoch
// (the epoch's order, then per batch: forward, backward, weight gradients,
// Adam), captured once and kept while the data, shapes, loss weights and
// tables stay the same.  No host synchronisation between epochs; the epoch
// losses are read at the end.
cudaError_t train_counted(mgk_surrogate* s, const mgk_train_config& cfg, const float* feat,
                          const mgk_sample_label* lab, uint32_t n, float* h_epoch_loss, cudaStream_t st) {
    const uint32_t B = cfg.batch, nb = n / B, E = cfg.epochs;
    const LossWeights w = loss_weights(cfg);
    if (E == 0) return cudaSuccess;
    if (!s->ctr) {
        cudaError_t e = dalloc(s, &s->ctr, sizeof(TrainCounters));
        if (e != cudaSuccess) return e;
    }
    // room for at least 64 epochs, so that shorter runs reuse the tables
    // (and the captured graph) of longer ones
    const uint32_t cap_e = std::max<uint32_t>(64u, E);
    if (cap_e * nb > s->table_cap || cap_e > s->epoch_cap) {
        cudaFree(s->adam_table);
        cudaFree(s->keys);
        cudaFree(s->epoch_loss);
        s->adam_table = nullptr;
        s->keys = nullptr;
        s->epoch_loss = nullptr;
        s->table_cap = s->epoch_cap = 0;
        cudaError_t e = cudaMalloc(&s->adam_table, size_t(cap_e) * nb * sizeof(AdamStep));
        if (e == cudaSuccess) e = cudaMalloc(&s->keys, size_t(cap_e) * sizeof(uint4));
        if (e == cudaSuccess) e = cudaMalloc(&s->epoch_loss, size_t(cap_e) * sizeof(float));
        if (e != cudaSuccess) return e;
        s->table_cap = cap_e * nb;
        s->epoch_cap = cap_e;
    }
    std::vector<AdamStep> table(size_t(E) * nb);
    for (uint32_t k = 0; k < E * nb; ++k)
        table[k] = adam_constants(cfg, double(k) / double(E * nb), s->step + k + 1, 1.0f);
    std::vector<uint4> keys(E);
    for (uint32_t ep = 0; ep < E; ++ep)
        keys[ep] = make_uint4(rng_u32(cfg.seed, 0x7E11u, ep, 0), rng_u32(cfg.seed, 0x7E11u, ep, 1),
                              rng_u32(cfg.seed, 0x7E11u, ep, 2), rng_u32(cfg.seed, 0x7E11u, ep, 3));
    cudaError_t e = cudaStreamSynchronize(st);  // the tables are not in use
    if (e == cudaSuccess) e = cudaMemcpy(s->adam_table, table.data(), table.size() * sizeof(AdamStep),
                                         cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->keys, keys.data(), keys.size() * sizeof(uint4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->ctr, 0, sizeof(TrainCounters), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->epoch_loss, 0, size_t(E) * sizeof(float), st);
    if (e == cudaSuccess && !s->img_valid) {
        e = launch_weight_image(s->wb, s->img, s->img_t, st);
        s->img_valid = e == cudaSuccess;
    }
    // one epoch's launches on stream q
    auto epoch = [&](cudaStream_t q) {
        cudaError_t r = launch_epoch_begin(s->perm, n, s->keys, s->ctr, q);
        for (uint32_t b = 0; b < nb && r == cudaSuccess; ++b) {
            // the gradient stays in the weight-gradient partials; Adam sums them
            // each kernel a programmatic dependent of the one before (the
            // first forward of the epoch follows the order's kernel)
            r = gradient_tc(s, feat, lab, 0, int(B), w, s->epoch_loss, q, s->ctr, false, pdl_on());
            if (r == cudaSuccess)
                r = launch_adam_counted(s->p, s->grad, s->dw_part, s->dw_jobs, s->m, s->v, s->wb, s->img, s->img_t,
                                        int(s->L.total), s->adam_table, s->ctr, q, pdl_on());
        }
        return r;
    };
    if (e == cudaSuccess) e = epoch(st);
    // MGK_SURROGATE_GRAPH=0: every epoch as ordinary launches
    const char* gv = std::getenv("MGK_SURROGATE_GRAPH");
    if (gv && gv[0] == '0')
        for (uint32_t ep = 1; ep < E && e == cudaSuccess; ++ep) e = epoch(st);
    else if (e == cudaSuccess && E > 1) {
        mgk_surrogate::GraphKey key{};
        key.feat = feat;
        key.lab = lab;
        key.n = n;
        key.B = B;
        key.w = w;
        key.table = s->adam_table;
        key.keys = s->keys;
        key.loss = s->epoch_loss;
        switch_values(key.env);
        if (!s->epoch_graph || std::memcmp(&key, &s->graph_key, sizeof(key)) != 0) {
            if (s->epoch_graph) {
                cudaGraphExecDestroy(s->epoch_graph);
                s->epoch_graph = nullptr;
            }
            if (!s->capture_stream) e = cudaStreamCreateWithFlags(&s->capture_stream, cudaStreamNonBlocking);
            cudaGraph_t graph = nullptr;
            if (e == cudaSuccess) e = cudaStreamBeginCapture(s->capture_stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                const cudaError_t r = epoch(s->capture_stream);
                e = cudaStreamEndCapture(s->capture_stream, &graph);
                if (e == cudaSuccess) e = r;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&s->epoch_graph, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e == cudaSuccess) s->graph_key = key;
        }
        for (uint32_t ep = 1; ep < E && e == cudaSuccess; ++ep) e = cudaGraphLaunch(s->epoch_graph, st);
    }
    std::vector<float> loss(E, 0.f);
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss.data(), s->epoch_loss, size_t(E) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    s->step += uint64_t(E) * nb;
    s->img_valid = true;  // the Adam kernels wrote the weight images
    if (h_epoch_loss)
        for (uint32_t ep = 0; ep < E; ++ep) h_epoch_loss[ep] = loss[ep] / float(nb);
    return cudaSuccess;
}

}  // namespace

extern "C" {

MGK_API void mgk_train_defaults(mgk_train_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->batch = 65536;
    c->epochs = 20;
    c->lr = 1e-3f;
    c->beta1 = 0.9f;
    c->beta2 = 0.999f;
    c->eps = 1e-8f;
    c->seed = 0x7EA1;
    c->w_cls = 1.0f;
    c->w_r = 10.0f;
    c->w_g = 100.0f;
    c->w_dir = 100.0f;
    c->w_conf = 0.1f;
    c->tol_r = 1e-3f;    // 0.01 M in r_hit
    c->tol_g = 1e-3f;
    c->tol_dir = 1e-3f;  // ~1 mrad
    c->lr_final = c->lr;
}

MGK_API uint64_t mgk_surrogate_param_count(void) { return param_layout().total; }

MGK_API mgk_result mgk_surrogate_destroy(mgk_surrogate* s) {
    if (!s) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    if (s->epoch_graph) cudaGraphExecDestroy(s->epoch_graph);
    if (s->capture_stream) cudaStreamDestroy(s->capture_stream);
    cudaFree(s->adam_table);
    cudaFree(s->keys);
    cudaFree(s->epoch_loss);
    for (void* q : s->owned) cudaFree(q);
    delete s;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_set_params(mgk_surrogate* s, const float* h) {
    if (!s || !h) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    const size_t n = s->L.total;
    std::vector<__nv_bfloat16> b(n);
    for (size_t i = 0; i < n; ++i) b[i] = __float2bfloat16_rn(h[i]);
    TRY(cudaMemcpy(s->p, h, n * 4, cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(s->wb, b.data(), n * 2, cudaMemcpyHostToDevice));
    s->img_valid = false;
    TRY(cudaMemset(s->m, 0, n * 4));
    TRY(cudaMemset(s->v, 0, n * 4));
    s->step = 0;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_get_params(mgk_surrogate* s, float* h) {
    if (!s || !h) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    TRY(cudaMemcpy(h, s->p, s->L.total * 4, cudaMemcpyDeviceToHost));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_create(mgk_context* ctx, uint64_t seed, mgk_surrogate** out) {
    if (!ctx || !out) return MGK_ERROR_INVALID_POINTER;
    *out = nullptr;
    mgk_surrogate* s = new (std::nothrow) mgk_surrogate();
    if (!s) return MGK_ERROR_HOST_ALLOCATION_FAILED;
    s->ctx = ctx;
    s->device = context_device(ctx);
    s->L = param_layout();
    if (const char* path = std::getenv("MGK_SURROGATE_TRAIN")) s->train_tc = std::strcmp(path, "mma") != 0;
    cudaSetDevice(s->device);
    const size_t n = s->L.total;
    if (dalloc(s, &s->p, n * 4) != cudaSuccess || dalloc(s, &s->grad, n * 4) != cudaSuccess ||
        dalloc(s, &s->m, n * 4) != cudaSuccess || dalloc(s, &s->v, n * 4) != cudaSuccess ||
        dalloc(s, &s->wb, n * 2) != cudaSuccess || dalloc(s, &s->img, mlp_image_bytes()) != cudaSuccess ||
        dalloc(s, &s->status, 16) != cudaSuccess || cudaMemset(s->status, 0, 16) != cudaSuccess ||
        cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess) {
        cudaGetLastError();
        mgk_surrogate_destroy(s);
        return MGK_ERROR_DEVICE_OUT_OF_MEMORY;
    }
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) on the real (unpadded) inputs
    std::vector<float> h(n, 0.f);
    const Layout& L = s->L;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        const int real_in = l == 0 ? MLP_IN : MLP_HID, real_out = l == MLP_LAYERS - 1 ? MLP_OUT : MLP_HID;
        const float k = 1.0f / std::sqrt(float(real_in));
        for (int o = 0; o < real_out; ++o)
            for (int i = 0; i < real_in; ++i)
                h[L.w[l] + size_t(o) * L.in[l] + i] = k * (2.0f * rng_unit(seed, 0xB17Au + l, o, i) - 1.0f);
    }
    mgk_result rc = mgk_surrogate_set_params(s, h.data());
    if (rc != MGK_SUCCESS) {
        mgk_surrogate_destroy(s);
        return rc;
    }
    *out = s;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_forward(mgk_surrogate* s, const float* d_feat, uint32_t n, float* d_out,
                                         void* stream) {
    if (!s || !d_feat || !d_out) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    TRY(surrogate_infer(s, d_feat, n, d_out, static_cast<cudaStream_t>(stream)));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_forward_tiled(mgk_surrogate* s, const float* d_feat, uint32_t n, float* d_out,
                                               void* stream) {
    if (!s || !d_feat || !d_out) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    TRY(surrogate_infer_tiled(s, d_feat, n, d_out, static_cast<cudaStream_t>(stream)));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_status(mgk_surrogate* s, uint32_t* status) {
    if (!s || !status) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(s->device);
    *status = surrogate_status(s);
    return *status == ~0u ? MGK_ERROR_CUDA : MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_gradient(mgk_surrogate* s, const mgk_train_config* cfg, const float* d_feat,
                                          const mgk_sample_label* d_lab, uint32_t n, float* h_grad, float* h_loss) {
    if (!s || !cfg || !d_feat || !d_lab || !h_grad) return MGK_ERROR_INVALID_POINTER;
    if (n == 0 || n % 1024) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    mgk_result rc = ensure_train_buffers(s, int(n));
    if (rc != MGK_SUCCESS) return rc;
    if (s->tb != int(n)) return MGK_ERROR_INVALID_ARGUMENT;
    cudaStream_t st = nullptr;
    rc = ensure_perm(s, n);
    if (rc != MGK_SUCCESS) return rc;
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    s->order_n = 0;
    TRY(cudaMemcpyAsync(s->perm, perm.data(), size_t(n) * 4, cudaMemcpyHostToDevice, st));
    TRY(cudaMemsetAsync(s->loss, 0, 4, st));
    TRY(gradient(s, d_feat, d_lab, 0, int(n), loss_weights(*cfg), s->loss, st));
    TRY(cudaMemcpyAsync(h_grad, s->grad, s->L.total * 4, cudaMemcpyDeviceToHost, st));
    float loss = 0.f;
    TRY(cudaMemcpyAsync(&loss, s->loss, 4, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    if (h_loss) *h_loss = loss;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_train(mgk_surrogate* s, const mgk_train_config* cfg, const float* d_feat,
                                       const mgk_sample_label* d_lab, uint32_t n, float* h_epoch_loss,
                                       void* stream) {
    if (!s || !cfg || !d_feat || !d_lab) return MGK_ERROR_INVALID_POINTER;
    const uint32_t B = cfg->batch;
    if (B == 0 || B % 1024 || n < B) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mgk_result rc = ensure_train_buffers(s, int(B));
    if (rc != MGK_SUCCESS) return rc;
    if (s->tb != int(B)) return MGK_ERROR_INVALID_ARGUMENT;
    rc = ensure_perm(s, n);
    if (rc != MGK_SUCCESS) return rc;
    if (s->train_tc) {
        TRY(train_counted(s, *cfg, d_feat, d_lab, n, h_epoch_loss, st));
        return MGK_SUCCESS;
    }
    const LossWeights w = loss_weights(*cfg);
    const uint32_t nb = n / B;
    for (uint32_t ep = 0; ep < cfg->epochs; ++ep) {
        s->order_n = 0;
        TRY(epoch_order(s, n, cfg->seed, ep, st));
        TRY(cudaMemsetAsync(s->loss, 0, 4, st));
        for (uint32_t b = 0; b < nb; ++b) {
            TRY(gradient(s, d_feat, d_lab, int(b * B), int(B), w, s->loss, st));
            ++s->step;
            const AdamStep a = adam_constants(*cfg, double(ep * nb + b) / double(cfg->epochs * nb), s->step, 1.0f);
            // the weight images follow the update (every weight is rewritten)
            TRY(launch_adam(s->p, s->grad, s->m, s->v, s->wb, s->img, s->img_t, int(s->L.total), a, st));
            s->img_valid = true;
        }
        float loss = 0.f;
        TRY(cudaMemcpyAsync(&loss, s->loss, 4, cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        if (h_epoch_loss) h_epoch_loss[ep] = loss / float(nb);
    }
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_shuffle(mgk_surrogate* s, uint64_t seed, uint32_t epoch, uint32_t n, void* stream) {
    if (!s) return MGK_ERROR_INVALID_POINTER;
    if (n == 0) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    mgk_result rc = ensure_perm(s, n);
    if (rc != MGK_SUCCESS) return rc;
    TRY(epoch_order(s, n, seed, epoch, static_cast<cudaStream_t>(stream)));
    s->order_n = n;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_order(mgk_surrogate* s, uint32_t* h_order, uint32_t n) {
    if (!s || !h_order) return MGK_ERROR_INVALID_POINTER;
    if (n > s->perm_n) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    TRY(cudaMemcpy(h_order, s->perm, size_t(n) * 4, cudaMemcpyDeviceToHost));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_gradient_step(mgk_surrogate* s, const mgk_train_config* cfg, const float* d_feat,
                                               const mgk_sample_label* d_lab, uint32_t first, uint32_t n,
                                               float* d_grad, float* d_loss_sum, void* stream) {
    if (!s || !cfg || !d_feat || !d_lab || !d_grad || !d_loss_sum) return MGK_ERROR_INVALID_POINTER;
    if (n == 0 || n % 1024 || uint64_t(first) + n > s->order_n) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    mgk_result rc = ensure_train_buffers(s, int(n));
    if (rc != MGK_SUCCESS) return rc;
    if (s->tb != int(n)) return MGK_ERROR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TRY(gradient(s, d_feat, d_lab, int(first), int(n), loss_weights(*cfg), d_loss_sum, st));
    TRY(cudaMemcpyAsync(d_grad, s->grad, s->L.total * 4, cudaMemcpyDeviceToDevice, st));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_surrogate_adam_step(mgk_surrogate* s, const mgk_train_config* cfg, const float* d_grad,
                                           float grad_scale, double progress, void* stream) {
    if (!s || !cfg || !d_grad) return MGK_ERROR_INVALID_POINTER;
    if (!(progress >= 0.0 && progress <= 1.0)) return MGK_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    ++s->step;
    const AdamStep a = adam_constants(*cfg, progress, s->step, grad_scale);
    TRY(launch_adam(s->p, d_grad, s->m, s->v, s->wb, s->img, s->img_t, int(s->L.total), a,
                    static_cast<cudaStream_t>(stream)));
    s->img_valid = true;
    return MGK_SUCCESS;
}

}  // extern "C"
