// The training loss of one sample of the deflection surrogate and its
// gradient with respect to the network's 16 (padded) outputs, shared by the
// loss kernel (mlp.cu: k_loss) and the loss fused into the tensor-core
// forward (mlp_train_tc.cu), so both compute it with the same operations.
//
// Outputs: [0] disk logit, [1] escape logit (the horizon logit is fixed at
// 0), [2] disk radius (scaled), [3] disk redshift, [4..6] escape direction,
// [7] confidence logit, [8..15] padding (gradient 0).  Loss terms: softmax
// cross-entropy of the class; squared errors of r and g (disk samples) and of
// the direction (escaping samples); binary cross-entropy of the confidence
// against "class right and the regression within the tolerances".
#pragma once

#include "mlp.h"

namespace mgk {

__device__ __forceinline__ float mlp_sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

// Returns the sample's loss; d[0..15] receives d(loss)/d(o).
__device__ __forceinline__ float mlp_row_loss(const float* o, const SampleLabel& L, const LossWeights& w,
                                              float* d) {
    float l = 0.f;
#pragma unroll
    for (int i = 0; i < MLP_OUT_PAD; ++i) d[i] = 0.f;
    // class cross-entropy over (disk, escape, horizon)
    const float z0 = o[0], z1 = o[1], mx = fmaxf(fmaxf(z0, z1), 0.f);
    const float e0 = expf(z0 - mx), e1 = expf(z1 - mx), e2 = expf(-mx), se = e0 + e1 + e2;
    const float p0 = e0 / se, p1 = e1 / se, p2 = e2 / se;
    const int c = L.cls;
    l += w.cls * -logf(fmaxf(c == 0 ? p0 : (c == 1 ? p1 : p2), 1e-30f));
    d[0] = w.cls * (p0 - (c == 0 ? 1.f : 0.f));
    d[1] = w.cls * (p1 - (c == 1 ? 1.f : 0.f));
    const int pred = (p0 >= p1 && p0 >= p2) ? 0 : (p1 >= p2 ? 1 : 2);
    bool good = pred == c;
    if (c == 0) {
        const float er = o[2] - L.r, eg = o[3] - L.g;
        l += w.r * er * er + w.g * eg * eg;
        d[2] = 2.f * w.r * er;
        d[3] = 2.f * w.g * eg;
        good = good && fabsf(er) < w.tol_r && fabsf(eg) < w.tol_g;
    } else if (c == 1) {
        float ed = 0.f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float e = o[4 + i] - L.dir[i];
            ed += e * e;
            d[4 + i] = 2.f * w.dir * e;
        }
        l += w.dir * ed;
        good = good && ed < w.tol_dir * w.tol_dir;
    }
    // confidence: BCE against "this prediction is within tolerance"
    const float q = mlp_sigmoid(o[7]), t = good ? 1.f : 0.f;
    l += w.conf * -(t * logf(fmaxf(q, 1e-30f)) + (1.f - t) * logf(fmaxf(1.f - q, 1e-30f)));
    d[7] = w.conf * (q - t);
    return l;
}

}  // namespace mgk
