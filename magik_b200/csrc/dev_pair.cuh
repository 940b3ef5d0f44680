// Packed FP32 arithmetic of the two-ray MIXED integrator (k_integrate_x2).
//
// On sm_100a one f32x2 instruction (FADD2 / FMUL2 / FFMA2) performs two
// IEEE-rounded FP32 operations for one issue slot.  The integrator is bound by
// instruction issue, so k_integrate_x2 keeps two rays per thread ("slots" 0
// and 1, the .x and .y halves of every float2) and evaluates each FP32
// operation of the MIXED attempt for both rays with one packed instruction.
// Every function here performs, in each half, exactly the operations of its
// scalar counterpart in dev_physics.cuh (rhs_kerr_fused,
// rhs_schwarzschild_fused, rkf45_stages, control_mixed) in the same order, so
// a ray's result does not depend on the slot or the kernel that integrated it.
#pragma once

#include <cuda_runtime.h>

#include "dev_physics.cuh"

namespace mgk {

using F2 = float2;

__device__ __forceinline__ F2 b2(float a) { return make_float2(a, a); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ F2 neg2(F2 a) { return make_float2(-a.x, -a.y); }
// a - b == a + (-b) with the same rounding
__device__ __forceinline__ F2 sub2(F2 a, F2 b) { return __fadd2_rn(a, neg2(b)); }

template <int S> __device__ __forceinline__ float lane_of(F2 v) { return S == 0 ? v.x : v.y; }
template <int S> __device__ __forceinline__ void set_lane(F2& v, float a) {
    if (S == 0) v.x = a;
    else v.y = a;
}
template <int S> __device__ __forceinline__ S7<float> slot_of(const S7<F2>& s) {
    return S7<float>{lane_of<S>(s.x), lane_of<S>(s.y), lane_of<S>(s.z), lane_of<S>(s.t),
                     lane_of<S>(s.px), lane_of<S>(s.py), lane_of<S>(s.pz)};
}
template <int S> __device__ __forceinline__ void set_slot(S7<F2>& s, const S7<float>& v) {
    set_lane<S>(s.x, v.x); set_lane<S>(s.y, v.y); set_lane<S>(s.z, v.z); set_lane<S>(s.t, v.t);
    set_lane<S>(s.px, v.px); set_lane<S>(s.py, v.py); set_lane<S>(s.pz, v.pz);
}

// msqrt / mrcp of both halves: the approximations are scalar instructions,
// the corrections packed.
__device__ __forceinline__ F2 msqrt2(F2 a) {
    a = make_float2(fmaxf(a.x, kSqrtFloor), fmaxf(a.y, kSqrtFloor));
    const F2 y = make_float2(rsqrt_approx(a.x), rsqrt_approx(a.y));
    const F2 g = mul2(a, y), h = mul2(b2(0.5f), y);
    const F2 d = fma2(neg2(g), g, a);
    return fma2(d, h, g);
}
__device__ __forceinline__ F2 mrcp2(F2 b) {
    const F2 y = make_float2(rcp_approx(b.x), rcp_approx(b.y));
    const F2 e = fma2(neg2(b), y, b2(1.0f));
    return fma2(e, y, y);
}

// ------------------------------------------------------------------ RHS
// rhs_kerr_fused for two rays.
__device__ __forceinline__ void rhs_kerr_x2(const S7<F2>& s, F2 pt, const MP<float>& m, S7<F2>& o) {
    const F2 x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const F2 a = b2(m.spin), a_sq = b2(m.a_sq);
    const F2 y_sq = mul2(y, y);
    const F2 w_sq = sub2(fma2(z, z, fma2(x, x, y_sq)), a_sq);
    const F2 sigma = msqrt2(fma2(w_sq, w_sq, mul2(b2(m.four_a_sq), y_sq)));
    const F2 r = msqrt2(mul2(b2(0.5f), add2(w_sq, sigma)));
    const F2 r_sq = mul2(r, r);
    const F2 d = add2(r_sq, a_sq);
    const F2 f_den = fma2(a_sq, y_sq, mul2(r_sq, r_sq));
    const F2 rs = mul2(r, sigma);
    const F2 rsd = mul2(rs, d);
    const F2 inv_all = mrcp2(mul2(rsd, f_den));
    const F2 inv_rsd = mul2(f_den, inv_all);
    const F2 inv_fden = mul2(rsd, inv_all);
    const F2 inv_d = mul2(rs, inv_rsd);
    const F2 inv_rs = mul2(d, inv_rsd);
    const F2 inv_r = mul2(sigma, inv_rs);
    const F2 sxz = mul2(r_sq, inv_rs);
    const F2 drx = mul2(x, sxz), dry = mul2(y, mul2(d, inv_rs)), drz = mul2(z, sxz);
    const F2 r_cu = mul2(r_sq, r);
    const F2 f_ = mul2(mul2(b2(2.0f), r_cu), inv_fden);
    const F2 kx_num = fma2(r, x, neg2(mul2(a, z)));
    const F2 kz_num = fma2(r, z, mul2(a, x));
    const F2 kx = mul2(kx_num, inv_d), kz = mul2(kz_num, inv_d), ky = mul2(y, inv_r);
    const F2 S = fma2(pz, kz, mul2(px, kx));
    const F2 kTp = sub2(fma2(py, ky, S), pt);
    const F2 f_kTp = mul2(f_, kTp);
    const F2 kTp2 = mul2(kTp, kTp);
    const F2 two_r = add2(r, r);
    const F2 Gp = fma2(neg2(two_r), S, fma2(pz, z, mul2(px, x)));
    const F2 Ad = mul2(f_kTp, inv_d);
    const F2 Ux = fma2(px, r, mul2(pz, a));
    const F2 Uz = fma2(pz, r, neg2(mul2(px, a)));
    const F2 c = mul2(py, mul2(inv_r, inv_r));
    const F2 cy = mul2(c, y);
    const F2 inv_fden_sq = mul2(inv_fden, inv_fden);
    const F2 dq = mul2(fma2(mul2(b2(m.three_a_sq), r_sq), y_sq, neg2(mul2(r_cu, r_cu))), inv_fden_sq);
    const F2 B = fma2(kTp2, dq, neg2(mul2(f_kTp, cy)));
    const F2 E = fma2(neg2(kTp2), mul2(mul2(mul2(b2(m.two_a_sq), r_cu), y), inv_fden_sq), mul2(f_kTp, mul2(c, r)));
    const F2 Q = fma2(Ad, Gp, B);
    const F2 nf = neg2(f_kTp);
    o.x = fma2(nf, kx, px);
    o.y = fma2(nf, ky, py);
    o.z = fma2(nf, kz, pz);
    o.t = sub2(f_kTp, pt);
    o.px = fma2(Q, drx, mul2(Ad, Ux));
    o.py = fma2(Q, dry, E);
    o.pz = fma2(Q, drz, mul2(Ad, Uz));
}

// rhs_schwarzschild_fused for two rays.
__device__ __forceinline__ void rhs_schwarzschild_x2(const S7<F2>& s, F2 pt, float mass_sign, S7<F2>& o) {
    const F2 x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const F2 r = msqrt2(fma2(z, z, fma2(y, y, mul2(x, x))));
    const F2 inv_r = mrcp2(r);
    const F2 kx = mul2(x, inv_r), ky = mul2(y, inv_r), kz = mul2(z, inv_r);
    const F2 kp = fma2(pz, kz, fma2(py, ky, mul2(px, kx)));
    const F2 kTp = sub2(kp, pt);
    const F2 fk = mul2(mul2(b2(mass_sign * 2.0f), inv_r), kTp);
    const F2 nfk = neg2(fk);
    o.x = fma2(nfk, kx, px);
    o.y = fma2(nfk, ky, py);
    o.z = fma2(nfk, kz, pz);
    o.t = sub2(fk, pt);
    const F2 sc = mul2(fk, inv_r);
    const F2 q = fma2(b2(0.5f), kTp, kp);
    o.px = mul2(sc, fma2(neg2(kx), q, px));
    o.py = mul2(sc, fma2(neg2(ky), q, py));
    o.pz = mul2(sc, fma2(neg2(kz), q, pz));
}

template <int METRIC>
__device__ __forceinline__ void rhs_x2(const S7<F2>& s, F2 pt, const MP<float>& m, S7<F2>& o) {
    static_assert(METRIC == 1 || METRIC == 2, "packed RHS: Schwarzschild and Kerr");
    if constexpr (METRIC == 2) rhs_kerr_x2(s, pt, m, o);
    else rhs_schwarzschild_x2(s, pt, m.mass_sign, o);
}

// ------------------------------------------------------------- RKF45
__device__ __forceinline__ S7<F2> axpy2(F2 c, const S7<F2>& k, const S7<F2>& y) {
    return S7<F2>{fma2(c, k.x, y.x), fma2(c, k.y, y.y), fma2(c, k.z, y.z), fma2(c, k.t, y.t),
                  fma2(c, k.px, y.px), fma2(c, k.py, y.py), fma2(c, k.pz, y.pz)};
}
// c * h with c a tableau constant; -(c h) == (-c) h exactly.
__device__ __forceinline__ F2 ch(float c, F2 h) { return mul2(b2(c), h); }

// rkf45_stages<METRIC, Fuse::Fma, float> for two rays.
template <int METRIC>
__device__ __forceinline__ void rkf45_stages_x2(const S7<F2>& y0, F2 pt, F2 h, const MP<float>& m, S7<F2>& y1,
                                                S7<F2> k[6]) {
    using C = FB<float>;
    rhs_x2<METRIC>(y0, pt, m, k[0]);
    rhs_x2<METRIC>(axpy2(ch(C::a21, h), k[0], y0), pt, m, k[1]);
    rhs_x2<METRIC>(axpy2(ch(C::a32, h), k[1], axpy2(ch(C::a31, h), k[0], y0)), pt, m, k[2]);
    rhs_x2<METRIC>(axpy2(ch(C::a43, h), k[2], axpy2(ch(-C::a42, h), k[1], axpy2(ch(C::a41, h), k[0], y0))), pt, m,
                   k[3]);
    rhs_x2<METRIC>(axpy2(ch(-C::a54, h), k[3],
                         axpy2(ch(C::a53, h), k[2], axpy2(ch(-C::a52, h), k[1], axpy2(ch(C::a51, h), k[0], y0)))),
                   pt, m, k[4]);
    rhs_x2<METRIC>(axpy2(ch(-C::a65, h), k[4],
                         axpy2(ch(C::a64, h), k[3],
                               axpy2(ch(-C::a63, h), k[2], axpy2(ch(C::a62, h), k[1], axpy2(ch(-C::a61, h), k[0], y0))))),
                   pt, m, k[5]);
    y1 = axpy2(ch(C::b6, h), k[5],
               axpy2(ch(-C::b5, h), k[4], axpy2(ch(C::b4, h), k[3], axpy2(ch(C::b3, h), k[2], axpy2(ch(C::b1, h), k[0], y0)))));
}

// The unscaled error estimate of one slot: rkf45_error_delta (or, with
// MGK_MIXED_ERR_F32 = 0, rkf45_error_unscaled of the stages converted to
// double, rounded back to float).
// With MGK_MIXED_ERR_F32 the slot's estimate is rkf45_error_delta, as in the
// one-ray kernel.
template <int S> __device__ __forceinline__ S7<float> error_f64_slot(const S7<F2> k[6]) {
#if MGK_MIXED_ERR_F32
    S7<float> ks[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) ks[i] = slot_of<S>(k[i]);
    return rkf45_error_delta(ks);
#else
    S7<double> kd[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) kd[i] = cvt<double>(slot_of<S>(k[i]));
    return cvt<float>(rkf45_error_unscaled<double>(kd));
#endif
}

// rcp_norm of both halves: the seed is integer arithmetic per half, the
// Newton step packed.
__device__ __forceinline__ F2 rcp_norm2(F2 x) {
    const F2 y = make_float2(__uint_as_float(0x7EF311C3u - __float_as_uint(x.x)),
                             __uint_as_float(0x7EF311C3u - __float_as_uint(x.y)));
    return mul2(y, fma2(neg2(x), y, b2(2.0f)));
}

// control_mixed for two rays: the error estimate per slot, packed norm,
// proposal per slot.
__device__ __forceinline__ void control_mixed_x2(const S7<F2>& y0, const S7<F2>& y1, const S7<F2> k[6], F2 h,
                                                 const MP<float>& m, F2& h_next, bool ok[2]) {
    const S7<float> e0 = error_f64_slot<0>(k), e1 = error_f64_slot<1>(k);
    const F2 atol = b2(m.abs_tol), rtol = b2(m.rel_tol);
    auto term = [&](float ea, float eb, F2 a0, F2 a1) {
        const F2 mx = make_float2(fmaxf(fabsf(a0.x), fabsf(a1.x)), fmaxf(fabsf(a0.y), fabsf(a1.y)));
        return mul2(make_float2(ea, eb), rcp_norm2(fma2(rtol, mx, atol)));
    };
    const F2 s0 = term(e0.t, e1.t, y0.t, y1.t), s1 = term(e0.x, e1.x, y0.x, y1.x);
    const F2 s2 = term(e0.y, e1.y, y0.y, y1.y), s3 = term(e0.z, e1.z, y0.z, y1.z);
    const F2 s5 = term(e0.px, e1.px, y0.px, y1.px), s6 = term(e0.py, e1.py, y0.py, y1.py);
    const F2 s7 = term(e0.pz, e1.pz, y0.pz, y1.pz);
    F2 acc = mul2(s0, s0);
    acc = fma2(s1, s1, acc);
    acc = fma2(s2, s2, acc);
    acc = fma2(s3, s3, acc);
    acc = fma2(s5, s5, acc);
    acc = fma2(s6, s6, acc);
    acc = fma2(s7, s7, acc);
    const F2 q = mul2(acc, mul2(mul2(h, h), b2(0.125f)));
    const float err[2] = {sqrtf(q.x), sqrtf(q.y)};
    const float hh[2] = {h.x, h.y};
    float hn[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float safe = err[i] > 1e-30f ? err[i] : 1e-30f;
        float v = (0.9f * hh[i]) * inv_root5(safe);
        if (v > m.h_max) v = m.h_max;
        hn[i] = v;
        ok[i] = safe < 1.0f;
    }
    h_next = make_float2(hn[0], hn[1]);
}

template <int METRIC>
__device__ __forceinline__ void attempt_x2(const MP<float>& m, const S7<F2>& y, F2 pt, F2 h, S7<F2>& y1, F2& h_next,
                                           bool ok[2]) {
    S7<F2> k[6];
    rkf45_stages_x2<METRIC>(y, pt, h, m, y1, k);
    control_mixed_x2(y, y1, k, h, m, h_next, ok);
}

}  // namespace mgk
