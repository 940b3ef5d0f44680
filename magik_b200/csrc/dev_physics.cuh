// Device physics of the geodesic path: metrics, RKF45 attempt, step control.
//
// Every function is templated on the scalar T (float / double) and on an FMA
// policy F.  The whole library is compiled with -fmad=false, so a plain
// a*b + c always rounds twice; mad<Fuse::Fma>() fuses exactly where written.
//   Fuse::None reproduces the reference's expression trees (metric_kerr.cuh,
//   metric_schwarzschild.cuh, internal_math.h) with separate roundings, i.e.
//   what the reference computes on the CPU.
//   Fuse::Fma uses the same trees with the marked multiply-adds fused, and
//   the rearranged RHS below (rhs_kerr_fused, rhs_schwarzschild_fused).
// Division and sqrt are IEEE-rounded (-prec-div/-prec-sqrt, no fast math),
// except in the float fused RHS (msqrt / mrcp below).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifndef MGK_HD
#define MGK_HD __host__ __device__ __forceinline__
#endif

namespace mgk {

enum class Fuse { None, Fma };

// Four-vectors (x, y, z, t) and symmetric 4x4 metrics.
template <class T> struct V4 { T x, y, z, t; };
template <class T> struct Sym4 { T tt, tx, ty, tz, xx, xy, xz, yy, yz, zz; };

// The metric plugins (src/renderer/relativity/metric.cuh): metric<TAG> for
// each supported MGK_METRIC_* tag.
template <int TAG> struct metric;

// 1: FP32 operations of the MIXED attempt that come in pairs run as f32x2
// instructions (one issue slot per pair, each half rounded as the scalar).
#ifndef MGK_PACKED_AXPY
#define MGK_PACKED_AXPY 1
#endif

template <Fuse F> __device__ __forceinline__ float mad(float a, float b, float c) {
    if constexpr (F == Fuse::Fma) return __fmaf_rn(a, b, c);
    else return __fadd_rn(__fmul_rn(a, b), c);
}
template <Fuse F> __device__ __forceinline__ double mad(double a, double b, double c) {
    if constexpr (F == Fuse::Fma) return __fma_rn(a, b, c);
    else return __dadd_rn(__dmul_rn(a, b), c);
}

// ------------------------------------------------- MIXED sqrt / reciprocal
// The fused RHS of the MIXED mode takes its square roots and its reciprocal
// from the hardware approximations (rsqrt.approx / rcp.approx, flush to zero)
// and one FMA correction each, after P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990:
//   sqrt(a): y ~ 1/sqrt(a), g = a y, h = y/2, d = a - g^2 (one rounding), g + d h
//   1/b:     y ~ 1/b, e = 1 - b y (one rounding), y + e y
// Neither needs the range checks and slow-path branches of the IEEE
// sequences, and their results are these functions exactly (mgk_check_rounding
// compares every float input on the device):
//   msqrt(a) = IEEE sqrt(max(a, 2^-100)), except NaN for a = +inf;
//   mrcp(b)  = IEEE 1/b for normal b with a normal reciprocal, +-0 for
//              |b| > 2^126, NaN for b = +-0, subnormal or infinite.
// The clamp keeps d = a - g^2 out of the subnormal range, where a single
// correction is not enough.  In the RHS the clamp and the special values are
// reached by degenerate states only (at the ring singularity); the oracle
// defines both functions the same way.
constexpr float kSqrtFloor = 7.888609052210118e-31f;  // 2^-100

__device__ __forceinline__ float rsqrt_approx(float a) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    return y;
}
__device__ __forceinline__ float rcp_approx(float b) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float msqrt(float a) {
    a = fmaxf(a, kSqrtFloor);
    const float y = rsqrt_approx(a);
    const float g = a * y, h = 0.5f * y;
    const float d = __fmaf_rn(-g, g, a);
    return __fmaf_rn(d, h, g);
}
__device__ __forceinline__ float mrcp(float b) {
    const float y = rcp_approx(b);
    const float e = __fmaf_rn(-b, y, 1.0f);
    return __fmaf_rn(e, y, y);
}
// The fused RHS in T: msqrt / mrcp in float, IEEE sqrt and division in double.
__device__ __forceinline__ float fused_sqrt(float a) { return msqrt(a); }
__device__ __forceinline__ double fused_sqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float fused_rcp(float b) { return mrcp(b); }
__device__ __forceinline__ double fused_rcp(double b) { return 1.0 / b; }

// Geodesic state without the conserved p_t: position (x, y, z, t) and
// covariant spatial momentum (px, py, pz).  p_t is carried beside it.
template <class T> struct S7 { T x, y, z, t, px, py, pz; };

template <class T> struct MP {  // per-metric integrator parameters (metric_kerr.cuh:112-123)
    T spin;        // as integrated (flipped when time reversed)
    T mass_sign;   // Schwarzschild
    T horizon;     // (1 + sqrt(1 - a^2)) * horizon_scalar, or 2 * scalar (Schwarzschild)
    T spin_abs_gt1;  // 1 if |spin| > 1 (Kerr never captures then)
    T h_max, abs_tol, rel_tol;
    uint32_t n_max;
    T a_sq, two_a_sq, three_a_sq, four_a_sq;  // a^2 and multiples, rounded in T (fused RHS)
};

// Fills the spin constants of m from m.spin (host or device; the same
// roundings as evaluating a * a, 2 a^2, 3 a^2, 4 a^2 in T).
template <class T> __host__ __device__ inline void set_spin_consts(MP<T>& m) {
    m.a_sq = m.spin * m.spin;
    m.two_a_sq = T(2) * m.a_sq;
    m.three_a_sq = T(3) * m.a_sq;
    m.four_a_sq = T(4) * m.a_sq;
}

// ------------------------------------------------------------------ RHS
// Kerr, metric_kerr.cuh:38-105: the reference's expression tree (REF32 runs
// it with Fuse::None and reproduces the reference's roundings).
template <Fuse F, class T>
__device__ __forceinline__ void rhs_kerr(const S7<T>& s, T pt, T a, S7<T>& o) {
    const T x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const T one = T(1), half = T(0.5), two = T(2);
    T a_sq = a * a;
    T y_sq = y * y;
    T w_sq = mad<F>(z, z, mad<F>(y, y, x * x)) - a_sq;
    T sigma = sqrt(mad<F>(w_sq, w_sq, (T(4) * a_sq) * y_sq));
    T r = sqrt(half * (w_sq + sigma));
    T r_sq = r * r;
    T r_cu = r_sq * r;
    T r_quad = r_sq * r_sq;
    T r_six = r_cu * r_cu;
    T d = r_sq + a_sq;
    T f_den = mad<F>(a_sq, y_sq, r_quad);
    T inv_r = one / r;
    T inv_sigma = one / sigma;
    T inv_d = one / d;
    T inv_f_den_sq = one / (f_den * f_den);
    T f_ = (two * r_cu) / f_den;
    T inv_rsq = inv_r * inv_r;
    T scale_xz = (half * inv_r) * mad<F>(w_sq, inv_sigma, one);
    T scale_y = (half * inv_r) * mad<F>(w_sq + two * a_sq, inv_sigma, one);
    T drx = x * scale_xz, dry = y * scale_y, drz = z * scale_xz;
    T inv_dsq = inv_d * inv_d;
    T kx_num = mad<F>(r, x, -(a * z));
    T kz_num = mad<F>(r, z, a * x);
    T kx = kx_num * inv_d;
    T kz = kz_num * inv_d;
    T ky = y * inv_r;
    T dfdq_scale = (two * mad<F>((T(3) * a_sq) * r_sq, y_sq, -r_six)) * inv_f_den_sq;
    T dfx = dfdq_scale * drx;
    T dfy = mad<F>(dfdq_scale, dry, -((((T(4) * a_sq) * r_cu) * y) * inv_f_den_sq));
    T dfz = dfdq_scale * drz;
    T two_r = two * r;
    T dkx_dx = mad<F>(mad<F>(x, drx, r), d, -((two_r * drx) * kx_num)) * inv_dsq;
    T dkx_dy = mad<F>(x * dry, d, -((two_r * dry) * kx_num)) * inv_dsq;
    T dkx_dz = mad<F>(mad<F>(x, drz, -a), d, -((two_r * drz) * kx_num)) * inv_dsq;
    T dky_dx = ((-y) * drx) * inv_rsq;
    T dky_dy = mad<F>(-y, dry, r) * inv_rsq;
    T dky_dz = ((-y) * drz) * inv_rsq;
    T dkz_dx = mad<F>(mad<F>(z, drx, a), d, -((two_r * drx) * kz_num)) * inv_dsq;
    T dkz_dy = mad<F>(z * dry, d, -((two_r * dry) * kz_num)) * inv_dsq;
    T dkz_dz = mad<F>(mad<F>(z, drz, r), d, -((two_r * drz) * kz_num)) * inv_dsq;
    T kTp = mad<F>(pz, kz, mad<F>(py, ky, px * kx)) - pt;
    T f_kTp = f_ * kTp;
    T half_kTp_sq = (half * kTp) * kTp;
    T bx = mad<F>(pz, dkz_dx, mad<F>(py, dky_dx, px * dkx_dx));
    T by = mad<F>(pz, dkz_dy, mad<F>(py, dky_dy, px * dkx_dy));
    T bz = mad<F>(pz, dkz_dz, mad<F>(py, dky_dz, px * dkx_dz));
    o.x = mad<F>(-f_kTp, kx, px);
    o.y = mad<F>(-f_kTp, ky, py);
    o.z = mad<F>(-f_kTp, kz, pz);
    o.t = -pt + f_kTp;
    o.px = mad<F>(f_kTp, bx, half_kTp_sq * dfx);
    o.py = mad<F>(f_kTp, by, half_kTp_sq * dfy);
    o.pz = mad<F>(f_kTp, bz, half_kTp_sq * dfz);
}

// Schwarzschild, metric_schwarzschild.cuh:8-72: the reference's tree.
template <Fuse F, class T>
__device__ __forceinline__ void rhs_schwarzschild(const S7<T>& s, T pt, T mass_sign, S7<T>& o) {
    const T x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const T one = T(1), half = T(0.5), two = T(2);
    T w_sq = mad<F>(z, z, mad<F>(y, y, x * x));
    T sigma = w_sq;
    T r = sqrt(half * (w_sq + sigma));
    T r_sq = r * r;
    T r_cu = r_sq * r;
    T r_quad = r_sq * r_sq;
    T r_six = r_cu * r_cu;
    T d = r_sq;
    T f_den = r_quad;
    T inv_r = one / r;
    T inv_sigma = one / sigma;
    T inv_d = one / d;
    T inv_f_den_sq = one / (f_den * f_den);
    T f_ = ((mass_sign * two) * r_cu) / f_den;
    T inv_rsq = inv_r * inv_r;
    T sc = (half * inv_r) * mad<F>(w_sq, inv_sigma, one);
    T drx = x * sc, dry = y * sc, drz = z * sc;
    T inv_dsq = inv_d * inv_d;
    T kx_num = r * x;
    T kz_num = r * z;
    T kx = kx_num * inv_d;
    T kz = kz_num * inv_d;
    T ky = y * inv_r;
    T dfdq_scale = ((mass_sign * two) * (-r_six)) * inv_f_den_sq;
    T dfx = dfdq_scale * drx, dfy = dfdq_scale * dry, dfz = dfdq_scale * drz;
    T two_r = two * r;
    T dkx_dx = mad<F>(mad<F>(x, drx, r), d, -((two_r * drx) * kx_num)) * inv_dsq;
    T dkx_dy = mad<F>(x * dry, d, -((two_r * dry) * kx_num)) * inv_dsq;
    T dkx_dz = mad<F>(x * drz, d, -((two_r * drz) * kx_num)) * inv_dsq;
    T dky_dx = ((-y) * drx) * inv_rsq;
    T dky_dy = mad<F>(-y, dry, r) * inv_rsq;
    T dky_dz = ((-y) * drz) * inv_rsq;
    T dkz_dx = mad<F>(z * drx, d, -((two_r * drx) * kz_num)) * inv_dsq;
    T dkz_dy = mad<F>(z * dry, d, -((two_r * dry) * kz_num)) * inv_dsq;
    T dkz_dz = mad<F>(mad<F>(z, drz, r), d, -((two_r * drz) * kz_num)) * inv_dsq;
    T kTp = mad<F>(pz, kz, mad<F>(py, ky, px * kx)) - pt;
    T f_kTp = f_ * kTp;
    T half_kTp_sq = (half * kTp) * kTp;
    T bx = mad<F>(pz, dkz_dx, mad<F>(py, dky_dx, px * dkx_dx));
    T by = mad<F>(pz, dkz_dy, mad<F>(py, dky_dy, px * dkx_dy));
    T bz = mad<F>(pz, dkz_dz, mad<F>(py, dky_dz, px * dkx_dz));
    o.x = mad<F>(-f_kTp, kx, px);
    o.y = mad<F>(-f_kTp, ky, py);
    o.z = mad<F>(-f_kTp, kz, pz);
    o.t = -pt + f_kTp;
    o.px = mad<F>(f_kTp, bx, half_kTp_sq * dfx);
    o.py = mad<F>(f_kTp, by, half_kTp_sq * dfy);
    o.pz = mad<F>(f_kTp, bz, half_kTp_sq * dfz);
}


// Kerr, fused formulation (MIXED and F64): the same Hamiltonian RHS,
//   dx/dl = p - f (k.p) k,   dp/dl = f (k.p) (grad k).p + (k.p)^2 grad f / 2,
// k = ((r x - a z)/d, y/r, (r z + a x)/d), d = r^2 + a^2, f = 2 r^3/(r^4 + a^2 y^2),
// rearranged to need fewer operations:
//  * one reciprocal 1/(r sigma d f_den) gives 1/d, 1/(r sigma), 1/r, 1/f_den;
//  * dr/dx_i = (x r/sigma, y d/(r sigma), z r/sigma), using r^2 = (w + sigma)/2;
//  * sum_j p_j dk_j/dx_i is formed without the nine derivatives:
//      px dkx/dx_i + pz dkz/dx_i = (dr_i G' + U'_i)/d,  py dky/dx_i = c (r delta_iy - y dr_i),
//    with S = px kx + pz kz (a partial sum of k.p), G' = (px x + pz z) - 2 r S,
//    U' = (px r + pz a, 0, pz r - px a) and c = py/r^2;
//  * (k.p)^2 df/dx_i / 2 = (k.p)^2 (dq dr_i - delta_iy 2 a^2 r^3 y / f_den^2),
//    dq = (3 a^2 r^2 y^2 - r^6) / f_den^2;
// so that with F = f (k.p), Ad = F/d, B = (k.p)^2 dq - F c y, Q = Ad G' + B and
// E = F c r - (k.p)^2 2 a^2 r^3 y / f_den^2:
//      dp_i/dl = Q dr_i + Ad U'_i + delta_iy E.
// FP32 operations taken in f32x2 pairs (same rounding per half as the scalar form).
template <class T> constexpr bool kPackFloat = MGK_PACKED_AXPY != 0 && sizeof(T) == 4;

template <class T> __device__ __forceinline__ void rhs_kerr_fused(const S7<T>& s, T pt, const MP<T>& m, S7<T>& o) {
    constexpr Fuse F = Fuse::Fma;
    const T x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const T a = m.spin, a_sq = m.a_sq;
    const T y_sq = y * y;
    const T w_sq = mad<F>(z, z, mad<F>(x, x, y_sq)) - a_sq;
    const T sigma = fused_sqrt(mad<F>(w_sq, w_sq, m.four_a_sq * y_sq));
    const T r = fused_sqrt(T(0.5) * (w_sq + sigma));
    const T r_sq = r * r;
    const T d = r_sq + a_sq;
    const T f_den = mad<F>(a_sq, y_sq, r_sq * r_sq);
    const T rs = r * sigma;
    const T rsd = rs * d;
    const T inv_all = fused_rcp(rsd * f_den);  // ~r^9: finite for r below ~1.9e4 in float
    T inv_rsd, inv_fden, inv_d, inv_rs, inv_r, sxz;
    if constexpr (kPackFloat<T>) {  // products that share a factor, in pairs
        const float2 p1 = __fmul2_rn(make_float2(f_den, rsd), make_float2(inv_all, inv_all));
        inv_rsd = p1.x; inv_fden = p1.y;
        const float2 p2 = __fmul2_rn(make_float2(rs, d), make_float2(inv_rsd, inv_rsd));
        inv_d = p2.x; inv_rs = p2.y;
        const float2 p3 = __fmul2_rn(make_float2(sigma, r_sq), make_float2(inv_rs, inv_rs));
        inv_r = p3.x; sxz = p3.y;
    } else {
        inv_rsd = f_den * inv_all;
        inv_fden = rsd * inv_all;
        inv_d = rs * inv_rsd;
        inv_rs = d * inv_rsd;
        inv_r = sigma * inv_rs;
        sxz = r_sq * inv_rs;
    }
    T drx, drz, kx, kz;
    const T dry = y * (d * inv_rs);
    const T r_cu = r_sq * r;
    const T f_ = (T(2) * r_cu) * inv_fden;
    const T kx_num = mad<F>(r, x, -(a * z));
    const T kz_num = mad<F>(r, z, a * x);
    if constexpr (kPackFloat<T>) {  // (x, z) pairs: one f32x2 multiply for two
        const float2 dr = __fmul2_rn(make_float2(x, z), make_float2(sxz, sxz));
        const float2 kk = __fmul2_rn(make_float2(kx_num, kz_num), make_float2(inv_d, inv_d));
        drx = dr.x; drz = dr.y; kx = kk.x; kz = kk.y;
    } else {
        drx = x * sxz; drz = z * sxz;
        kx = kx_num * inv_d; kz = kz_num * inv_d;
    }
    const T ky = y * inv_r;
    const T S = mad<F>(pz, kz, px * kx);
    const T kTp = mad<F>(py, ky, S) - pt;
    T f_kTp, kTp2;
    if constexpr (kPackFloat<T>) {
        const float2 p4 = __fmul2_rn(make_float2(f_, kTp), make_float2(kTp, kTp));
        f_kTp = p4.x; kTp2 = p4.y;
    } else {
        f_kTp = f_ * kTp;
        kTp2 = kTp * kTp;
    }
    const T two_r = r + r;
    const T Gp = mad<F>(-two_r, S, mad<F>(pz, z, px * x));
    const T Ad = f_kTp * inv_d;
    const T Ux = mad<F>(px, r, pz * a);
    const T Uz = mad<F>(pz, r, -(px * a));
    const T c = py * (inv_r * inv_r);
    const T cy = c * y;
    const T inv_fden_sq = inv_fden * inv_fden;
    const T dq = mad<F>(m.three_a_sq * r_sq, y_sq, -(r_cu * r_cu)) * inv_fden_sq;
    const T B = mad<F>(kTp2, dq, -(f_kTp * cy));
    const T E = mad<F>(-kTp2, ((m.two_a_sq * r_cu) * y) * inv_fden_sq, f_kTp * (c * r));
    const T Q = mad<F>(Ad, Gp, B);
    if constexpr (kPackFloat<T>) {
        const float2 nf = make_float2(-f_kTp, -f_kTp);
        const float2 oxz = __ffma2_rn(nf, make_float2(kx, kz), make_float2(px, pz));
        const float2 au = __fmul2_rn(make_float2(Ad, Ad), make_float2(Ux, Uz));
        const float2 opxz = __ffma2_rn(make_float2(Q, Q), make_float2(drx, drz), au);
        o.x = oxz.x; o.z = oxz.y; o.px = opxz.x; o.pz = opxz.y;
    } else {
        o.x = mad<F>(-f_kTp, kx, px);
        o.z = mad<F>(-f_kTp, kz, pz);
        o.px = mad<F>(Q, drx, Ad * Ux);
        o.pz = mad<F>(Q, drz, Ad * Uz);
    }
    o.y = mad<F>(-f_kTp, ky, py);
    o.t = f_kTp - pt;
    o.py = mad<F>(Q, dry, E);
}

// Schwarzschild, fused formulation: with a = 0, k = x/r, f = 2 m/r,
// dk_i/dx_j = (delta_ij - k_i k_j)/r and df/dx_i = -f k_i/r, so
//   dp_i/dl = (f (k.p)/r) (p_i - k_i (k.p_s + (k.p)/2)),  k.p = k.p_s - p_t.
template <class T>
__device__ __forceinline__ void rhs_schwarzschild_fused(const S7<T>& s, T pt, T mass_sign, S7<T>& o) {
    constexpr Fuse F = Fuse::Fma;
    const T x = s.x, y = s.y, z = s.z, px = s.px, py = s.py, pz = s.pz;
    const T r = fused_sqrt(mad<F>(z, z, mad<F>(y, y, x * x)));
    const T inv_r = fused_rcp(r);
    T kx, kz;
    if constexpr (kPackFloat<T>) {
        const float2 k = __fmul2_rn(make_float2(x, z), make_float2(inv_r, inv_r));
        kx = k.x; kz = k.y;
    } else {
        kx = x * inv_r; kz = z * inv_r;
    }
    const T ky = y * inv_r;
    const T kp = mad<F>(pz, kz, mad<F>(py, ky, px * kx));
    const T kTp = kp - pt;
    const T fk = ((mass_sign * T(2)) * inv_r) * kTp;
    const T sc = fk * inv_r;
    const T q = mad<F>(T(0.5), kTp, kp);
    if constexpr (kPackFloat<T>) {
        // fma(-k, q, p) == fma(k, -q, p): negation is exact
        const float2 K = make_float2(kx, kz), P = make_float2(px, pz);
        const float2 oxz = __ffma2_rn(make_float2(-fk, -fk), K, P);
        const float2 opxz = __fmul2_rn(make_float2(sc, sc), __ffma2_rn(K, make_float2(-q, -q), P));
        o.x = oxz.x; o.z = oxz.y; o.px = opxz.x; o.pz = opxz.y;
    } else {
        o.x = mad<F>(-fk, kx, px);
        o.z = mad<F>(-fk, kz, pz);
        o.px = sc * mad<F>(-kx, q, px);
        o.pz = sc * mad<F>(-kz, q, pz);
    }
    o.y = mad<F>(-fk, ky, py);
    o.t = fk - pt;
    o.py = sc * mad<F>(-ky, q, py);
}

// Minkowski, metric_minkowski.cuh:8-13.
template <class T> __device__ __forceinline__ void rhs_minkowski(const S7<T>& s, T pt, S7<T>& o) {
    o.x = s.px; o.y = s.py; o.z = s.pz; o.t = -pt;
    o.px = T(0); o.py = T(0); o.pz = T(0);
}

// The right-hand side and the capture test of the metric with tag METRIC,
// through its plugin (metric<METRIC>::geodesic_rhs / in_domain).
template <int METRIC, Fuse F, class T>
__device__ __forceinline__ void rhs(const S7<T>& s, T pt, const MP<T>& m, S7<T>& o) {
    metric<METRIC>::template geodesic_rhs<F, T>(s, pt, m, o);
}
template <int METRIC, class T> __device__ __forceinline__ bool in_domain(T x, T y, T z, const MP<T>& m) {
    return metric<METRIC>::template in_domain<T>(x, y, z, m);
}

// kerr_schild_r, metric_kerr.cuh:8-13 (host or device).
template <class T> MGK_HD T kerr_schild_r(T x, T y, T z, T a) {
    T R = (x * x + y * y + z * z - a * a);
    T r_squared = T(0.5) * R + T(0.5) * sqrt(R * R + T(4) * a * a * y * y);
    return sqrt(r_squared);
}

// ------------------------------------------------------------- RKF45
// Fehlberg 4(5) tableau as written in internal_math.h:2169-2177.
template <class T> struct FB {
    static constexpr T a21 = T(1) / T(4);
    static constexpr T a31 = T(3) / T(32), a32 = T(9) / T(32);
    static constexpr T a41 = T(1932) / T(2197), a42 = T(7200) / T(2197), a43 = T(7296) / T(2197);
    static constexpr T a51 = T(439) / T(216), a52 = T(8), a53 = T(3680) / T(513), a54 = T(845) / T(4104);
    static constexpr T a61 = T(8) / T(27), a62 = T(2), a63 = T(3544) / T(2565), a64 = T(1859) / T(4104),
                       a65 = T(11) / T(40);
    static constexpr T b1 = T(16) / T(135), b3 = T(6656) / T(12825), b4 = T(28561) / T(56430), b5 = T(9) / T(50),
                       b6 = T(2) / T(55);
    static constexpr T e1 = T(-1) / T(360), e3 = T(128) / T(4275), e4 = T(2197) / T(75240), e5 = T(1) / T(50),
                       e6 = T(2) / T(55);
};

template <Fuse F, class T> __device__ __forceinline__ S7<T> axpy(T c, const S7<T>& k, const S7<T>& y) {
    return S7<T>{mad<F>(c, k.x, y.x), mad<F>(c, k.y, y.y), mad<F>(c, k.z, y.z), mad<F>(c, k.t, y.t),
                 mad<F>(c, k.px, y.px), mad<F>(c, k.py, y.py), mad<F>(c, k.pz, y.pz)};
}
#if MGK_PACKED_AXPY
// The FP32 fused form as three packed f32x2 FMAs and one scalar: each half
// rounds exactly as fmaf, for one issue slot per pair (the integrator is
// bound by instruction issue).  The pairs (x, z) and (px, pz) are the ones
// the fused Kerr RHS also works on.
template <> __device__ __forceinline__ S7<float> axpy<Fuse::Fma, float>(float c, const S7<float>& k,
                                                                        const S7<float>& y) {
    const float2 cc = make_float2(c, c);
    const float2 xz = __ffma2_rn(cc, make_float2(k.x, k.z), make_float2(y.x, y.z));
    const float2 pxz = __ffma2_rn(cc, make_float2(k.px, k.pz), make_float2(y.px, y.pz));
    const float2 yt = __ffma2_rn(cc, make_float2(k.y, k.t), make_float2(y.y, y.t));
    return S7<float>{xz.x, yt.x, xz.y, yt.y, pxz.x, __fmaf_rn(c, k.py, y.py), pxz.y};
}
#endif
template <class T> __device__ __forceinline__ S7<T> scl(T c, const S7<T>& k) {
    return S7<T>{c * k.x, c * k.y, c * k.z, c * k.t, c * k.px, c * k.py, c * k.pz};
}
template <class T, class U> __device__ __forceinline__ S7<T> cvt(const S7<U>& s) {
    return S7<T>{T(s.x), T(s.y), T(s.z), T(s.t), T(s.px), T(s.py), T(s.pz)};
}

// One attempt: six stages, the 5th-order solution y1 and the stages k.
template <int METRIC, Fuse F, class T>
__device__ __forceinline__ void rkf45_stages(const S7<T>& y0, T pt, T h, const MP<T>& m, S7<T>& y1, S7<T> k[6]) {
    using C = FB<T>;
    rhs<METRIC, F, T>(y0, pt, m, k[0]);
    rhs<METRIC, F, T>(axpy<F>(C::a21 * h, k[0], y0), pt, m, k[1]);
    rhs<METRIC, F, T>(axpy<F>(C::a32 * h, k[1], axpy<F>(C::a31 * h, k[0], y0)), pt, m, k[2]);
    rhs<METRIC, F, T>(axpy<F>(C::a43 * h, k[2], axpy<F>(-(C::a42 * h), k[1], axpy<F>(C::a41 * h, k[0], y0))), pt, m,
                      k[3]);
    rhs<METRIC, F, T>(axpy<F>(-(C::a54 * h), k[3],
                              axpy<F>(C::a53 * h, k[2], axpy<F>(-(C::a52 * h), k[1], axpy<F>(C::a51 * h, k[0], y0)))),
                      pt, m, k[4]);
    rhs<METRIC, F, T>(
        axpy<F>(-(C::a65 * h), k[4],
                axpy<F>(C::a64 * h, k[3],
                        axpy<F>(-(C::a63 * h), k[2], axpy<F>(C::a62 * h, k[1], axpy<F>(-(C::a61 * h), k[0], y0))))),
        pt, m, k[5]);
    y1 = axpy<F>(C::b6 * h, k[5],
                 axpy<F>(-(C::b5 * h), k[4],
                         axpy<F>(C::b4 * h, k[3], axpy<F>(C::b3 * h, k[2], axpy<F>(C::b1 * h, k[0], y0)))));
}

template <Fuse F, class T> __device__ __forceinline__ S7<T> rkf45_error(T h, const S7<T> k[6]) {
    using C = FB<T>;
    return axpy<F>(-(C::e6 * h), k[5],
                   axpy<F>(-(C::e5 * h), k[4], axpy<F>(C::e4 * h, k[3], axpy<F>(C::e3 * h, k[2], scl(C::e1 * h, k[0])))));
}

// RMS error norm, relativity_utilities.cuh:15-29 (component order t, x, y, z,
// then momentum).  The p_t error term is identically zero (dp_t/dlambda = 0)
// and the scale is positive (abs_tol > 0 is enforced), so it is left out.
template <Fuse F, class T>
__device__ __forceinline__ T rms_error(const S7<T>& e, const S7<T>& y0, const S7<T>& y1, T atol, T rtol) {
    auto term = [&](T ei, T a0, T a1) { return ei / mad<F>(rtol, fmax(fabs(a0), fabs(a1)), atol); };
    T s0 = term(e.t, y0.t, y1.t), s1 = term(e.x, y0.x, y1.x), s2 = term(e.y, y0.y, y1.y), s3 = term(e.z, y0.z, y1.z);
    T s5 = term(e.px, y0.px, y1.px), s6 = term(e.py, y0.py, y1.py), s7 = term(e.pz, y0.pz, y1.pz);
    T acc = s0 * s0;
    acc = mad<F>(s1, s1, acc);
    acc = mad<F>(s2, s2, acc);
    acc = mad<F>(s3, s3, acc);
    acc = mad<F>(s5, s5, acc);
    acc = mad<F>(s6, s6, acc);
    acc = mad<F>(s7, s7, acc);
    return sqrt(acc / T(8));
}

// ---------------------------------------------------------- step control
// Step-size factor err^(-1/5) for the proposal h_new = 0.9 h err^(-1/5)
// (internal_math.h:2190 writes it as pow(1/err, 0.2)).  Computed with IEEE
// operations only, so the CPU oracle reproduces it bit for bit: split
// a = m 2^e with m in [1, 2), e = 5q + r; start from a quadratic fit of
// m^(-1/5) times 2^(-r/5) 2^(-q), then Newton steps y <- y (6 - a y^5) / 5.
// 2^(-r/5), r = 0..4, for inv_root5 (constant memory: one indexed load).
__constant__ float kRoot5Scale[5] = {1.0f, 0.8705505632961241f, 0.757858283255199f, 0.6597539553864471f,
                                     0.5743491774985174f};
__constant__ double kRoot5ScaleD[5] = {1.0, 0.8705505632961241, 0.757858283255199, 0.6597539553864471,
                                       0.5743491774985174};

__device__ __forceinline__ float inv_root5(float a) {
    if (!(a <= 3.4028235e38f)) return 0.0f;  // err = inf: no step
    const uint32_t b = __float_as_uint(a);
    const int ex = int(b >> 23) - 127;
    const float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
    const int q = ex >= 0 ? ex / 5 : -((4 - ex) / 5);
    const int r = ex - 5 * q;
    float y = __fmaf_rn(__fmaf_rn(0.05264997f, m, -0.28570902f), m, 1.23209767f);
    y = y * kRoot5Scale[r];
    y = y * __uint_as_float(uint32_t(127 - q) << 23);
    // the fit is within 1e-3; one Newton step leaves 3e-6, ample for a step proposal
    const float y2 = y * y, y4 = y2 * y2, t = a * (y4 * y);
    return y * __fmaf_rn(-0.2f, t, 1.2f);
}
__device__ __forceinline__ double inv_root5(double a) {
    if (!(a <= 1.7976931348623157e308)) return 0.0;
    const uint64_t b = uint64_t(__double_as_longlong(a));
    const int ex = int(b >> 52) - 1023;
    const double m = __longlong_as_double((long long)((b & 0xfffffffffffffull) | 0x3ff0000000000000ull));
    const int q = ex >= 0 ? ex / 5 : -((4 - ex) / 5);
    const int r = ex - 5 * q;
    double y = __fma_rn(__fma_rn(0.05264997, m, -0.28570902), m, 1.23209767);
    y = y * kRoot5ScaleD[r];
    y = y * __longlong_as_double((long long)(uint64_t(1023 - q) << 52));
#pragma unroll
    for (int it = 0; it < 3; ++it) {
        double y2 = y * y, y4 = y2 * y2, t = a * (y4 * y);
        y = y * __fma_rn(-0.2, t, 1.2);
    }
    return y;
}

// Reciprocal of a positive normal float from integer and FMA operations only
// (bit-identical on the CPU): the seed 0x7EF311C3 - bits(x) is within 12 %,
// one Newton step y <- y (2 - x y) brings it within 1.44 %, from below.  A
// norm term e_i / scale_i is then at most 1.44 % small: the MIXED error
// control accepts steps whose error is up to 1.5 % above the tolerance.
__device__ __forceinline__ float rcp_norm(float x) {
    const float y = __uint_as_float(0x7EF311C3u - __float_as_uint(x));
    return y * __fmaf_rn(-x, y, 2.0f);
}

// MIXED RMS norm of the unscaled error E (the step's error is h E): as
// rms_error<Fuse::Fma, float> of h E, with the divisions replaced by rcp_norm
// and h applied once, to the sum of squares.
__device__ __forceinline__ float rms_error_mixed(const S7<float>& e, const S7<float>& y0, const S7<float>& y1,
                                                 float h, float atol, float rtol) {
    auto term = [&](float ei, float a0, float a1) {
        return ei * rcp_norm(__fmaf_rn(rtol, fmaxf(fabsf(a0), fabsf(a1)), atol));
    };
    float s0 = term(e.t, y0.t, y1.t), s1 = term(e.x, y0.x, y1.x), s2 = term(e.y, y0.y, y1.y);
    float s3 = term(e.z, y0.z, y1.z);
    float s5 = term(e.px, y0.px, y1.px), s6 = term(e.py, y0.py, y1.py), s7 = term(e.pz, y0.pz, y1.pz);
    float acc = s0 * s0;
    acc = __fmaf_rn(s1, s1, acc);
    acc = __fmaf_rn(s2, s2, acc);
    acc = __fmaf_rn(s3, s3, acc);
    acc = __fmaf_rn(s5, s5, acc);
    acc = __fmaf_rn(s6, s6, acc);
    acc = __fmaf_rn(s7, s7, acc);
    return sqrtf(acc * ((h * h) * 0.125f));
}

// The unscaled error estimate E = sum_j (b5_j - b4_j) k_j of the Fehlberg
// pair in FP64 from the FP32 stages (the step's error is h E).
template <class T> __device__ __forceinline__ S7<T> rkf45_error_unscaled(const S7<T> k[6]) {
    using C = FB<T>;
    return axpy<Fuse::Fma>(-C::e6, k[5], axpy<Fuse::Fma>(-C::e5, k[4], axpy<Fuse::Fma>(C::e4, k[3],
                           axpy<Fuse::Fma>(C::e3, k[2], scl(C::e1, k[0])))));
}

// The unscaled error estimate in FP32 over the stage differences: the
// Fehlberg error weights sum to zero (-1/360 + 128/4275 + 2197/75240 - 1/50
// - 2/55 = 0), so E = sum_j e_j (k_j - k_1).  Written this way the common
// part of the stages cancels exactly (the differences are formed first, each
// rounded relative to itself), and the FP32 rounding left in E is of order
// 2^-24 h |dk/dlambda| instead of 2^-24 |k|: far below any tolerance the
// step control works to.  The pairs run as f32x2 instructions.
__device__ __forceinline__ S7<float> rkf45_error_delta(const S7<float> k[6]) {
    using C = FB<float>;
    auto dif = [](const S7<float>& a, const S7<float>& b) {
        const float2 xz = __fadd2_rn(make_float2(a.x, a.z), make_float2(-b.x, -b.z));
        const float2 pxz = __fadd2_rn(make_float2(a.px, a.pz), make_float2(-b.px, -b.pz));
        const float2 yt = __fadd2_rn(make_float2(a.y, a.t), make_float2(-b.y, -b.t));
        return S7<float>{xz.x, yt.x, xz.y, yt.y, pxz.x, a.py - b.py, pxz.y};
    };
    const S7<float> d3 = dif(k[2], k[0]), d4 = dif(k[3], k[0]), d5 = dif(k[4], k[0]), d6 = dif(k[5], k[0]);
    return axpy<Fuse::Fma>(-C::e6, d6, axpy<Fuse::Fma>(-C::e5, d5, axpy<Fuse::Fma>(C::e4, d4, scl(C::e3, d3))));
}

// MIXED control: the error estimate (whose terms cancel badly when summed
// directly in FP32) over the stage differences in FP32 (MGK_MIXED_ERR_F32,
// the default) or summed directly in FP64; its norm and the proposal need
// only a few digits and run in FP32.
#ifndef MGK_MIXED_ERR_F32
#define MGK_MIXED_ERR_F32 1
#endif
__device__ __forceinline__ void control_mixed(const S7<float>& y0, const S7<float>& y1, const S7<float> k[6],
                                              float h, const MP<float>& m, float& h_next, bool& ok) {
#if MGK_MIXED_ERR_F32
    S7<float> e = rkf45_error_delta(k);
#else
    S7<double> kd[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) kd[i] = cvt<double>(k[i]);
    S7<float> e = cvt<float>(rkf45_error_unscaled<double>(kd));
#endif
    float err = rms_error_mixed(e, y0, y1, h, m.abs_tol, m.rel_tol);
    float safe = err > 1e-30f ? err : 1e-30f;
    float hn = (0.9f * h) * inv_root5(safe);
    if (hn > m.h_max) hn = m.h_max;
    h_next = hn;
    ok = safe < 1.0f;
}

// FP64 control (F64 mode, and MIXED attempts inside the FP64 band).
__device__ __forceinline__ void control_f64(const S7<double>& y0, const S7<double>& y1, const S7<double> k[6],
                                            double h, const MP<double>& m, double& h_next, bool& ok) {
    S7<double> e = rkf45_error<Fuse::Fma, double>(h, k);
    double err = rms_error<Fuse::Fma, double>(e, y0, y1, m.abs_tol, m.rel_tol);
    double safe = err > 1e-30 ? err : 1e-30;
    double hn = (0.9 * h) * inv_root5(safe);
    if (hn > m.h_max) hn = m.h_max;
    h_next = hn;
    ok = safe < 1.0;
}

// Reference step proposal 0.9*h*pow(1/err, 0.2f) (internal_math.h:2179-2195)
// in float, with the pow evaluated in double and rounded once to float.
__device__ __forceinline__ float propose_h_ref(float h, float err_safe, float h_max) {
    float g = float(pow(double(1.0f / err_safe), double(0.2f)));
    float h_new = (0.9f * h) * g;
    if (h_new > h_max) h_new = h_max;
    return h_new;
}

}  // namespace mgk
