// CPU oracle for the geodesic hot path (TEST INFRASTRUCTURE ONLY).
//
// This header restates, on the CPU, the algorithm of Magik's relativistic
// integrator so that the CUDA path in magik_b200/csrc can be checked against
// it.  Only tests/, the smoke check and the CPU-baseline leg of bench.py may
// use it; the product never links it.
//
// Parity is pinned: in FP32 "reference" mode (Fuse::None, float, powf) this
// restatement reproduces the step list of the reference's own CPU tracer
// (src/renderer/relativity/host_trace_geodesic.cu, compiled unchanged from the
// reference sources into oracle/_ref by oracle/Makefile) bit for bit; the
// tests check that on thousands of seeded initial conditions.
//
// Everything is templated on the scalar type T (float / double / an
// op-counting type) and on an FMA policy F:
//   Fuse::None - every a*b+c is a separately rounded multiply and add, in the
//                reference's expression order (what g++ emits for x86-64).
//   Fuse::Fma  - the same expression tree with the multiply-add pairs marked
//                by mad() fused into one correctly rounded fma(), and the
//                five RHS quotients formed from one reciprocal.  The CUDA
//                kernels use the same tree with __fmaf_rn / __fma_rn at the
//                same sites, so both sides round identically.
// Build with -ffp-contract=off so the compiler adds no fusion of its own.
#pragma once

#include <cmath>
#include <limits>
#include <cstdint>
#include <cstring>
#include <type_traits>

namespace orc {

enum class Fuse { None, Fma };

// ---------------------------------------------------------------- arithmetic
template <Fuse F, class T> inline T mad(T a, T b, T c) {
    if constexpr (F == Fuse::Fma) {
        using std::fma;
        return fma(a, b, c);
    } else {
        return a * b + c;
    }
}
template <class T> inline T sq_root(T v) { using std::sqrt; return sqrt(v); }

// The square root and reciprocal of the fused RHS in float (the library's
// MIXED mode evaluates them from hardware approximations with one FMA
// correction each; dev_physics.cuh: msqrt, mrcp), defined by their results:
//   msqrt(a) = IEEE sqrt(max(a, 2^-100)), NaN for a = +inf;
//   mrcp(b)  = IEEE 1/b for normal b with a normal reciprocal, +-0 for
//              |b| > 2^126, NaN for b = +-0, subnormal or infinite.
// std::fmax, like the device's fmaxf, returns the other operand for a NaN.
inline float msqrt(float a) {
    a = std::fmax(a, 0x1p-100f);
    if (std::isinf(a)) return std::numeric_limits<float>::quiet_NaN();
    return std::sqrt(a);
}
inline float mrcp(float b) {
    const float ab = std::fabs(b);
    if (std::isnan(b) || ab < 0x1p-126f || std::isinf(b)) return std::numeric_limits<float>::quiet_NaN();
    if (ab > 0x1p126f) return std::copysign(0.0f, b);
    return 1.0f / b;
}
template <class T> inline T fused_sqrt(T v) { return sq_root(v); }
template <> inline float fused_sqrt<float>(float v) { return msqrt(v); }
template <class T> inline T fused_rcp(T v) { return T(1) / v; }
template <> inline float fused_rcp<float>(float v) { return mrcp(v); }
template <class T> inline T fmax_(T a, T b) { using std::fmax; return fmax(a, b); }
template <class T> inline T fabs_(T a) { using std::fabs; return fabs(a); }

template <class T> struct V4 { T x, y, z, t; };
template <class T> struct V3 { T x, y, z; };
template <class T> struct GState { V4<T> x; V4<T> p; };  // four-position, covariant four-momentum

// ------------------------------------------------------------------ metrics
// Kerr RHS, Kerr-Schild Cartesian form, spin axis +y.
// Follows src/renderer/relativity/metric_kerr.cuh:38-105 expression by
// expression (Fuse::None reproduces it exactly).
template <Fuse F, class T> inline GState<T> rhs_kerr(const GState<T>& s, T a) {
    const T x = s.x.x, y = s.x.y, z = s.x.z;
    const T pt = s.p.t, px = s.p.x, py = s.p.y, pz = s.p.z;
    const T one = T(1), half = T(0.5), two = T(2);

    T a_sq = a * a;
    T y_sq = y * y;
    T w_sq = mad<F>(z, z, mad<F>(y, y, x * x)) - a_sq;
    T sigma = sq_root(mad<F>(w_sq, w_sq, (T(4) * a_sq) * y_sq));
    T r = sq_root(half * (w_sq + sigma));
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

    GState<T> o;
    o.x = V4<T>{mad<F>(-f_kTp, kx, px), mad<F>(-f_kTp, ky, py), mad<F>(-f_kTp, kz, pz), -pt + f_kTp};
    o.p = V4<T>{mad<F>(f_kTp, bx, half_kTp_sq * dfx), mad<F>(f_kTp, by, half_kTp_sq * dfy),
                mad<F>(f_kTp, bz, half_kTp_sq * dfz), T(0)};
    return o;
}

// Schwarzschild RHS; src/renderer/relativity/metric_schwarzschild.cuh:8-72.
// mass_sign = +1 or -1 (negative mass support, :45-47).
template <Fuse F, class T> inline GState<T> rhs_schwarzschild(const GState<T>& s, T mass_sign) {
    const T x = s.x.x, y = s.x.y, z = s.x.z;
    const T pt = s.p.t, px = s.p.x, py = s.p.y, pz = s.p.z;
    const T one = T(1), half = T(0.5), two = T(2);

    T w_sq = mad<F>(z, z, mad<F>(y, y, x * x));
    T sigma = w_sq;
    T r = sq_root(half * (w_sq + sigma));
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
    T scale = (half * inv_r) * mad<F>(w_sq, inv_sigma, one);
    T drx = x * scale, dry = y * scale, drz = z * scale;

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

    GState<T> o;
    o.x = V4<T>{mad<F>(-f_kTp, kx, px), mad<F>(-f_kTp, ky, py), mad<F>(-f_kTp, kz, pz), -pt + f_kTp};
    o.p = V4<T>{mad<F>(f_kTp, bx, half_kTp_sq * dfx), mad<F>(f_kTp, by, half_kTp_sq * dfy),
                mad<F>(f_kTp, bz, half_kTp_sq * dfz), T(0)};
    return o;
}

// Fused formulation of the Kerr RHS (the library's MIXED and F64 modes): the
// same Hamiltonian right-hand side as rhs_kerr, rearranged so that one
// reciprocal gives 1/d, 1/(r sigma), 1/r and 1/f_den, dr/dx_i = (x r/sigma,
// y d/(r sigma), z r/sigma), and sum_j p_j dk_j/dx_i needs no derivative of k:
//   px dkx/dx_i + pz dkz/dx_i = (dr_i G' + U'_i)/d,  py dky/dx_i = (py/r^2)(r delta_iy - y dr_i),
// S = px kx + pz kz, G' = (px x + pz z) - 2 r S, U' = (px r + pz a, 0, pz r - px a),
// so that dp_i/dl = Q dr_i + Ad U'_i + delta_iy E with F = f (k.p), Ad = F/d,
// B = (k.p)^2 dq - F c y, Q = Ad G' + B, E = F c r - (k.p)^2 2 a^2 r^3 y/f_den^2,
// c = py/r^2, dq = (3 a^2 r^2 y^2 - r^6)/f_den^2.
// The device code evaluates exactly these operations in this order.
template <class T> inline GState<T> rhs_kerr_fused(const GState<T>& s, T a) {
    constexpr Fuse F = Fuse::Fma;
    const T x = s.x.x, y = s.x.y, z = s.x.z;
    const T pt = s.p.t, px = s.p.x, py = s.p.y, pz = s.p.z;
    const T a_sq = a * a;
    const T y_sq = y * y;
    const T w_sq = mad<F>(z, z, mad<F>(x, x, y_sq)) - a_sq;
    const T sigma = fused_sqrt(mad<F>(w_sq, w_sq, (T(4) * a_sq) * y_sq));
    const T r = fused_sqrt(T(0.5) * (w_sq + sigma));
    const T r_sq = r * r;
    const T d = r_sq + a_sq;
    const T f_den = mad<F>(a_sq, y_sq, r_sq * r_sq);
    const T rs = r * sigma;
    const T rsd = rs * d;
    const T inv_all = fused_rcp(rsd * f_den);
    const T inv_rsd = f_den * inv_all;
    const T inv_fden = rsd * inv_all;
    const T inv_d = rs * inv_rsd;
    const T inv_rs = d * inv_rsd;
    const T inv_r = sigma * inv_rs;
    const T sxz = r_sq * inv_rs;
    const T drx = x * sxz, dry = y * (d * inv_rs), drz = z * sxz;
    const T r_cu = r_sq * r;
    const T f_ = (T(2) * r_cu) * inv_fden;
    const T kx_num = mad<F>(r, x, -(a * z));
    const T kz_num = mad<F>(r, z, a * x);
    const T kx = kx_num * inv_d, kz = kz_num * inv_d, ky = y * inv_r;
    const T S = mad<F>(pz, kz, px * kx);
    const T kTp = mad<F>(py, ky, S) - pt;
    const T f_kTp = f_ * kTp;
    const T kTp2 = kTp * kTp;
    const T two_r = r + r;
    const T Gp = mad<F>(-two_r, S, mad<F>(pz, z, px * x));
    const T Ad = f_kTp * inv_d;
    const T Ux = mad<F>(px, r, pz * a);
    const T Uz = mad<F>(pz, r, -(px * a));
    const T c = py * (inv_r * inv_r);
    const T cy = c * y;
    const T inv_fden_sq = inv_fden * inv_fden;
    const T dq = mad<F>((T(3) * a_sq) * r_sq, y_sq, -(r_cu * r_cu)) * inv_fden_sq;
    const T B = mad<F>(kTp2, dq, -(f_kTp * cy));
    const T E = mad<F>(-kTp2, ((T(2) * a_sq) * r_cu) * y * inv_fden_sq, f_kTp * (c * r));
    const T Q = mad<F>(Ad, Gp, B);
    GState<T> o;
    o.x = V4<T>{mad<F>(-f_kTp, kx, px), mad<F>(-f_kTp, ky, py), mad<F>(-f_kTp, kz, pz), f_kTp - pt};
    o.p = V4<T>{mad<F>(Q, drx, Ad * Ux), mad<F>(Q, dry, E), mad<F>(Q, drz, Ad * Uz), T(0)};
    return o;
}

// Fused formulation of the Schwarzschild RHS: with a = 0, k = x/r, f = 2 m/r,
//   dp_i/dl = (f (k.p)/r) (p_i - k_i (k.p_s + (k.p)/2)),  k.p = k.p_s - p_t.
template <class T> inline GState<T> rhs_schwarzschild_fused(const GState<T>& s, T mass_sign) {
    constexpr Fuse F = Fuse::Fma;
    const T x = s.x.x, y = s.x.y, z = s.x.z;
    const T pt = s.p.t, px = s.p.x, py = s.p.y, pz = s.p.z;
    const T r = fused_sqrt(mad<F>(z, z, mad<F>(y, y, x * x)));
    const T inv_r = fused_rcp(r);
    const T kx = x * inv_r, ky = y * inv_r, kz = z * inv_r;
    const T kp = mad<F>(pz, kz, mad<F>(py, ky, px * kx));
    const T kTp = kp - pt;
    const T fk = ((mass_sign * T(2)) * inv_r) * kTp;
    const T sc = fk * inv_r;
    const T q = mad<F>(T(0.5), kTp, kp);
    GState<T> o;
    o.x = V4<T>{mad<F>(-fk, kx, px), mad<F>(-fk, ky, py), mad<F>(-fk, kz, pz), fk - pt};
    o.p = V4<T>{sc * mad<F>(-kx, q, px), sc * mad<F>(-ky, q, py), sc * mad<F>(-kz, q, pz), T(0)};
    return o;
}

// Minkowski RHS; src/renderer/relativity/metric_minkowski.cuh:8-13.
template <class T> inline GState<T> rhs_minkowski(const GState<T>& s) {
    GState<T> o;
    o.x = V4<T>{s.p.x, s.p.y, s.p.z, -s.p.t};
    o.p = V4<T>{T(0), T(0), T(0), T(0)};
    return o;
}

enum MetricId : int { MINKOWSKI = 0, SCHWARZSCHILD = 1, KERR = 2 };

// Per-metric integrator parameters; mirrors the params_t of
// metric_kerr.cuh:112-123 / metric_schwarzschild.cuh:79-90.
template <class T> struct MetricParams {
    int metric;
    bool time_reversed;
    T spin;            // already sign-flipped when time_reversed (metric_kerr.cuh:141)
    T mass_sign;       // Schwarzschild only
    T horizon_scalar;  // event_horizon_scalar
    T h_max;           // 1000 (metric_kerr.cuh:143)
    T abs_tol, rel_tol;
    uint32_t n_max;
};

template <Fuse F, class T> inline GState<T> rhs(const GState<T>& s, const MetricParams<T>& m) {
    if constexpr (F == Fuse::Fma) {
        if (m.metric == KERR) return rhs_kerr_fused<T>(s, m.spin);
        if (m.metric == SCHWARZSCHILD) return rhs_schwarzschild_fused<T>(s, m.mass_sign);
    } else {
        if (m.metric == KERR) return rhs_kerr<F, T>(s, m.spin);
        if (m.metric == SCHWARZSCHILD) return rhs_schwarzschild<F, T>(s, m.mass_sign);
    }
    return rhs_minkowski<T>(s);
}

// kerr_schild_r, metric_kerr.cuh:8-13.
template <class T> inline T kerr_schild_r(T x, T y, T z, T a) {
    T R = (x * x + y * y + z * z - a * a);
    T r_squared = T(0.5) * R + T(0.5) * sq_root(R * R + T(4) * a * a * y * y);
    return sq_root(r_squared);
}

// Horizon test in_domain (true = captured).  Kerr: metric_kerr.cuh:169-175
// (NaN r counts as captured); Schwarzschild: metric_schwarzschild.cuh:136-141;
// Minkowski never captures (metric_minkowski.cuh:60-63).
template <class T> inline bool in_domain(const V4<T>& x, const MetricParams<T>& m) {
    if (m.metric == KERR) {
        if (fabs_(m.spin) > T(1)) return false;
        T r = kerr_schild_r(x.x, x.y, x.z, m.spin);
        if (((T(1) + sq_root(T(1) - m.spin * m.spin)) * m.horizon_scalar) < r) return false;
        return true;
    }
    if (m.metric == SCHWARZSCHILD) {
        T r = sq_root(x.x * x.x + x.y * x.y + x.z * x.z);
        if (m.mass_sign < T(0)) return r < T(1e-3);
        return r <= T(2) * m.horizon_scalar;
    }
    return false;
}

// ----------------------------------------------------------------- RKF45
// Controller variants.
//  Ctl::Ref   - FP32/FP64 controller exactly as internal_math.h:2160-2205 and
//               relativity_utilities.cuh:15-29 in the scalar T; pow() is the
//               C library's pow for T (powf for float).
//  Ctl::RefD  - as Ref, but the pow(1/err, 0.2f) is evaluated in double and
//               rounded to float (what the CUDA kernels do so that both sides
//               agree with the C library's correctly rounded powf).
//  Ctl::Wide  - error estimate, norm and step proposal in double, from the
//               T-valued stages (the mixed-precision mode).
enum class Ctl { Ref, RefD, Wide };

// Butcher tableau of Fehlberg 4(5) as written in internal_math.h:2169-2177.
template <class T> struct Fehlberg {
    static constexpr T a21 = T(1) / T(4);
    static constexpr T a31 = T(3) / T(32), a32 = T(9) / T(32);
    static constexpr T a41 = T(1932) / T(2197), a42 = T(7200) / T(2197), a43 = T(7296) / T(2197);
    static constexpr T a51 = T(439) / T(216), a52 = T(8), a53 = T(3680) / T(513), a54 = T(845) / T(4104);
    static constexpr T a61 = T(8) / T(27), a62 = T(2), a63 = T(3544) / T(2565), a64 = T(1859) / T(4104),
                       a65 = T(11) / T(40);
    static constexpr T b1 = T(16) / T(135), b3 = T(6656) / T(12825), b4 = T(28561) / T(56430),
                       b5 = T(9) / T(50), b6 = T(2) / T(55);
    static constexpr T e1 = T(-1) / T(360), e3 = T(128) / T(4275), e4 = T(2197) / T(75240),
                       e5 = T(1) / T(50), e6 = T(2) / T(55);
};

template <Fuse F, class T> inline V4<T> axpy4(T c, const V4<T>& k, const V4<T>& y) {
    return V4<T>{mad<F>(c, k.x, y.x), mad<F>(c, k.y, y.y), mad<F>(c, k.z, y.z), mad<F>(c, k.t, y.t)};
}
template <Fuse F, class T> inline GState<T> axpy(T c, const GState<T>& k, const GState<T>& y) {
    return GState<T>{axpy4<F>(c, k.x, y.x), axpy4<F>(c, k.p, y.p)};
}
template <class T> inline GState<T> scale(T c, const GState<T>& k) {
    return GState<T>{V4<T>{c * k.x.x, c * k.x.y, c * k.x.z, c * k.x.t},
                     V4<T>{c * k.p.x, c * k.p.y, c * k.p.z, c * k.p.t}};
}

// One RKF45 attempt: stage values, 5th-order solution and error vector.
// Same tree as internal_math.h:2169-2177 (vector operators expanded).
template <Fuse F, class T>
inline void rkf45_attempt(const GState<T>& y0, T h, const MetricParams<T>& m, GState<T>* y1, GState<T> k[6]) {
    using C = Fehlberg<T>;
    k[0] = rhs<F>(y0, m);
    k[1] = rhs<F>(axpy<F>(C::a21 * h, k[0], y0), m);
    k[2] = rhs<F>(axpy<F>(C::a32 * h, k[1], axpy<F>(C::a31 * h, k[0], y0)), m);
    k[3] = rhs<F>(axpy<F>(C::a43 * h, k[2], axpy<F>(-(C::a42 * h), k[1], axpy<F>(C::a41 * h, k[0], y0))), m);
    k[4] = rhs<F>(axpy<F>(-(C::a54 * h), k[3],
                          axpy<F>(C::a53 * h, k[2], axpy<F>(-(C::a52 * h), k[1], axpy<F>(C::a51 * h, k[0], y0)))),
                  m);
    k[5] = rhs<F>(
        axpy<F>(-(C::a65 * h), k[4],
                axpy<F>(C::a64 * h, k[3],
                        axpy<F>(-(C::a63 * h), k[2],
                                axpy<F>(C::a62 * h, k[1], axpy<F>(-(C::a61 * h), k[0], y0))))),
        m);
    *y1 = axpy<F>(C::b6 * h, k[5],
                  axpy<F>(-(C::b5 * h), k[4],
                          axpy<F>(C::b4 * h, k[3], axpy<F>(C::b3 * h, k[2], axpy<F>(C::b1 * h, k[0], y0)))));
}

template <Fuse F, class T>
inline GState<T> rkf45_error(T h, const GState<T> k[6]) {
    using C = Fehlberg<T>;
    return axpy<F>(-(C::e6 * h), k[5],
                   axpy<F>(-(C::e5 * h), k[4],
                           axpy<F>(C::e4 * h, k[3], axpy<F>(C::e3 * h, k[2], scale(C::e1 * h, k[0])))));
}

// RMS error, relativity_utilities.cuh:15-29 (component order t, x, y, z).
template <Fuse F, class T>
inline T rms_error(const GState<T>& e, const GState<T>& y0, const GState<T>& y1, T atol, T rtol) {
    auto term = [&](T ei, T a0, T a1) { return ei / mad<F>(rtol, fmax_(fabs_(a0), fabs_(a1)), atol); };
    T s0 = term(e.x.t, y0.x.t, y1.x.t), s1 = term(e.x.x, y0.x.x, y1.x.x);
    T s2 = term(e.x.y, y0.x.y, y1.x.y), s3 = term(e.x.z, y0.x.z, y1.x.z);
    T s4 = term(e.p.t, y0.p.t, y1.p.t), s5 = term(e.p.x, y0.p.x, y1.p.x);
    T s6 = term(e.p.y, y0.p.y, y1.p.y), s7 = term(e.p.z, y0.p.z, y1.p.z);
    T acc = s0 * s0;
    acc = mad<F>(s1, s1, acc);
    acc = mad<F>(s2, s2, acc);
    acc = mad<F>(s3, s3, acc);
    acc = mad<F>(s4, s4, acc);
    acc = mad<F>(s5, s5, acc);
    acc = mad<F>(s6, s6, acc);
    acc = mad<F>(s7, s7, acc);
    return sq_root(acc / T(8));
}

template <class T> inline GState<T> widen(const GState<double>& s) {
    return GState<T>{V4<T>{T(s.x.x), T(s.x.y), T(s.x.z), T(s.x.t)}, V4<T>{T(s.p.x), T(s.p.y), T(s.p.z), T(s.p.t)}};
}
template <class T> inline GState<double> to_double(const GState<T>& s) {
    return GState<double>{V4<double>{double(s.x.x), double(s.x.y), double(s.x.z), double(s.x.t)},
                          V4<double>{double(s.p.x), double(s.p.y), double(s.p.z), double(s.p.t)}};
}

// Step proposal h_new = 0.9*h*(1/err)^0.2, capped at h_max
// (internal_math.h:2179-2195).  Returns the proposal in T.
template <Ctl K, class T> inline T propose_h(T h, T err_safe, T h_max) {
    T h_new;
    if constexpr (K == Ctl::Ref) {
        using std::pow;
        h_new = (T(0.9) * h) * T(pow(T(1) / err_safe, T(0.2)));
    } else {
        T g = T(std::pow(double(T(1) / err_safe), double(T(0.2))));
        h_new = (T(0.9) * h) * g;
    }
    if (h_new > h_max) h_new = h_max;
    return h_new;
}

// Step-size factor err^(-1/5) of the MIXED and F64 controllers, IEEE
// operations only (the CUDA kernels compute the same bits): a = m 2^e with
// m in [1, 2), e = 5q + r; a quadratic fit of m^(-1/5) (within 1e-3) times
// 2^(-r/5) 2^(-q), then Newton steps y <- y (6 - a y^5) / 5 (one in float,
// three in double).
inline float inv_root5(float a) {
    if (!(a <= 3.4028235e38f)) return 0.0f;
    uint32_t b;
    std::memcpy(&b, &a, 4);
    const int ex = int(b >> 23) - 127;
    uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
    float m;
    std::memcpy(&m, &mb, 4);
    const int q = ex >= 0 ? ex / 5 : -((4 - ex) / 5);
    const int r = ex - 5 * q;
    const float D[5] = {1.0f, 0.8705505632961241f, 0.757858283255199f, 0.6597539553864471f, 0.5743491774985174f};
    float y = std::fma(std::fma(0.05264997f, m, -0.28570902f), m, 1.23209767f);
    y = y * D[r];
    uint32_t pb = uint32_t(127 - q) << 23;
    float p2;
    std::memcpy(&p2, &pb, 4);
    y = y * p2;
    const float y2 = y * y, y4 = y2 * y2, t = a * (y4 * y);
    return y * std::fma(-0.2f, t, 1.2f);
}
inline double inv_root5(double a) {
    if (!(a <= 1.7976931348623157e308)) return 0.0;
    uint64_t b;
    std::memcpy(&b, &a, 8);
    const int ex = int(b >> 52) - 1023;
    uint64_t mb = (b & 0xfffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    std::memcpy(&m, &mb, 8);
    const int q = ex >= 0 ? ex / 5 : -((4 - ex) / 5);
    const int r = ex - 5 * q;
    const double D[5] = {1.0, 0.8705505632961241, 0.757858283255199, 0.6597539553864471, 0.5743491774985174};
    double y = std::fma(std::fma(0.05264997, m, -0.28570902), m, 1.23209767);
    y = y * D[r];
    uint64_t pb = uint64_t(1023 - q) << 52;
    double p2;
    std::memcpy(&p2, &pb, 8);
    y = y * p2;
    for (int it = 0; it < 3; ++it) {
        double y2 = y * y, y4 = y2 * y2, t = a * (y4 * y);
        y = y * std::fma(-0.2, t, 1.2);
    }
    return y;
}

// FP64 control: error estimate, norm and proposal all in double.
inline void control_f64(const GState<double>& y0, const GState<double>& y1, const GState<double> k[6], double h,
                        const MetricParams<double>& m, double* h_next, bool* ok) {
    GState<double> e = rkf45_error<Fuse::Fma, double>(h, k);
    double err = rms_error<Fuse::Fma, double>(e, y0, y1, m.abs_tol, m.rel_tol);
    double safe = err > 1e-30 ? err : 1e-30;
    double hn = (0.9 * h) * inv_root5(safe);
    if (hn > m.h_max) hn = m.h_max;
    *h_next = hn;
    *ok = safe < 1.0;
}

// Reciprocal for the MIXED norm: integer seed 0x7EF311C3 - bits(x) and one
// Newton step with fma (identical to the kernels' rcp_norm; within 1.44 %,
// from below).
inline float rcp_norm(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    b = 0x7EF311C3u - b;
    float y;
    std::memcpy(&y, &b, 4);
    return y * std::fma(-x, y, 2.0f);
}

// MIXED RMS norm of the unscaled error E (the step's error is h E):
// relativity_utilities.cuh:15-29 with e_i / scale_i formed as
// E_i * rcp_norm(scale_i) and h applied once, to the sum of squares;
// component order t, x, y, z, then momentum.
inline float rms_error_mixed(const GState<float>& e, const GState<float>& y0, const GState<float>& y1, float h,
                             float atol, float rtol) {
    auto term = [&](float ei, float a0, float a1) {
        return ei * rcp_norm(std::fma(rtol, std::fmax(std::fabs(a0), std::fabs(a1)), atol));
    };
    float s0 = term(e.x.t, y0.x.t, y1.x.t), s1 = term(e.x.x, y0.x.x, y1.x.x), s2 = term(e.x.y, y0.x.y, y1.x.y);
    float s3 = term(e.x.z, y0.x.z, y1.x.z);
    float s5 = term(e.p.x, y0.p.x, y1.p.x), s6 = term(e.p.y, y0.p.y, y1.p.y), s7 = term(e.p.z, y0.p.z, y1.p.z);
    float acc = s0 * s0;
    acc = std::fma(s1, s1, acc);
    acc = std::fma(s2, s2, acc);
    acc = std::fma(s3, s3, acc);
    acc = std::fma(s5, s5, acc);
    acc = std::fma(s6, s6, acc);
    acc = std::fma(s7, s7, acc);
    return std::sqrt(acc * ((h * h) * 0.125f));
}

// The unscaled error estimate E = sum_j (b5_j - b4_j) k_j of the Fehlberg
// pair (internal_math.h:2177 without the factor h).
template <class T> inline GState<T> rkf45_error_unscaled(const GState<T> k[6]) {
    using C = Fehlberg<T>;
    return axpy<Fuse::Fma>(-C::e6, k[5], axpy<Fuse::Fma>(-C::e5, k[4], axpy<Fuse::Fma>(C::e4, k[3],
                           axpy<Fuse::Fma>(C::e3, k[2], scale(C::e1, k[0])))));
}

// The unscaled estimate in float over the stage differences: the error
// weights sum to zero, so E = e3 (k3 - k1) + e4 (k4 - k1) - e5 (k5 - k1)
// - e6 (k6 - k1); the differences first, then the weighted sum with fma.
inline GState<float> rkf45_error_delta(const GState<float> k[6]) {
    using C = Fehlberg<float>;
    auto dif = [](const GState<float>& a, const GState<float>& b) {
        GState<float> d;
        d.x = V4<float>{a.x.x - b.x.x, a.x.y - b.x.y, a.x.z - b.x.z, a.x.t - b.x.t};
        d.p = V4<float>{a.p.x - b.p.x, a.p.y - b.p.y, a.p.z - b.p.z, a.p.t - b.p.t};
        return d;
    };
    const GState<float> d3 = dif(k[2], k[0]), d4 = dif(k[3], k[0]), d5 = dif(k[4], k[0]), d6 = dif(k[5], k[0]);
    return axpy<Fuse::Fma>(-C::e6, d6, axpy<Fuse::Fma>(-C::e5, d5, axpy<Fuse::Fma>(C::e4, d4, scale(C::e3, d3))));
}

// MIXED control: the error estimate over the stage differences in float
// (rkf45_error_delta; summed directly in double when MGK_MIXED_ERR_F32 is 0);
// its norm and the proposal in float.
#ifndef MGK_MIXED_ERR_F32
#define MGK_MIXED_ERR_F32 1
#endif
inline void control_mixed(const GState<float>& y0, const GState<float>& y1, const GState<float> k[6], float h,
                          const MetricParams<float>& m, float* h_next, bool* ok) {
#if MGK_MIXED_ERR_F32
    GState<float> e = rkf45_error_delta(k);
#else
    GState<double> kd[6];
    for (int i = 0; i < 6; ++i) kd[i] = to_double(k[i]);
    GState<float> e = widen<float>(rkf45_error_unscaled<double>(kd));
#endif
    float err = rms_error_mixed(e, y0, y1, h, m.abs_tol, m.rel_tol);
    float safe = err > 1e-30f ? err : 1e-30f;
    float hn = (0.9f * h) * inv_root5(safe);
    if (hn > m.h_max) hn = m.h_max;
    *h_next = hn;
    *ok = safe < 1.0f;
}

// Result of one attempt sequence (= one accepted step of the reference).
template <class T> struct StepOut {
    GState<T> y1;
    T h_taken;
    T h_next;
    uint32_t attempts;
    uint32_t wide_attempts;  // attempts carried out entirely in double (near horizon)
};

// The reference's solve_step for one accepted step (internal_math.h:2160-2205):
// up to n_max attempts, the last one accepted whatever its error.
// Minkowski uses explicit Euler with a fixed h (metric_minkowski.cuh:49-53).
template <Fuse F, Ctl K, class T>
inline StepOut<T> solve_step(const GState<T>& y0, T h, const MetricParams<T>& m) {
    StepOut<T> o{};
    if (m.metric == MINKOWSKI) {
        GState<T> f = rhs_minkowski<T>(y0);
        o.y1 = axpy<F>(h, f, y0);
        o.h_taken = h;
        o.h_next = h;
        o.attempts = 1;
        return o;
    }
    T temp_h = h;
    GState<T> k[6];
    for (uint32_t i = 0; i < m.n_max; ++i) {
        rkf45_attempt<F, T>(y0, temp_h, m, &o.y1, k);
        ++o.attempts;
        bool ok;
        if constexpr (K == Ctl::Wide) {
            static_assert(std::is_same_v<T, double>, "the FP64 controller runs on double state");
            double hn;
            control_f64(y0, o.y1, k, temp_h, m, &hn, &ok);
            o.h_taken = temp_h;
            temp_h = hn;
        } else {
            GState<T> e = rkf45_error<F, T>(temp_h, k);
            T err = rms_error<F, T>(e, y0, o.y1, m.abs_tol, m.rel_tol);
            T safe = err > T(1e-30) ? err : T(1e-30);
            T hn = propose_h<K, T>(temp_h, safe, m.h_max);
            o.h_taken = temp_h;
            temp_h = hn;
            ok = safe < T(1);
        }
        if (ok) break;
    }
    o.h_next = temp_h;
    return o;
}

// --------------------------------------------------- frames and observers
template <class T> struct Sym4 { T tt, tx, ty, tz, xx, xy, xz, yy, yz, zz; };

// compute_g, metric_kerr.cuh:177-190 / metric_schwarzschild.cuh:143-153.
template <class T> inline Sym4<T> compute_g(const V4<T>& q, const MetricParams<T>& m) {
    if (m.metric == MINKOWSKI) return Sym4<T>{T(-1), 0, 0, 0, T(1), 0, 0, T(1), 0, T(1)};
    T f, kx, ky, kz;
    if (m.metric == KERR) {
        const T a = m.spin;
        const T r = kerr_schild_r(q.x, q.y, q.z, a);
        f = T(2) * r * r * r / (r * r * r * r + a * a * q.y * q.y);
        kx = (r * q.x - a * q.z) / (r * r + a * a);
        ky = q.y / r;
        kz = (r * q.z + a * q.x) / (r * r + a * a);
    } else {
        const T r = sq_root(q.x * q.x + q.y * q.y + q.z * q.z);
        f = T(2) * m.mass_sign / r;
        kx = q.x / r; ky = q.y / r; kz = q.z / r;
    }
    return Sym4<T>{T(-1) + f, f * kx, f * ky, f * kz, T(1) + f * kx * kx, f * kx * ky, f * kx * kz,
                   T(1) + f * ky * ky, f * ky * kz, T(1) + f * kz * kz};
}

// reference_observer, metric_kerr.cuh:207-226 / metric_schwarzschild.cuh:167-171.
template <class T> inline V4<T> reference_observer(const V4<T>& q, const MetricParams<T>& m) {
    if (m.metric == MINKOWSKI) return V4<T>{0, 0, 0, T(1)};
    if (m.metric == SCHWARZSCHILD) {
        Sym4<T> g = compute_g(q, m);
        return V4<T>{0, 0, 0, T(1) / sq_root(-g.tt)};
    }
    const T a = m.spin;
    T r = kerr_schild_r(q.x, q.y, q.z, a);
    T r_sq = r * r;
    T a_sq = a * a;
    T cos_theta = q.y / r;
    T sin2_theta = T(1) - cos_theta * cos_theta;
    T sigma = r_sq + a_sq * cos_theta * cos_theta;
    T delta = r_sq - T(2) * r + a_sq;
    T Lambda = (r_sq + a_sq) * (r_sq + a_sq) - a_sq * delta * sin2_theta;
    T u_t = sq_root(Lambda / (delta * sigma));
    T u_phi = T(2) * a * r / sq_root(Lambda * delta * sigma);
    return V4<T>{q.z * u_phi, T(0), -q.x * u_phi, u_t};
}

// inner_product, relativity_utilities.cuh:122-130.
template <class T> inline T inner_product(const Sym4<T>& g, const V4<T>& u, const V4<T>& v) {
    return g.tt * u.t * v.t + g.tx * (u.t * v.x + u.x * v.t) + g.ty * (u.t * v.y + u.y * v.t) +
           g.tz * (u.t * v.z + u.z * v.t) + g.xx * u.x * v.x + g.xy * (u.x * v.y + u.y * v.x) +
           g.xz * (u.x * v.z + u.z * v.x) + g.yy * u.y * v.y + g.yz * (u.y * v.z + u.z * v.y) + g.zz * u.z * v.z;
}
// contract (lower an index with g), relativity_utilities.cuh:132-139.
template <class T> inline V4<T> contract(const Sym4<T>& g, const V4<T>& u) {
    return V4<T>{g.tx * u.t + g.xx * u.x + g.xy * u.y + g.xz * u.z, g.ty * u.t + g.xy * u.x + g.yy * u.y + g.yz * u.z,
                 g.tz * u.t + g.xz * u.x + g.yz * u.y + g.zz * u.z, g.tt * u.t + g.tx * u.x + g.ty * u.y + g.tz * u.z};
}
template <class T> inline V4<T> add4(V4<T> a, V4<T> b) { return V4<T>{a.x + b.x, a.y + b.y, a.z + b.z, a.t + b.t}; }
template <class T> inline V4<T> sub4(V4<T> a, V4<T> b) { return V4<T>{a.x - b.x, a.y - b.y, a.z - b.z, a.t - b.t}; }
template <class T> inline V4<T> mul4(T s, V4<T> a) { return V4<T>{s * a.x, s * a.y, s * a.z, s * a.t}; }
template <class T> inline V4<T> div4(V4<T> a, T s) { return V4<T>{a.x / s, a.y / s, a.z / s, a.t / s}; }
// vector_dot_product of two 4-vectors, internal_math.h:1094-1097 (u^mu p_mu).
template <class T> inline T dot4(V4<T> a, V4<T> b) { return ((a.x * b.x) + (a.y * b.y) + (a.z * b.z)) + (a.t * b.t); }

template <class T> struct Tetrad { V4<T> t, x, y, z; };
// build_tetrad (Gram-Schmidt, order z, x, y), relativity_utilities.cuh:141-156.
template <class T> inline Tetrad<T> build_tetrad(const Sym4<T>& g, const V4<T>& X, const V4<T>& Y, const V4<T>& Z,
                                                 const V4<T>& u) {
    Tetrad<T> e;
    e.t = u;
    e.z = add4(Z, mul4(inner_product(g, Z, u), u));
    e.z = div4(e.z, sq_root(inner_product(g, e.z, e.z)));
    e.x = sub4(add4(X, mul4(inner_product(g, X, u), u)), mul4(inner_product(g, X, e.z), e.z));
    e.x = div4(e.x, sq_root(inner_product(g, e.x, e.x)));
    e.y = sub4(sub4(add4(Y, mul4(inner_product(g, Y, u), u)), mul4(inner_product(g, Y, e.z), e.z)),
               mul4(inner_product(g, Y, e.x), e.x));
    e.y = div4(e.y, sq_root(inner_product(g, e.y, e.y)));
    return e;
}
// local_to_global, relativity_utilities.cuh:158-161.
template <class T> inline V4<T> local_to_global(const Tetrad<T>& e, V4<T> l) {
    return add4(add4(add4(mul4(l.t, e.t), mul4(l.x, e.x)), mul4(l.y, e.y)), mul4(l.z, e.z));
}

}  // namespace orc
