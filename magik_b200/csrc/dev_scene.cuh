// Scene around the integrator: observer frames, camera rays, per-step
// termination tests, disk emitter, blackbody, star lookup.
//
// Frames follow relativity_utilities.cuh:57-195 and the metric files'
// compute_g / reference_observer; termination follows kernel_intersect.cu:55-138
// (traceables before the horizon) and kernel_enforce_ray_limits.cu:37-64; the
// emitter follows bxdf_utilities.cuh:89-109,156-163 (redshift, g^5 boost,
// NaN/negative clamp) with a Keplerian thin disk in place of the reference's
// boxes.  Functions marked MGK_HD also run on the host (scene set-up).
#pragma once

#include <cmath>
#include <cstdint>

#include "dev_physics.cuh"
#include "../../include/mgk.h"
#include "../src/renderer/relativity/metric.cuh"

namespace mgk {

// ------------------------------------------------------------------ RNG
// triplet_hash (internal_math.h:2027-2037) chained over (seed, stream, index, dim).
MGK_HD uint32_t triplet_hash(uint32_t x) {
    x ^= x >> 17; x *= 0xED5AD4BBu; x ^= x >> 11; x *= 0xAC4C1B51u;
    x ^= x >> 15; x *= 0x31848BABu; x ^= x >> 14;
    return x;
}
MGK_HD uint32_t rng_u32(uint64_t seed, uint32_t stream, uint32_t index, uint32_t dim) {
    uint32_t h = triplet_hash(uint32_t(seed) ^ 0x9E3779B9u);
    h = triplet_hash(h ^ uint32_t(seed >> 32));
    h = triplet_hash(h ^ stream);
    h = triplet_hash(h ^ index);
    h = triplet_hash(h ^ (dim * 0x85EBCA6Bu + 1u));
    return h;
}
MGK_HD float rng_unit(uint64_t seed, uint32_t stream, uint32_t index, uint32_t dim) {
    return float(rng_u32(seed, stream, index, dim) >> 8) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------- frames

// inner_product / contract, relativity_utilities.cuh:122-139.
template <class T> MGK_HD T inner_product(const Sym4<T>& g, const V4<T>& u, const V4<T>& v) {
    return g.tt * u.t * v.t + g.tx * (u.t * v.x + u.x * v.t) + g.ty * (u.t * v.y + u.y * v.t) +
           g.tz * (u.t * v.z + u.z * v.t) + g.xx * u.x * v.x + g.xy * (u.x * v.y + u.y * v.x) +
           g.xz * (u.x * v.z + u.z * v.x) + g.yy * u.y * v.y + g.yz * (u.y * v.z + u.z * v.y) + g.zz * u.z * v.z;
}
template <class T> MGK_HD V4<T> contract(const Sym4<T>& g, const V4<T>& u) {
    return V4<T>{g.tx * u.t + g.xx * u.x + g.xy * u.y + g.xz * u.z, g.ty * u.t + g.xy * u.x + g.yy * u.y + g.yz * u.z,
                 g.tz * u.t + g.xz * u.x + g.yz * u.y + g.zz * u.z, g.tt * u.t + g.tx * u.x + g.ty * u.y + g.tz * u.z};
}
template <class T> MGK_HD V4<T> v_add(V4<T> a, V4<T> b) { return V4<T>{a.x + b.x, a.y + b.y, a.z + b.z, a.t + b.t}; }
template <class T> MGK_HD V4<T> v_sub(V4<T> a, V4<T> b) { return V4<T>{a.x - b.x, a.y - b.y, a.z - b.z, a.t - b.t}; }
template <class T> MGK_HD V4<T> v_mul(T s, V4<T> a) { return V4<T>{s * a.x, s * a.y, s * a.z, s * a.t}; }
template <class T> MGK_HD V4<T> v_div(V4<T> a, T s) { return V4<T>{a.x / s, a.y / s, a.z / s, a.t / s}; }
// vector_dot_product of 4-vectors (internal_math.h:1094-1097): u^mu p_mu.
template <class T> MGK_HD T dot4(V4<T> a, V4<T> b) { return ((a.x * b.x) + (a.y * b.y) + (a.z * b.z)) + (a.t * b.t); }

template <class T> struct Tetrad { V4<T> t, x, y, z; };
// build_tetrad: Gram-Schmidt of the seeds against u in the order z, x, y
// (relativity_utilities.cuh:141-156).
template <class T> MGK_HD Tetrad<T> build_tetrad(const Sym4<T>& g, V4<T> X, V4<T> Y, V4<T> Z, V4<T> u) {
    Tetrad<T> e;
    e.t = u;
    e.z = v_add(Z, v_mul(inner_product(g, Z, u), u));
    e.z = v_div(e.z, T(sqrt(inner_product(g, e.z, e.z))));
    e.x = v_sub(v_add(X, v_mul(inner_product(g, X, u), u)), v_mul(inner_product(g, X, e.z), e.z));
    e.x = v_div(e.x, T(sqrt(inner_product(g, e.x, e.x))));
    e.y = v_sub(v_sub(v_add(Y, v_mul(inner_product(g, Y, u), u)), v_mul(inner_product(g, Y, e.z), e.z)),
                v_mul(inner_product(g, Y, e.x), e.x));
    e.y = v_div(e.y, T(sqrt(inner_product(g, e.y, e.y))));
    return e;
}
// local_to_global, relativity_utilities.cuh:158-161.
template <class T> MGK_HD V4<T> local_to_global(const Tetrad<T>& e, V4<T> l) {
    return v_add(v_add(v_add(v_mul(l.t, e.t), v_mul(l.x, e.x)), v_mul(l.y, e.y)), v_mul(l.z, e.z));
}

// ---------------------------------------------------------- scene table
// Per-scene constants, computed once on the host in double.
struct SceneConsts {
    double cam_pos[4];
    double u_obs[4];
    double M[4][4];       // p_mu = M . (n_x, n_y, n_z, |n|)
    double pix_a, pix_b;  // camera-frame x = (px + jx) * pix_a + pix_b
    double pix_c, pix_d;  // camera-frame y = (py + jy) * pix_c + pix_d
    double r_plus;
    double spin_t;
    double omega_sign;
};

inline SceneConsts scene_consts(const mgk_scene& s) {
    SceneConsts c{};
    const double a = s.time_reversed ? -s.spin : s.spin;
    double ci = std::cos(s.cam_incl_rad), si = std::sin(s.cam_incl_rad);
    V4<double> q{0.0, s.cam_r * ci, s.cam_r * si, 0.0};
    V4<double> X{1, 0, 0, 0}, Y{0, si, -ci, 0}, Z{0, ci, si, 0};  // right, up, back
    if (s.cam_explicit) {
        q = V4<double>{s.cam_pos[0], s.cam_pos[1], s.cam_pos[2], 0.0};
        X = V4<double>{s.cam_axes[0], s.cam_axes[1], s.cam_axes[2], 0.0};
        Y = V4<double>{s.cam_axes[3], s.cam_axes[4], s.cam_axes[5], 0.0};
        Z = V4<double>{s.cam_axes[6], s.cam_axes[7], s.cam_axes[8], 0.0};
    }
    c.cam_pos[0] = q.x; c.cam_pos[1] = q.y; c.cam_pos[2] = q.z; c.cam_pos[3] = q.t;
    V4<double> u{};
    Sym4<double> g{};
    double r_plus = 0.0;
    with_metric(s.metric, [&](auto mt) {
        using MT = decltype(mt);
        MP<double> m{};
        MT::template make_params<double>(s, m);
        u = MT::template reference_observer<double>(q.x, q.y, q.z, m);
        g = MT::template compute_g<double>(q.x, q.y, q.z, m);
        r_plus = MT::outer_horizon(s);
    });
    const double* v = s.cam_velocity;
    if (s.cam_explicit && (v[0] != 0.0 || v[1] != 0.0 || v[2] != 0.0)) {
        // rest_frame_four_velocity (relativity_utilities.cuh:163-173): the proper
        // velocity in the reference observer's tetrad, flipped when time reversed
        Tetrad<double> e0 = build_tetrad<double>(g, V4<double>{1, 0, 0, 0}, V4<double>{0, 1, 0, 0},
                                                 V4<double>{0, 0, 1, 0}, u);
        const double f = s.time_reversed ? -1.0 : 1.0;
        const double wx = f * v[0], wy = f * v[1], wz = f * v[2];
        u = local_to_global<double>(e0, V4<double>{wx, wy, wz, std::sqrt(wx * wx + wy * wy + wz * wz + 1.0)});
    }
    Tetrad<double> e = build_tetrad<double>(g, X, Y, Z, u);
    V4<double> cols[4] = {contract(g, e.x), contract(g, e.y), contract(g, e.z), contract(g, e.t)};
    for (int j = 0; j < 4; ++j) {
        c.M[0][j] = cols[j].x; c.M[1][j] = cols[j].y; c.M[2][j] = cols[j].z; c.M[3][j] = cols[j].t;
    }
    c.u_obs[0] = u.x; c.u_obs[1] = u.y; c.u_obs[2] = u.z; c.u_obs[3] = u.t;
    double tan_half = s.sensor_diag_mm / (2.0 * s.focal_length_mm);
    double W = s.width, H = s.height;
    c.pix_a = 2.0 * tan_half / W;
    c.pix_b = -tan_half;
    c.pix_c = -2.0 * tan_half / W;
    c.pix_d = tan_half * H / W;
    c.r_plus = r_plus;
    c.spin_t = a;
    c.omega_sign = s.time_reversed ? -1.0 : 1.0;
    return c;
}

// Device-side copy of everything a kernel needs, in the kernel's scalar T.
template <class T> struct DevScene {
    MP<T> m;
    MP<double> md;     // the same parameters in double (MIXED-mode FP64 attempts)
    T cam[4];
    T u_obs[4];
    T M[4][4];
    T pix_a, pix_b, pix_c, pix_d;
    T h0;
    T disk_r_in, disk_r_out, disk_T_in;
    T disk_lo, disk_hi;  // chord pre-test window of the disk
    T escape_r2;
    T spin_phys, omega_sign;
    T kerr_a;          // spin used by the disk radius (0 unless Kerr)
    double r_plus;     // for the FP64 band test
    double band_pre2;  // (r_plus + band + margin)^2 + a^2: Euclidean pre-check of the band
    double atol_d, rtol_d, hmax_d, spin_d;
    T star_inv_r2;
    T lambda[MGK_MAX_BINS];
    T planck_a[MGK_MAX_BINS];  // 2 h c^2 / lambda_k^5
    T planck_b[MGK_MAX_BINS];  // h c / (k_B lambda_k)
    float xyz_w[3 * MGK_MAX_BINS];
    uint64_t seed;
    uint32_t width, height, spp, n_bins, max_steps, disk_on;
    int32_t metric;
    float inv_spp;
    uint32_t sample_offset;  // the frame's index of this render's first sample
    // MGK_SPECTRAL_SAMPLED
    uint32_t spectral_mode;
    float cmf_icdf[MGK_CMF_ICDF_ENTRIES];  // CIE inverse CDF, nm
    T planck_c1, planck_c2;  // 2 h c^2 and h c / k_B (SI), for the sampled wavelength
    T sensor_gain;           // radiance * throughput -> sensor irradiance (device_color_utilities.cuh:22-29)
    T lambda_lo, dlambda;    // bin edges lambda_lo + k dlambda, nm
    T inv_sigma_sqrt2;       // 1 / (redistribution sigma * sqrt 2), 1/nm
    // room scene (walls and light as axis-aligned boxes)
    uint32_t room_on, room_limit;
    T room_lo[3], room_hi[3];
    T light_lo[3], light_hi[3];
    T light_scale;
    uint64_t ray_base;  // global index of the launch's ray 0 (per-ray random numbers)
};

// ------------------------------------------------------------ camera
// One camera ray: jittered pinhole direction -> local photon direction in
// the observer's tetrad -> covariant momentum; also c0 = u_obs . p.
template <Fuse F, class T>
__device__ __forceinline__ void camera_ray(const DevScene<T>& P, uint64_t ray_id, S7<T>& y, T& pt, T& c0) {
    uint32_t pixel = uint32_t(ray_id / P.spp), sample = uint32_t(ray_id % P.spp) + P.sample_offset;
    uint32_t px = pixel % P.width, py = pixel / P.width;
    T jx = T(rng_unit(P.seed, sample, pixel, 0));
    T jy = T(rng_unit(P.seed, sample, pixel, 1));
    T sx = mad<F>(T(px) + jx, P.pix_a, P.pix_b);
    T sy = mad<F>(T(py) + jy, P.pix_c, P.pix_d);
    T len = sqrt(mad<F>(sy, sy, mad<F>(sx, sx, T(1))));
    T nx = sx / len, ny = sy / len, nz = T(-1) / len;
    T nl = sqrt(mad<F>(nz, nz, mad<F>(ny, ny, nx * nx)));
    T p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        T acc = P.M[i][0] * nx;
        acc = mad<F>(P.M[i][1], ny, acc);
        acc = mad<F>(P.M[i][2], nz, acc);
        acc = mad<F>(P.M[i][3], nl, acc);
        p[i] = acc;
    }
    y = S7<T>{P.cam[0], P.cam[1], P.cam[2], P.cam[3], p[0], p[1], p[2]};
    pt = p[3];
    c0 = ((P.u_obs[0] * p[0]) + (P.u_obs[1] * p[1]) + (P.u_obs[2] * p[2])) + (P.u_obs[3] * p[3]);
}

// ----------------------------------------------------------- emitters
template <class T> __device__ __forceinline__ T redshift_clamp(T z) {
    if (isnan(z) || isinf(z)) z = T(1e-10);  // relativity_utilities.cuh:62-67
    return z;
}

// Circular Keplerian orbit at (x, 0, z), normalised in the integrated frame.
template <int METRIC, class T>
__device__ __forceinline__ V4<T> disk_velocity(T xh, T zh, T r, const DevScene<T>& P) {
    T omega = P.omega_sign / (r * sqrt(r) + P.spin_phys);
    T vx = zh * omega, vz = -xh * omega;
    Sym4<T> g = metric<METRIC>::template compute_g<T>(xh, T(0), zh, P.m);
    T n = g.tt + T(2) * (g.tx * vx + g.tz * vz) + g.xx * vx * vx + T(2) * g.xz * vx * vz + g.zz * vz * vz;
    T ut = T(1) / sqrt(-n);
    return V4<T>{vx * ut, T(0), vz * ut, ut};
}

// Planck's law in SI units, internal_math.h:2511-2526.
template <class T> __device__ __forceinline__ T planck(T wavelength_nm, T temperature) {
    if (temperature <= T(0)) return T(0);
    const T h = T(6.62607015E-34), c = T(299792458.0), kb = T(1.380649E-23);
    T wl = wavelength_nm * T(1e-9);
    T term_0 = h * c;
    T term_1 = T(2) * term_0 * c;
    T term_2 = wl * wl * wl * wl * wl;
    T term_3 = exp(term_0 / (wl * kb * temperature)) - T(1);
    return (term_1 / term_2) * (T(1) / term_3);
}

template <class T> __device__ __forceinline__ T clamp_radiance(T v) {
    return (isnan(v) || isinf(v) || v < T(0)) ? T(0) : v;  // bxdf_utilities.cuh:158-159
}

// The matter plugins (src/renderer/bxdf/matter.cuh) use these two, defined
// further down with the room and the star grid.
template <class T> __device__ __forceinline__ T white_led(T x);
MGK_HD uint32_t cube_cell(float dx, float dy, float dz, uint32_t n);

}  // namespace mgk

#include "../src/renderer/bxdf/matter.cuh"

namespace mgk {

// Termination record of a ray.
template <class T> struct Term {
    uint32_t cls;
    T z, r_hit, d0, d1, d2;
};

// ------------------------------------------------------------ crossings
// A disk or escape crossing between y0 and y1 is located on the geodesic:
// secant iterations on the crossing function, each evaluating a fresh RK
// sub-step of length s from y0 (explicit Euler for Minkowski), at most
// MGK_REFINE_ITERS + 1 sub-steps.  This removes the chord error of linear
// interpolation over a long step.  The escape sphere takes one sub-step, to
// where the step's chord meets the sphere (the root of a quadratic): in the
// far field the path departs from its chord by about one M over a step, so
// the sub-step ends within ~1e-3 M of the sphere, and the escape direction is
// taken at the escape radius itself (the remaining bending there changes by
// ~2 M b / r^3 = 4e-8 rad per M).  Interpolating |x|^2 linearly instead put
// the sub-step anywhere between ~0.85 R and R, which moved the measured
// direction by the far-field bending in between (~5e-6 rad) from one step
// sequence to another.
template <int METRIC, Fuse F, class T>
__device__ __forceinline__ S7<T> sub_step(const S7<T>& y0, T pt, T s, const MP<T>& m) {
    S7<T> y1;
    if constexpr (metric<METRIC>::explicit_euler) {
        S7<T> f;
        rhs<METRIC, F, T>(y0, pt, m, f);
        y1 = axpy<F>(s, f, y0);
    } else {
        S7<T> k[6];
        rkf45_stages<METRIC, F, T>(y0, pt, s, m, y1, k);
    }
    return y1;
}

template <class T> MGK_HD T axis_of(const S7<T>& q, int axis) { return axis == 0 ? q.x : (axis == 1 ? q.y : q.z); }
template <class T> MGK_HD T axis_of(const V4<T>& q, int axis) { return axis == 0 ? q.x : (axis == 1 ? q.y : q.z); }

// kind 0, 1, 2: the plane x, y or z = v; kind 3: the sphere |x|^2 = v.
template <Fuse F, class T> __device__ __forceinline__ T cross_g(int kind, const S7<T>& q, T v) {
    return kind == 3 ? mad<F>(q.z, q.z, mad<F>(q.y, q.y, q.x * q.x)) - v : axis_of(q, kind) - v;
}

// Chord parameter t in (0, 1] where the chord y0 -> y1 meets the sphere
// |x|^2 = |x0|^2 - g0 (g0 < 0: y0 inside): the positive root of
// qa t^2 + 2 qb t + g0 = 0, in the cancellation-free form for either sign of
// qb; `fallback` when the root is not in (0, 1].
template <Fuse F, class T>
__device__ __forceinline__ T chord_sphere(const S7<T>& y0, const S7<T>& y1, T g0, T fallback) {
    const T dx = y1.x - y0.x, dy = y1.y - y0.y, dz = y1.z - y0.z;
    const T qa = mad<F>(dz, dz, mad<F>(dy, dy, dx * dx));
    const T qb = mad<F>(y0.z, dz, mad<F>(y0.y, dy, y0.x * dx));
    const T disc = mad<F>(qb, qb, -(qa * g0));
    const T sq = sqrt(disc > T(0) ? disc : T(0));
    const T t = qb >= T(0) ? g0 / (-qb - sq) : (sq - qb) / qa;
    return (t > T(0) && t <= T(1)) ? t : fallback;
}

// Disk: kind 1, v = 0; escape sphere: kind 3, v = R^2; room faces: planes.
template <int METRIC, Fuse F, class T>
__device__ __forceinline__ S7<T> refine(int kind, const S7<T>& y0, const S7<T>& y1, T pt, T h, T v, const MP<T>& m,
                                        uint32_t& evals) {
    T g0 = cross_g<F>(kind, y0, v), g1 = cross_g<F>(kind, y1, v);
    T s_prev = h, g_prev = g1;
    T s = h * (g0 / (g0 - g1));
    if (kind == 3) s = h * chord_sphere<F>(y0, y1, g0, g0 / (g0 - g1));
    S7<T> ys = sub_step<METRIC, F, T>(y0, pt, s, m);
    ++evals;
    T gs = cross_g<F>(kind, ys, v);
    // The escape sphere lies in the far field, where one sub-step to the
    // chord's intersection ends within ~1e-3 M of it; planes (the disk in
    // strong field, the room's faces) iterate.
    const int iters = kind < 3 ? MGK_REFINE_ITERS : 0;
    for (int it = 0; it < iters; ++it) {
        T den = gs - g_prev;
        if (gs == T(0) || den == T(0)) break;
        T s_new = s - gs * (s - s_prev) / den;
        if (!(s_new > T(0) && s_new < h)) break;
        T ds = s_new - s;
        s_prev = s;
        g_prev = gs;
        s = s_new;
        ys = sub_step<METRIC, F, T>(y0, pt, s, m);
        ++evals;
        gs = cross_g<F>(kind, ys, v);
        if (fabs(ds) <= T(1e-6) * h) break;
    }
    return ys;
}

// Chord pre-test of the disk: the crossing radius estimated linearly lies
// within a 2 % margin of [r_in, r_out].
template <Fuse F, class T>
__device__ __forceinline__ bool disk_candidate(const DevScene<T>& P, const S7<T>& y0, const S7<T>& y1) {
    if (!P.disk_on) return false;
    T s0 = y0.y, s1 = y1.y;
    bool cross = (s0 > T(0)) ? (s1 <= T(0)) : ((s0 < T(0)) ? (s1 >= T(0)) : false);
    if (!cross) return false;
    T t = s0 / (s0 - s1);
    T xh = mad<F>(t, y1.x - y0.x, y0.x);
    T zh = mad<F>(t, y1.z - y0.z, y0.z);
    T a = P.kerr_a;
    T w = mad<F>(zh, zh, xh * xh) - a * a;
    T rc = sqrt(w > T(0) ? w : T(0));
    return rc >= P.disk_lo && rc <= P.disk_hi;
}

// ---------------------------------------------------------------- room
// The reference's test scene (matter_examples.cuh:33-77, kernel_intersect.cu:
// 81-100, traceables.cuh:17-74): the camera inside a box whose walls reflect
// (walls normal to x like mirrors, the others Lambertian) and a light box that
// absorbs and emits a white-LED spectrum.
//
// Cheap test after every step (integrator): the step ends outside the room,
// or its chord's bounding box overlaps the light.  Conservative; the crossing
// kernel runs the exact chord test.
template <class T>
__device__ __forceinline__ bool room_candidate(const DevScene<T>& P, const S7<T>& y0, const S7<T>& y1) {
    if (!P.room_on) return false;
    const bool inside = y1.x >= P.room_lo[0] && y1.x <= P.room_hi[0] && y1.y >= P.room_lo[1] &&
                        y1.y <= P.room_hi[1] && y1.z >= P.room_lo[2] && y1.z <= P.room_hi[2];
    const bool light = fmax(y0.x, y1.x) >= P.light_lo[0] && fmin(y0.x, y1.x) <= P.light_hi[0] &&
                       fmax(y0.y, y1.y) >= P.light_lo[1] && fmin(y0.y, y1.y) <= P.light_hi[1] &&
                       fmax(y0.z, y1.z) >= P.light_lo[2] && fmin(y0.z, y1.z) <= P.light_hi[2];
    return !inside || light;
}

// First room event on the chord a0 -> a1 (chord parameter t in [0, 1]):
// leaving the room through a wall (the face whose plane the chord crosses
// first among the axes on which a1 lies outside), or entering the light
// (slab test, traceables.cuh:17-74 with the chord as the segment).  axis < 0:
// none.  side 0 / 1: the face at the box's minimum / maximum on that axis.
template <class T> struct RoomEvent {
    T t;
    int axis, side;
    bool light;
};
template <class T>
MGK_HD RoomEvent<T> room_chord(const T* lo, const T* hi, const T* llo, const T* lhi, const T* a0, const T* a1) {
    RoomEvent<T> ev{T(2), -1, 0, false};
    for (int a = 0; a < 3; ++a) {
        const bool above = a1[a] > hi[a], below = a1[a] < lo[a];
        if (!(above || below)) continue;
        const T b = above ? hi[a] : lo[a];
        T t = (b - a0[a]) / (a1[a] - a0[a]);
        if (!(t >= T(0))) t = T(0);  // started outside on this axis
        if (t < ev.t) { ev.t = t; ev.axis = a; ev.side = above ? 1 : 0; }
    }
    T tn = T(0), tf = T(1);
    int an = -1, sn = 0;
    bool miss = false;
    // the chord's bounding box must overlap the light (the integrator's pre-test)
    for (int a = 0; a < 3; ++a)
        if (!(fmax(a0[a], a1[a]) >= llo[a] && fmin(a0[a], a1[a]) <= lhi[a])) miss = true;
    for (int a = 0; a < 3 && !miss; ++a) {
        const T d = a1[a] - a0[a];
        if (d == T(0)) {
            if (a0[a] < llo[a] || a0[a] > lhi[a]) miss = true;
            continue;
        }
        const T t_lo = (llo[a] - a0[a]) / d, t_hi = (lhi[a] - a0[a]) / d;
        const T t_near = d > T(0) ? t_lo : t_hi, t_far = d > T(0) ? t_hi : t_lo;
        if (t_near > tn) { tn = t_near; an = a; sn = d > T(0) ? 0 : 1; }
        if (t_far < tf) tf = t_far;
    }
    // an < 0: the chord starts inside the light (not an entry)
    if (!miss && an >= 0 && tn <= tf && tn < ev.t) {
        ev.t = tn; ev.axis = an; ev.side = sn; ev.light = true;
    }
    return ev;
}

// White-LED spectral radiance: five Gaussians s exp(-(x - o)^2 / (2 w^2))
// with the reference's centres, widths and weights (internal_math.h:
// 2441-2445, 2501-2509).
template <class T> __device__ __forceinline__ T white_led(T x) {
    const T o[5] = {T(577.0), T(451.0), T(455.0), T(528.0), T(690.0)};
    const T w[5] = {T(50.7937003968), T(7.07106781187), T(14.1421356237), T(13.7840487521), T(44.72135955)};
    const T s[5] = {T(157.0), T(200.0), T(50.0), T(20.0), T(10.0)};
    T acc = T(0);
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const T d = x - o[i];
        acc = acc + exp(T(-0.5) * ((d * d) / (w[i] * w[i]))) * s[i];
    }
    return acc;
}

// Uniform direction on the unit sphere from the ray's random numbers
// (dimensions base .. base + 32): cos(theta) = 1 - 2 u as in
// sample_lambertian_brdf (brdf.cuh:12-29), the azimuth's (cos, sin) from a
// point of the unit disc found by rejection (up to 16 tries; IEEE square
// root and division only, so host and device agree bit for bit).
template <class T> MGK_HD void sphere_dir(uint64_t seed, uint32_t sample, uint32_t pixel, uint32_t base, T out[3]) {
    const T cz = T(1) - T(2) * T(rng_unit(seed, sample, pixel, base));
    const T q = T(1) - cz * cz;
    const T sz = sqrt(q > T(0) ? q : T(0));
    T cx = T(1), cy = T(0);
    for (uint32_t j = 0; j < 16; ++j) {
        const T vx = T(2) * T(rng_unit(seed, sample, pixel, base + 1u + 2u * j)) - T(1);
        const T vy = T(2) * T(rng_unit(seed, sample, pixel, base + 2u + 2u * j)) - T(1);
        const T r2 = vx * vx + vy * vy;
        if (r2 <= T(1) && r2 > T(1e-12)) {
            const T r = sqrt(r2);
            cx = vx / r;
            cy = vy / r;
            break;
        }
    }
    out[0] = cx * sz; out[1] = cy * sz; out[2] = cz;
}

// Reflection off a wall at the located point X with covariant momentum p
// (apply_reflected, bxdf_utilities.cuh:53-109,139-154): the wall's observer
// is the reference observer (zero proper velocity, matter_examples.cuh:35-38);
// the ray's direction and the wall normal are taken to its rest frame
// (tetrad seeds x, y, z), the normal is turned to face the ray, the
// direction is mirrored (walls normal to x) or replaced by a cosine-weighted
// one around the normal (Lambertian: normalised uniform sphere direction plus
// normal), and mapped back to a null covariant momentum.  c0 becomes
// (u . p_out) times the redshift at the wall, so that redshifts multiply
// along the path.
template <int METRIC, class T>
__device__ __forceinline__ void reflect_wall(const DevScene<T>& P, int axis, int side, const S7<T>& X, T& pt, T& c0,
                                             uint32_t bounce, uint64_t ray_id, S7<T>& out) {
    const Sym4<T> g = metric<METRIC>::template compute_g<T>(X.x, X.y, X.z, P.m);
    const V4<T> u = metric<METRIC>::template reference_observer<T>(X.x, X.y, X.z, P.m);
    const Tetrad<T> e = build_tetrad<T>(g, V4<T>{T(1), T(0), T(0), T(0)}, V4<T>{T(0), T(1), T(0), T(0)},
                                        V4<T>{T(0), T(0), T(1), T(0)}, u);
    const V4<T> p{X.px, X.py, X.pz, pt};
    const T zr = redshift_clamp<T>(c0 / dot4(u, p));
    T d[3] = {dot4(e.x, p), dot4(e.y, p), dot4(e.z, p)};
    const T dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    d[0] = d[0] / dl; d[1] = d[1] / dl; d[2] = d[2] / dl;
    // facing normal in the global frame points into the room; its rest-frame
    // components are e_i^mu n_mu
    const T ns = side ? T(-1) : T(1);
    T n[3] = {axis_of(e.x, axis) * ns, axis_of(e.y, axis) * ns, axis_of(e.z, axis) * ns};
    const T nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] = n[0] / nl; n[1] = n[1] / nl; n[2] = n[2] / nl;
    if (n[0] * d[0] + n[1] * d[1] + n[2] * d[2] > T(0)) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
    T o[3];
    if (axis == 0) {
        const T k = T(2) * (d[0] * n[0] + d[1] * n[1] + d[2] * n[2]);
        o[0] = d[0] - k * n[0]; o[1] = d[1] - k * n[1]; o[2] = d[2] - k * n[2];
    } else {
        const uint32_t pixel = uint32_t(ray_id / P.spp), sample = uint32_t(ray_id % P.spp) + P.sample_offset;
        T q[3];
        sphere_dir<T>(P.seed, sample, pixel, 8u + 64u * bounce, q);
        o[0] = q[0] + n[0]; o[1] = q[1] + n[1]; o[2] = q[2] + n[2];
        if (!(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] > T(1e-12))) { o[0] = n[0]; o[1] = n[1]; o[2] = n[2]; }
    }
    const T ol = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    o[0] = o[0] / ol; o[1] = o[1] / ol; o[2] = o[2] / ol;
    const T l = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    const V4<T> pu = local_to_global<T>(e, V4<T>{o[0], o[1], o[2], l});
    const V4<T> po = contract<T>(g, pu);
    c0 = dot4(u, po) * zr;
    pt = po.t;
    // restart 1/256 inside the wall, on the face (offset_geodesic,
    // bxdf_utilities.cuh:111-137, with a fixed offset)
    T x[3] = {X.x, X.y, X.z};
    for (int a = 0; a < 3; ++a) x[a] = fmin(fmax(x[a], P.room_lo[a]), P.room_hi[a]);
    x[axis] = side ? P.room_hi[axis] - T(0.00390625) : P.room_lo[axis] + T(0.00390625);
    out = S7<T>{x[0], x[1], x[2], X.t, po.x, po.y, po.z};
}

template <Fuse F, class T> __device__ __forceinline__ T radius2(const S7<T>& y) {
    return mad<F>(y.z, y.z, mad<F>(y.y, y.y, y.x * y.x));
}

// Horizon and step-cap tests of a step without crossing candidates.
// r_KS >= sqrt(|x|^2 - a^2): positions far outside the capture radius skip
// the exact horizon test; NaN positions always take it.
template <int METRIC, Fuse F, class T>
__device__ __forceinline__ uint32_t plain_terminal(const DevScene<T>& P, const S7<T>& y1, T r2, uint32_t steps) {
    if constexpr (metric<METRIC>::has_horizon) {
        bool test = true;
        if constexpr (metric<METRIC>::ks_radius_bound) {
            T q = r2 - P.kerr_a * P.kerr_a;
            test = !(q > T(4) * P.m.horizon * P.m.horizon);
        }
        if (test && in_domain<METRIC, T>(y1.x, y1.y, y1.z, P.m)) return MGK_RAY_HORIZON;
    }
    if (steps >= P.max_steps) return MGK_RAY_STEP_LIMIT;
    return MGK_RAY_ALIVE;
}

// Ray state that a room reflection changes.
struct Bounce {
    uint32_t count;  // reflections so far
    uint64_t ray_id;  // global ray index (random numbers)
    bool reflected;  // set by resolve: the ray continues from y_end with the new pt, c0
};

// All tests after the accepted step y0 -> y1 of length h, in this order:
// thin disk (located crossing inside [r_in, r_out]) unless a room event comes
// first on the chord, room walls and light, escape radius, horizon, step cap.
// y_end receives the located crossing for disk, light and sky hits, and the
// restart state after a reflection (pt and c0 then change too).  ROOM =
// false compiles the room tests out (scenes without the room).
template <int METRIC, Fuse F, class T, bool ROOM>
__device__ __forceinline__ Term<T> resolve(const DevScene<T>& P, const S7<T>& y0, const S7<T>& y1, T& pt, T h,
                                           T& c0, uint32_t steps, Bounce& bn, S7<T>& y_end, uint32_t& evals) {
    Term<T> o{MGK_RAY_ALIVE, T(0), T(0), T(0), T(0), T(0)};
    y_end = y1;
    bn.reflected = false;
    RoomEvent<T> ev{T(2), -1, 0, false};
    if constexpr (ROOM) {
        const T a0[3] = {y0.x, y0.y, y0.z}, a1[3] = {y1.x, y1.y, y1.z};
        ev = room_chord<T>(P.room_lo, P.room_hi, P.light_lo, P.light_hi, a0, a1);
    }
    if (disk_candidate<F, T>(P, y0, y1) && !(ROOM && ev.axis >= 0 && ev.t < y0.y / (y0.y - y1.y))) {
        S7<T> ys = refine<METRIC, F, T>(1, y0, y1, pt, h, T(0), P.m, evals);
        T rh = kerr_schild_r(ys.x, ys.y, ys.z, P.kerr_a);
        if (rh >= P.disk_r_in && rh <= P.disk_r_out) {
            V4<T> u = matter<MGK_RAY_DISK>::template four_velocity<METRIC, T>(P, ys.x, ys.y, ys.z, rh);
            o.cls = MGK_RAY_DISK;
            o.z = redshift_clamp<T>(c0 / dot4(u, V4<T>{ys.px, ys.py, ys.pz, pt}));
            o.r_hit = rh;
            y_end = ys;
            return o;
        }
    }
    if (ROOM && ev.axis >= 0) {
        const T* face = ev.light ? (ev.side ? P.light_hi : P.light_lo) : (ev.side ? P.room_hi : P.room_lo);
        const S7<T> ys = ev.t > T(0) ? refine<METRIC, F, T>(ev.axis, y0, y1, pt, h, face[ev.axis], P.m, evals) : y0;
        y_end = ys;
        if (ev.light) {
            // absorbed: the light's spectrum at the redshift seen by its (static) observer
            const V4<T> u = matter<MGK_RAY_LIGHT>::template four_velocity<METRIC, T>(P, ys.x, ys.y, ys.z, T(0));
            o.cls = MGK_RAY_LIGHT;
            o.z = redshift_clamp<T>(c0 / dot4(u, V4<T>{ys.px, ys.py, ys.pz, pt}));
            return o;
        }
        if (bn.count >= P.room_limit) {
            // one reflection more than the limit ends the ray
            // (kernel_enforce_ray_limits.cu:49)
            bn.count += 1u;
            o.cls = MGK_RAY_STEP_LIMIT;
            return o;
        }
        reflect_wall<METRIC, T>(P, ev.axis, ev.side, ys, pt, c0, bn.count, bn.ray_id, y_end);
        bn.count += 1u;
        bn.reflected = true;
        if (steps >= P.max_steps) o.cls = MGK_RAY_STEP_LIMIT;
        return o;
    }
    T r2 = radius2<F>(y1);
    if (r2 >= P.escape_r2) {
        S7<T> ys = refine<METRIC, F, T>(3, y0, y1, pt, h, P.escape_r2, P.m, evals);
        T pn = sqrt(mad<F>(ys.pz, ys.pz, mad<F>(ys.py, ys.py, ys.px * ys.px)));
        o.cls = MGK_RAY_ESCAPED;
        o.d0 = ys.px / pn; o.d1 = ys.py / pn; o.d2 = ys.pz / pn;
        static_assert(matter<MGK_RAY_ESCAPED>::at_infinity, "the sky is static at infinity");
        o.z = redshift_clamp<T>(c0 / pt);  // u . p = p_t
        y_end = ys;
        return o;
    }
    o.cls = plain_terminal<METRIC, F, T>(P, y1, r2, steps);
    return o;
}

// -------------------------------------------------------------- stars
// Cube-map grid over the celestial sphere: face (largest |component|), then
// N x N cells; each cell lists the stars whose disc reaches into it, in
// ascending star index.
struct StarGrid {
    const uint32_t* cell_start;  // 6*N*N + 1
    const uint32_t* cell_stars;
    uint32_t n;
};

MGK_HD uint32_t cube_cell(float dx, float dy, float dz, uint32_t n) {
    float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    uint32_t face;
    float u, v, m;
    if (ax >= ay && ax >= az) { face = dx >= 0.f ? 0u : 1u; m = ax; u = dy; v = dz; }
    else if (ay >= az) { face = dy >= 0.f ? 2u : 3u; m = ay; u = dx; v = dz; }
    else { face = dz >= 0.f ? 4u : 5u; m = az; u = dx; v = dy; }
    float fu = (u / m + 1.0f) * 0.5f * float(n), fv = (v / m + 1.0f) * 0.5f * float(n);
    int iu = int(fu), iv = int(fv);
    iu = iu < 0 ? 0 : (iu >= int(n) ? int(n) - 1 : iu);
    iv = iv < 0 ? 0 : (iv >= int(n) ? int(n) - 1 : iv);
    return (face * n + uint32_t(iv)) * n + uint32_t(iu);
}

}  // namespace mgk
