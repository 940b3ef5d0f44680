// CPU oracle, part 2: the rendered scene around the integrator (TEST
// INFRASTRUCTURE ONLY).
//
//  * counter-based RNG (the reference's triplet_hash, internal_math.h:2027-2037)
//  * pinhole camera with seeded jitter; observer = the metric's reference
//    observer (kernel_generate_initial_conditions.cu:54-74,
//    relativity_utilities.cuh:163-195)
//  * per accepted step: thin-disk crossing, room walls and light, escape
//    radius, horizon (kernel_intersect.cu:55-138 order: traceables before the
//    horizon), step cap and reflection cap (kernel_enforce_ray_limits.cu:37-64)
//  * wall reflection in the wall's rest frame, mirror on walls normal to x,
//    Lambertian elsewhere (matter_examples.cuh:33-58, bxdf_utilities.cuh:53-154)
//  * Keplerian disk emitter, redshift (bxdf_utilities.cuh:89-109,156-163),
//    blackbody (internal_math.h:2511-2526) at N wavelengths, star field,
//    white-LED light (matter_examples.cuh:60-77, internal_math.h:2441-2509)
//  * spectral -> XYZ with per-bin CMF weights (device_color_utilities.cuh:40-54)
//
// The "mixed" precision mode (FP32 state and step control, FP64 attempts
// within 0.05 M of the outer horizon) is defined here exactly as the CUDA
// kernels implement it, so that the two can be compared bit for bit.
#pragma once

#include <algorithm>
#include <type_traits>
#include <vector>

#include "oracle.hpp"
#include "../include/mgk.h"

namespace orc {

// ------------------------------------------------------------------ RNG
// triplet_hash, internal_math.h:2027-2037.
inline uint32_t triplet_hash(uint32_t x) {
    x ^= x >> 17; x *= 0xED5AD4BBu; x ^= x >> 11; x *= 0xAC4C1B51u;
    x ^= x >> 15; x *= 0x31848BABu; x ^= x >> 14;
    return x;
}
inline uint32_t rng_u32(uint64_t seed, uint32_t stream, uint32_t index, uint32_t dim) {
    uint32_t h = triplet_hash(uint32_t(seed) ^ 0x9E3779B9u);
    h = triplet_hash(h ^ uint32_t(seed >> 32));
    h = triplet_hash(h ^ stream);
    h = triplet_hash(h ^ index);
    h = triplet_hash(h ^ (dim * 0x85EBCA6Bu + 1u));
    return h;
}
inline float rng_unit(uint64_t seed, uint32_t stream, uint32_t index, uint32_t dim) {
    return float(rng_u32(seed, stream, index, dim) >> 8) * (1.0f / 16777216.0f);
}

// -------------------------------------------------------------- scene setup
// Host-side constants derived once per scene, in double, then rounded to the
// kernel's scalar type.  The library computes the same table (mgk_scene_setup).
struct SceneConsts {
    double cam_pos[4];     // (x, y, z, t)
    double u_obs[4];       // observer four-velocity (contravariant)
    double M[4][4];        // p_mu = M . (n_x, n_y, n_z, |n|): g * [e_x e_y e_z e_t]
    double pix_a, pix_b;   // camera x = (px + jx) * pix_a + pix_b
    double pix_c, pix_d;   // camera y = (py + jy) * pix_c + pix_d
    double r_plus;         // outer horizon radius (M = 1)
    double spin_t;         // spin as integrated (sign-flipped when time reversed)
    double omega_sign;     // +1 / -1: sense of the disk's orbit in the integrated frame
};

inline MetricParams<double> metric_params_d(const mgk_scene& s) {
    MetricParams<double> m{};
    m.metric = s.metric;
    m.time_reversed = s.time_reversed != 0;
    m.spin = s.time_reversed ? -s.spin : s.spin;
    m.mass_sign = s.mass_sign < 0 ? -1.0 : 1.0;
    m.horizon_scalar = s.horizon_scalar;
    m.h_max = s.h_max;
    m.abs_tol = s.abs_tol;
    m.rel_tol = s.rel_tol;
    m.n_max = s.n_max_substep;
    return m;
}
template <class T> inline MetricParams<T> metric_params(const mgk_scene& s) {
    MetricParams<double> d = metric_params_d(s);
    MetricParams<T> m{};
    m.metric = d.metric; m.time_reversed = d.time_reversed;
    m.spin = T(d.spin); m.mass_sign = T(d.mass_sign); m.horizon_scalar = T(d.horizon_scalar);
    m.h_max = T(d.h_max); m.abs_tol = T(d.abs_tol); m.rel_tol = T(d.rel_tol); m.n_max = d.n_max;
    return m;
}

inline SceneConsts scene_consts(const mgk_scene& s) {
    SceneConsts c{};
    MetricParams<double> m = metric_params_d(s);
    double ci = std::cos(s.cam_incl_rad), si = std::sin(s.cam_incl_rad);
    V4<double> q{0.0, s.cam_r * ci, s.cam_r * si, 0.0};
    // orbit camera basis: right = +x, up = (0, sin i, -cos i), back = (0, cos i, sin i)
    V4<double> X{1, 0, 0, 0}, Y{0, si, -ci, 0}, Z{0, ci, si, 0};
    if (s.cam_explicit) {  // position and orientation columns as given
        q = V4<double>{s.cam_pos[0], s.cam_pos[1], s.cam_pos[2], 0.0};
        X = V4<double>{s.cam_axes[0], s.cam_axes[1], s.cam_axes[2], 0.0};
        Y = V4<double>{s.cam_axes[3], s.cam_axes[4], s.cam_axes[5], 0.0};
        Z = V4<double>{s.cam_axes[6], s.cam_axes[7], s.cam_axes[8], 0.0};
    }
    c.cam_pos[0] = q.x; c.cam_pos[1] = q.y; c.cam_pos[2] = q.z; c.cam_pos[3] = q.t;
    V4<double> u = reference_observer(q, m);
    Sym4<double> g = compute_g(q, m);
    const double* v = s.cam_velocity;
    if (s.cam_explicit && (v[0] != 0.0 || v[1] != 0.0 || v[2] != 0.0)) {
        // a moving observer: rest_frame_four_velocity, relativity_utilities.cuh:163-173
        Tetrad<double> e0 = build_tetrad(g, V4<double>{1, 0, 0, 0}, V4<double>{0, 1, 0, 0}, V4<double>{0, 0, 1, 0}, u);
        const double f = s.time_reversed ? -1.0 : 1.0;
        const double wx = f * v[0], wy = f * v[1], wz = f * v[2];
        u = local_to_global(e0, V4<double>{wx, wy, wz, std::sqrt(wx * wx + wy * wy + wz * wz + 1.0)});
    }
    Tetrad<double> e = build_tetrad(g, X, Y, Z, u);
    V4<double> cols[4] = {contract(g, e.x), contract(g, e.y), contract(g, e.z), contract(g, e.t)};
    for (int j = 0; j < 4; ++j) {
        c.M[0][j] = cols[j].x; c.M[1][j] = cols[j].y; c.M[2][j] = cols[j].z; c.M[3][j] = cols[j].t;
    }
    c.u_obs[0] = u.x; c.u_obs[1] = u.y; c.u_obs[2] = u.z; c.u_obs[3] = u.t;
    double tan_half = s.sensor_diag_mm / (2.0 * s.focal_length_mm);  // thin_lens.cuh:60-76 geometry
    double W = s.width, H = s.height;
    c.pix_a = 2.0 * tan_half / W;
    c.pix_b = -tan_half;
    c.pix_c = -2.0 * tan_half / W;
    c.pix_d = tan_half * H / W;
    double a = s.metric == KERR ? s.spin : 0.0;
    c.r_plus = s.metric == MINKOWSKI ? 0.0 : 1.0 + std::sqrt(std::max(0.0, 1.0 - a * a));
    c.spin_t = m.spin;
    c.omega_sign = s.time_reversed ? -1.0 : 1.0;
    return c;
}

// ------------------------------------------------------------ camera rays
template <class T> struct RayInit { GState<T> y; T c0; T h0; };

template <Fuse F, class T>
inline RayInit<T> camera_ray(const mgk_scene& s, const SceneConsts& c, uint64_t ray_id) {
    uint32_t spp = s.spp;
    uint32_t pixel = uint32_t(ray_id / spp), sample = uint32_t(ray_id % spp) + s.sample_offset;
    uint32_t px = pixel % s.width, py = pixel / s.width;
    T jx = T(rng_unit(s.seed, sample, pixel, 0));
    T jy = T(rng_unit(s.seed, sample, pixel, 1));
    T sx = mad<F>(T(px) + jx, T(c.pix_a), T(c.pix_b));
    T sy = mad<F>(T(py) + jy, T(c.pix_c), T(c.pix_d));
    T len = sq_root(mad<F>(sy, sy, mad<F>(sx, sx, T(1))));
    T nx = sx / len, ny = sy / len, nz = T(-1) / len;
    T nl = sq_root(mad<F>(nz, nz, mad<F>(ny, ny, nx * nx)));
    T v[4] = {nx, ny, nz, nl};
    T p[4];
    for (int i = 0; i < 4; ++i) {
        T acc = T(c.M[i][0]) * v[0];
        acc = mad<F>(T(c.M[i][1]), v[1], acc);
        acc = mad<F>(T(c.M[i][2]), v[2], acc);
        acc = mad<F>(T(c.M[i][3]), v[3], acc);
        p[i] = acc;
    }
    RayInit<T> r;
    r.y.x = V4<T>{T(c.cam_pos[0]), T(c.cam_pos[1]), T(c.cam_pos[2]), T(c.cam_pos[3])};
    r.y.p = V4<T>{p[0], p[1], p[2], p[3]};
    V4<T> u{T(c.u_obs[0]), T(c.u_obs[1]), T(c.u_obs[2]), T(c.u_obs[3])};
    r.c0 = dot4(u, r.y.p);
    r.h0 = s.metric == MINKOWSKI ? T(1000) : T(1);  // initial_h_step, metric_*.cuh
    return r;
}

// ----------------------------------------------------------- emitters
// Redshift factor with the reference's NaN/Inf clamp (relativity_utilities.cuh:62-67).
template <class T> inline T redshift_clamp(T z) {
    if (std::isnan(z) || std::isinf(z)) z = T(1e-10);
    return z;
}

// Four-velocity of a circular Keplerian orbit at (x, 0, z) in the integrated
// Kerr-Schild frame, normalised with that frame's metric.
template <class T> inline V4<T> disk_velocity(T xh, T zh, T r, const MetricParams<T>& m, T spin_phys, T omega_sign) {
    T omega = omega_sign / (r * sq_root(r) + spin_phys);
    T vx = zh * omega, vz = -xh * omega;
    Sym4<T> g = compute_g(V4<T>{xh, T(0), zh, T(0)}, m);
    T n = g.tt + T(2) * (g.tx * vx + g.tz * vz) + g.xx * vx * vx + T(2) * g.xz * vx * vz + g.zz * vz * vz;
    T ut = T(1) / sq_root(-n);
    return V4<T>{vx * ut, T(0), vz * ut, ut};
}

// Planck's law B_lambda(lambda, T) in SI units, internal_math.h:2511-2526.
template <class T> inline T planck(T wavelength_nm, T temperature) {
    if (temperature <= T(0)) return T(0);
    const T h = T(6.62607015E-34), c = T(299792458.0), kb = T(1.380649E-23);
    T wl = wavelength_nm * T(1e-9);
    T term_0 = h * c;
    T term_1 = T(2) * term_0 * c;
    T term_2 = wl * wl * wl * wl * wl;
    T term_3 = std::exp(term_0 / (wl * kb * temperature)) - T(1);
    return (term_1 / term_2) * (T(1) / term_3);
}

// --------------------------------------------------------------- tracing
struct RayResult {
    double x[4], p[4];
    double z;         // redshift factor (disk or sky), 0 otherwise
    double r_hit;     // disk hit radius
    double dir[3];    // escape direction (normalised covariant spatial momentum)
    uint32_t cls;     // mgk_ray_class
    uint32_t steps;   // accepted steps
    uint32_t attempts;
    uint32_t wide_attempts;
    uint32_t refine_evals;  // RK sub-steps spent locating a crossing
    uint32_t bounces;       // reflections off the room's walls
};

// ------------------------------------------------------------ crossings
// A disk or escape crossing found between y0 and y1 is located on the
// geodesic itself: secant iterations on the crossing function g, each
// evaluating a fresh RK sub-step of length s from y0 (the 5th-order stage
// solution; explicit Euler for Minkowski), at most MGK_REFINE_ITERS + 1
// sub-steps.  This removes the chord error that linear interpolation of a
// long step leaves, so the hit no longer depends on the step sequence.
template <Fuse F, class T> inline GState<T> sub_step(const GState<T>& y0, T s, const MetricParams<T>& m) {
    if (m.metric == MINKOWSKI) return axpy<F>(s, rhs_minkowski<T>(y0), y0);
    GState<T> y1, k[6];
    rkf45_attempt<F, T>(y0, s, m, &y1, k);
    return y1;
}

template <class T> inline T coord(const V4<T>& q, int axis) { return axis == 0 ? q.x : (axis == 1 ? q.y : q.z); }

// kind 0, 1, 2: the plane x, y or z = v (disk: y = 0; room faces);
// kind 3: the escape sphere |x|^2 = v.
template <Fuse F, class T>
inline GState<T> refine(int kind, const GState<T>& y0, const GState<T>& y1, T h, T v, const MetricParams<T>& m,
                        uint32_t* evals) {
    auto g = [&](const GState<T>& q) {
        return kind == 3 ? mad<F>(q.x.z, q.x.z, mad<F>(q.x.y, q.x.y, q.x.x * q.x.x)) - v : coord(q.x, kind) - v;
    };
    T g0 = g(y0), g1 = g(y1);
    T s_prev = h, g_prev = g1;
    T s = h * (g0 / (g0 - g1));
    if (kind == 3) {
        // the escape sphere: one sub-step to where the chord meets it (the
        // positive root of qa t^2 + 2 qb t + g0 = 0), as the kernels do
        const T dx = y1.x.x - y0.x.x, dy = y1.x.y - y0.x.y, dz = y1.x.z - y0.x.z;
        const T qa = mad<F>(dz, dz, mad<F>(dy, dy, dx * dx));
        const T qb = mad<F>(y0.x.z, dz, mad<F>(y0.x.y, dy, y0.x.x * dx));
        const T disc = mad<F>(qb, qb, -(qa * g0));
        const T sq = sq_root(disc > T(0) ? disc : T(0));
        const T t = qb >= T(0) ? g0 / (-qb - sq) : (sq - qb) / qa;
        s = h * ((t > T(0) && t <= T(1)) ? t : g0 / (g0 - g1));
    }
    GState<T> ys = sub_step<F>(y0, s, m);
    ++*evals;
    T gs = g(ys);
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
        ys = sub_step<F>(y0, s, m);
        ++*evals;
        gs = g(ys);
        if (fabs_(ds) <= T(1e-6) * h) break;
    }
    return ys;
}

template <class T> struct Hit {
    uint32_t cls = MGK_RAY_ALIVE;
    T z = 0, r_hit = 0, dir[3] = {0, 0, 0};
};

template <class T> struct Resolved {
    Hit<T> hit;
    GState<T> y_end;  // the refined state for disk and sky hits, else y1
    uint32_t evals = 0;
};

// Disk pre-test on the chord: the crossing radius, estimated linearly, lies
// within a 2 % margin of [r_in, r_out].
template <Fuse F, class T>
inline bool disk_candidate(const mgk_scene& s, const MetricParams<T>& m, const GState<T>& y0, const GState<T>& y1) {
    if (!(s.disk_r_out > 0.0)) return false;
    T s0 = y0.x.y, s1 = y1.x.y;
    bool cross = (s0 > T(0)) ? (s1 <= T(0)) : ((s0 < T(0)) ? (s1 >= T(0)) : false);
    if (!cross) return false;
    T t = s0 / (s0 - s1);
    T xh = mad<F>(t, y1.x.x - y0.x.x, y0.x.x);
    T zh = mad<F>(t, y1.x.z - y0.x.z, y0.x.z);
    T a = m.metric == KERR ? m.spin : T(0);
    T w = mad<F>(zh, zh, xh * xh) - a * a;
    T rc = sq_root(w > T(0) ? w : T(0));
    return rc >= T(0.98 * s.disk_r_in - 0.02) && rc <= T(1.02 * s.disk_r_out + 0.02);
}

// ------------------------------------------------------------------ room
// The reference's box-and-light scene (stage.h:19-22, matter_examples.cuh:
// 33-77, kernel_intersect.cu:81-100).  First event on the chord a0 -> a1:
// leaving the room (the face crossed first among the axes on which a1 lies
// outside) or entering the light (slab test as traceables.cuh:17-74, on the
// chord segment).  axis < 0: none; side 0 / 1: face at the minimum / maximum.
template <class T> struct RoomEvent {
    T t = T(2);
    int axis = -1, side = 0;
    bool light = false;
};
template <class T> inline RoomEvent<T> room_event(const mgk_scene& s, const V4<T>& p0, const V4<T>& p1) {
    RoomEvent<T> ev;
    if (!s.room_on) return ev;
    const T a0[3] = {p0.x, p0.y, p0.z}, a1[3] = {p1.x, p1.y, p1.z};
    for (int a = 0; a < 3; ++a) {
        const T lo = T(s.room_min[a]), hi = T(s.room_max[a]);
        const bool above = a1[a] > hi, below = a1[a] < lo;
        if (!(above || below)) continue;
        const T b = above ? hi : lo;
        T t = (b - a0[a]) / (a1[a] - a0[a]);
        if (!(t >= T(0))) t = T(0);
        if (t < ev.t) { ev.t = t; ev.axis = a; ev.side = above ? 1 : 0; }
    }
    T tn = T(0), tf = T(1);
    int an = -1, sn = 0;
    bool miss = false;
    for (int a = 0; a < 3; ++a)  // chord bounding box overlaps the light
        if (!(std::fmax(a0[a], a1[a]) >= T(s.light_min[a]) && std::fmin(a0[a], a1[a]) <= T(s.light_max[a])))
            miss = true;
    for (int a = 0; a < 3 && !miss; ++a) {
        const T llo = T(s.light_min[a]), lhi = T(s.light_max[a]);
        const T d = a1[a] - a0[a];
        if (d == T(0)) {
            if (a0[a] < llo || a0[a] > lhi) miss = true;
            continue;
        }
        const T t_lo = (llo - a0[a]) / d, t_hi = (lhi - a0[a]) / d;
        const T t_near = d > T(0) ? t_lo : t_hi, t_far = d > T(0) ? t_hi : t_lo;
        if (t_near > tn) { tn = t_near; an = a; sn = d > T(0) ? 0 : 1; }
        if (t_far < tf) tf = t_far;
    }
    if (!miss && an >= 0 && tn <= tf && tn < ev.t) {
        ev.t = tn; ev.axis = an; ev.side = sn; ev.light = true;
    }
    return ev;
}

// evaluate_white_led_spectrum, internal_math.h:2501-2509, with
// gaussian_distribution (internal_math.h:2441-2445).
template <class T> inline T white_led(T x) {
    auto gauss = [](T v, T o, T w, T sc) { return T(std::exp(T(-0.5) * (((v - o) * (v - o)) / (w * w)))) * sc; };
    T acc = T(0);
    acc = acc + gauss(x, T(577.0), T(50.7937003968), T(157.0));
    acc = acc + gauss(x, T(451.0), T(7.07106781187), T(200.0));
    acc = acc + gauss(x, T(455.0), T(14.1421356237), T(50.0));
    acc = acc + gauss(x, T(528.0), T(13.7840487521), T(20.0));
    acc = acc + gauss(x, T(690.0), T(44.72135955), T(10.0));
    return acc;
}

// Uniform unit-sphere direction (the distribution of sample_lambertian_brdf's
// p, brdf.cuh:18-25): cos(theta) = 1 - 2 u, azimuth from a rejection-sampled
// point of the unit disc, from the ray's random dimensions base .. base + 32.
template <class T> inline void sphere_dir(uint64_t seed, uint32_t sample, uint32_t pixel, uint32_t base, T out[3]) {
    const T cz = T(1) - T(2) * T(rng_unit(seed, sample, pixel, base));
    const T q = T(1) - cz * cz;
    const T sz = sq_root(q > T(0) ? q : T(0));
    T cx = T(1), cy = T(0);
    for (uint32_t j = 0; j < 16; ++j) {
        const T vx = T(2) * T(rng_unit(seed, sample, pixel, base + 1u + 2u * j)) - T(1);
        const T vy = T(2) * T(rng_unit(seed, sample, pixel, base + 2u + 2u * j)) - T(1);
        const T r2 = vx * vx + vy * vy;
        if (r2 <= T(1) && r2 > T(1e-12)) {
            const T r = sq_root(r2);
            cx = vx / r;
            cy = vy / r;
            break;
        }
    }
    out[0] = cx * sz; out[1] = cy * sz; out[2] = cz;
}

// Reflection at the located wall point ys (apply_reflected and its context,
// bxdf_utilities.cuh:53-109,139-154): rest frame of the reference observer,
// facing normal, mirror (walls normal to x) or normalised(uniform sphere
// direction + normal), back to a null covariant momentum; c0 takes the
// redshift at the wall along; the ray restarts 1/256 inside the face.
template <class T>
inline GState<T> reflect_wall(const mgk_scene& s, const MetricParams<T>& m, int axis, int side, const GState<T>& ys,
                              T* c0, uint32_t bounce, uint64_t ray_id) {
    const Sym4<T> g = compute_g(ys.x, m);
    const V4<T> u = reference_observer(ys.x, m);
    const Tetrad<T> e = build_tetrad(g, V4<T>{T(1), T(0), T(0), T(0)}, V4<T>{T(0), T(1), T(0), T(0)},
                                     V4<T>{T(0), T(0), T(1), T(0)}, u);
    const V4<T>& p = ys.p;
    const T zr = redshift_clamp<T>(*c0 / dot4(u, p));
    T d[3] = {dot4(e.x, p), dot4(e.y, p), dot4(e.z, p)};
    const T dl = sq_root(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (T& v : d) v = v / dl;
    const T ns = side ? T(-1) : T(1);
    T n[3] = {coord(e.x, axis) * ns, coord(e.y, axis) * ns, coord(e.z, axis) * ns};
    const T nl = sq_root(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (T& v : n) v = v / nl;
    if (n[0] * d[0] + n[1] * d[1] + n[2] * d[2] > T(0))
        for (T& v : n) v = -v;
    T o[3];
    if (axis == 0) {
        const T k = T(2) * (d[0] * n[0] + d[1] * n[1] + d[2] * n[2]);
        for (int i = 0; i < 3; ++i) o[i] = d[i] - k * n[i];
    } else {
        T q[3];
        sphere_dir<T>(s.seed, uint32_t(ray_id % s.spp) + s.sample_offset, uint32_t(ray_id / s.spp), 8u + 64u * bounce, q);
        for (int i = 0; i < 3; ++i) o[i] = q[i] + n[i];
        if (!(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] > T(1e-12)))
            for (int i = 0; i < 3; ++i) o[i] = n[i];
    }
    const T ol = sq_root(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    for (T& v : o) v = v / ol;
    const T l = sq_root(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    const V4<T> po = contract(g, local_to_global(e, V4<T>{o[0], o[1], o[2], l}));
    *c0 = dot4(u, po) * zr;
    T x[3] = {ys.x.x, ys.x.y, ys.x.z};
    for (int a = 0; a < 3; ++a) x[a] = std::fmin(std::fmax(x[a], T(s.room_min[a])), T(s.room_max[a]));
    x[axis] = side ? T(s.room_max[axis]) - T(0.00390625) : T(s.room_min[axis]) + T(0.00390625);
    GState<T> out;
    out.x = V4<T>{x[0], x[1], x[2], ys.x.t};
    out.p = po;
    return out;
}

struct Bounce {
    uint32_t count = 0;
    uint64_t ray_id = 0;
    bool reflected = false;
};

// Tests after the accepted step y0 -> y1 of length h, in this order: thin
// disk (unless a room event comes first on the chord), room walls and light,
// escape radius, horizon, step cap.  A wall reflection leaves the ray alive
// with y_end its restart state and *c0 updated.
template <Fuse F, class T>
inline Resolved<T> resolve(const mgk_scene& s, const MetricParams<T>& m, const GState<T>& y0, const GState<T>& y1,
                           T h, T* c0, uint32_t steps, T spin_phys, T omega_sign, Bounce* bn) {
    Resolved<T> o;
    o.y_end = y1;
    bn->reflected = false;
    T a = m.metric == KERR ? m.spin : T(0);
    const RoomEvent<T> ev = room_event<T>(s, y0.x, y1.x);
    if (disk_candidate<F, T>(s, m, y0, y1) && !(ev.axis >= 0 && ev.t < y0.x.y / (y0.x.y - y1.x.y))) {
        GState<T> ys = refine<F, T>(1, y0, y1, h, T(0), m, &o.evals);
        T rh = kerr_schild_r(ys.x.x, ys.x.y, ys.x.z, a);
        if (rh >= T(s.disk_r_in) && rh <= T(s.disk_r_out)) {
            V4<T> u = disk_velocity<T>(ys.x.x, ys.x.z, rh, m, spin_phys, omega_sign);
            o.hit.cls = MGK_RAY_DISK;
            o.hit.z = redshift_clamp<T>(*c0 / dot4(u, ys.p));
            o.hit.r_hit = rh;
            o.y_end = ys;
            return o;
        }
    }
    if (ev.axis >= 0) {
        const double* face = ev.light ? (ev.side ? s.light_max : s.light_min) : (ev.side ? s.room_max : s.room_min);
        const GState<T> ys = ev.t > T(0) ? refine<F, T>(ev.axis, y0, y1, h, T(face[ev.axis]), m, &o.evals) : y0;
        o.y_end = ys;
        if (ev.light) {
            o.hit.cls = MGK_RAY_LIGHT;
            o.hit.z = redshift_clamp<T>(*c0 / dot4(reference_observer(ys.x, m), ys.p));
            return o;
        }
        if (bn->count >= s.room_reflection_limit) {
            bn->count += 1;
            o.hit.cls = MGK_RAY_STEP_LIMIT;
            return o;
        }
        o.y_end = reflect_wall<T>(s, m, ev.axis, ev.side, ys, c0, bn->count, bn->ray_id);
        bn->count += 1;
        bn->reflected = true;
        if (steps >= s.max_steps) o.hit.cls = MGK_RAY_STEP_LIMIT;
        return o;
    }
    T R2 = T(s.escape_radius) * T(s.escape_radius);
    T r2 = mad<F>(y1.x.z, y1.x.z, mad<F>(y1.x.y, y1.x.y, y1.x.x * y1.x.x));
    if (r2 >= R2) {
        GState<T> ys = refine<F, T>(3, y0, y1, h, R2, m, &o.evals);
        T pn = sq_root(mad<F>(ys.p.z, ys.p.z, mad<F>(ys.p.y, ys.p.y, ys.p.x * ys.p.x)));
        o.hit.cls = MGK_RAY_ESCAPED;
        o.hit.dir[0] = ys.p.x / pn; o.hit.dir[1] = ys.p.y / pn; o.hit.dir[2] = ys.p.z / pn;
        o.hit.z = redshift_clamp<T>(*c0 / ys.p.t);  // static emitter at infinity: u . p = p_t
        o.y_end = ys;
        return o;
    }
    if (in_domain(y1.x, m)) { o.hit.cls = MGK_RAY_HORIZON; return o; }
    if (steps >= s.max_steps) { o.hit.cls = MGK_RAY_STEP_LIMIT; return o; }
    return o;
}

// One attempt of the mixed mode: FP32 stages and state, FP64 error control;
// the whole attempt in FP64 when the current position lies within
// MGK_WIDE_BAND of the outer horizon.  Returns the accepted flag.
struct MixedAttempt {
    GState<float> y1;
    float h_next;
    bool accept_ok;  // error < 1
    bool wide;
};
inline MixedAttempt mixed_attempt(const GState<float>& y0, float h, const MetricParams<float>& mf,
                                  const MetricParams<double>& md, double r_cur, double r_plus) {
    MixedAttempt o{};
    bool wide = (mf.metric != MINKOWSKI) && (r_cur - r_plus < MGK_WIDE_BAND);
    o.wide = wide;
    if (wide) {
        GState<double> yd = to_double(y0), y1d;
        GState<double> k[6];
        rkf45_attempt<Fuse::Fma, double>(yd, double(h), md, &y1d, k);
        double hn;
        control_f64(yd, y1d, k, double(h), md, &hn, &o.accept_ok);
        o.h_next = float(hn);
        o.y1 = widen<float>(y1d);
    } else {
        GState<float> k[6];
        rkf45_attempt<Fuse::Fma, float>(y0, h, mf, &o.y1, k);
        control_mixed(y0, o.y1, k, h, mf, &o.h_next, &o.accept_ok);
    }
    return o;
}

// Outer KS radius of a position (used for the FP64 band test).
template <class T> inline double ks_radius(const V4<T>& q, const MetricParams<double>& md) {
    double a = md.metric == KERR ? md.spin : 0.0;
    return kerr_schild_r(double(q.x), double(q.y), double(q.z), a);
}

template <class T> inline void store_result(RayResult* r, const GState<T>& y, const Hit<T>& h, uint32_t steps,
                                            uint32_t attempts, uint32_t wide, uint32_t evals, uint32_t bounces) {
    r->x[0] = y.x.x; r->x[1] = y.x.y; r->x[2] = y.x.z; r->x[3] = y.x.t;
    r->p[0] = y.p.x; r->p[1] = y.p.y; r->p[2] = y.p.z; r->p[3] = y.p.t;
    r->z = h.z; r->r_hit = h.r_hit;
    r->dir[0] = h.dir[0]; r->dir[1] = h.dir[1]; r->dir[2] = h.dir[2];
    r->cls = h.cls; r->steps = steps; r->attempts = attempts; r->wide_attempts = wide; r->refine_evals = evals;
    r->bounces = bounces;
}

// Trace one camera ray of the scene to termination in the given precision.
inline RayResult trace_ray(const mgk_scene& s, const SceneConsts& c, uint64_t ray_id) {
    RayResult res{};
    if (s.precision == MGK_PRECISION_F64 || s.precision == MGK_PRECISION_REF32) {
        const bool f64 = s.precision == MGK_PRECISION_F64;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            MetricParams<T> m = metric_params<T>(s);
            RayInit<T> ri;
            if constexpr (std::is_same_v<T, double>) ri = camera_ray<Fuse::Fma, T>(s, c, ray_id);
            else ri = camera_ray<Fuse::None, T>(s, c, ray_id);
            GState<T> y = ri.y;
            T h = ri.h0;
            T c0 = ri.c0;
            uint32_t steps = 0, attempts = 0, evals = 0;
            Bounce bn;
            bn.ray_id = ray_id;
            Resolved<T> rs;
            while (true) {
                StepOut<T> so;
                if constexpr (std::is_same_v<T, double>) so = solve_step<Fuse::Fma, Ctl::Wide, T>(y, h, m);
                else so = solve_step<Fuse::None, Ctl::RefD, T>(y, h, m);
                attempts += so.attempts;
                ++steps;
                if constexpr (std::is_same_v<T, double>)
                    rs = resolve<Fuse::Fma, T>(s, m, y, so.y1, so.h_taken, &c0, steps,
                                               T(s.metric == KERR ? s.spin : 0.0), T(c.omega_sign), &bn);
                else
                    rs = resolve<Fuse::None, T>(s, m, y, so.y1, so.h_taken, &c0, steps,
                                                T(s.metric == KERR ? s.spin : 0.0), T(c.omega_sign), &bn);
                evals += rs.evals;
                y = rs.y_end;
                h = bn.reflected ? ri.h0 : so.h_next;
                if (rs.hit.cls != MGK_RAY_ALIVE) break;
            }
            store_result(&res, y, rs.hit, steps, attempts, std::is_same_v<T, double> ? attempts : 0u, evals,
                         bn.count);
        };
        if (f64) run(double{}); else run(float{});
    } else {
        using T = float;
        MetricParams<T> mf = metric_params<T>(s);
        MetricParams<double> md = metric_params_d(s);
        RayInit<T> ri = camera_ray<Fuse::Fma, T>(s, c, ray_id);
        GState<T> y = ri.y;
        T h = ri.h0;
        uint32_t steps = 0, attempts = 0, wide = 0, tries = 0, evals = 0;
        T c0 = ri.c0;
        Bounce bn;
        bn.ray_id = ray_id;
        double r_cur = ks_radius(y.x, md);
        Resolved<T> rs;
        while (true) {
            GState<T> y1;
            T h_used = h;
            if (mf.metric == MINKOWSKI) {
                y1 = axpy<Fuse::Fma>(h, rhs_minkowski<T>(y), y);
                ++attempts;
            } else {
                MixedAttempt a = mixed_attempt(y, h, mf, md, r_cur, c.r_plus);
                ++attempts; ++tries;
                wide += a.wide ? 1 : 0;
                h = a.h_next;
                if (!a.accept_ok && tries < mf.n_max) continue;
                y1 = a.y1;
            }
            tries = 0;
            ++steps;
            rs = resolve<Fuse::Fma, T>(s, mf, y, y1, h_used, &c0, steps, T(s.metric == KERR ? s.spin : 0.0),
                                       T(c.omega_sign), &bn);
            evals += rs.evals;
            y = rs.y_end;
            if (bn.reflected) h = ri.h0;
            if (rs.hit.cls != MGK_RAY_ALIVE) break;
            r_cur = ks_radius(y.x, md);
        }
        store_result(&res, y, rs.hit, steps, attempts, wide, evals, bn.count);
    }
    return res;
}

// ------------------------------------------------------------ star field
// Oracle-side star lookup: stars binned by polar angle, all stars of the
// bands that can reach within the star radius are tested (independent of the
// library's cube-map grid).
struct StarIndex {
    double band;                       // band height in radians
    std::vector<std::vector<uint32_t>> bands;
    const mgk_star* stars = nullptr;
    uint32_t n = 0;
    void build(const mgk_star* s, uint32_t count, double radius) {
        stars = s; n = count;
        band = std::max(0.01, 2.0 * radius);
        size_t nb = size_t(M_PI / band) + 1;
        bands.assign(nb, {});
        for (uint32_t i = 0; i < count; ++i) {
            double th = std::acos(std::max(-1.0, std::min(1.0, double(s[i].dir[1]))));
            bands[std::min(nb - 1, size_t(th / band))].push_back(i);
        }
    }
};

// Spectrum of one terminated ray at the n bin-centre wavelengths.
template <class T>
inline void ray_spectrum(const mgk_scene& s, const StarIndex* stars, const Hit<T>& h, const T* lambda, T* out) {
    const uint32_t nb = s.n_bins;
    for (uint32_t k = 0; k < nb; ++k) out[k] = T(0);
    T z = h.z;
    T z2 = z * z;
    T z5 = z2 * z2 * z;
    auto clamp = [](T v) { return (std::isnan(v) || std::isinf(v) || v < T(0)) ? T(0) : v; };
    if (h.cls == MGK_RAY_DISK) {
        T temp = T(s.disk_T_in) * T(std::pow(double(h.r_hit / T(s.disk_r_in)), -0.75));
        for (uint32_t k = 0; k < nb; ++k) out[k] = clamp(planck<T>(z * lambda[k], temp) * z5);
    } else if (h.cls == MGK_RAY_LIGHT) {
        // ABSORBED with the LED spectrum at the shifted wavelength, times z^5
        // (matter_examples.cuh:67-76, bxdf_utilities.cuh:156-163)
        for (uint32_t k = 0; k < nb; ++k) out[k] = clamp(white_led<T>(z * lambda[k]) * T(s.light_scale) * z5);
    } else if (h.cls == MGK_RAY_ESCAPED && stars && stars->n) {
        double th = std::acos(std::max(-1.0, std::min(1.0, double(h.dir[1]))));
        double rad = s.star_radius_rad;
        long lo = long((th - rad) / stars->band) - 1, hi = long((th + rad) / stars->band) + 1;
        std::vector<uint32_t> hits;
        T inv_r2 = T(1) / (T(rad) * T(rad));
        for (long b = std::max(0L, lo); b <= std::min(long(stars->bands.size()) - 1, hi); ++b)
            for (uint32_t i : stars->bands[size_t(b)]) hits.push_back(i);
        std::sort(hits.begin(), hits.end());
        for (uint32_t i : hits) {
            const mgk_star& st = stars->stars[i];
            T dx = h.dir[0] - T(st.dir[0]), dy = h.dir[1] - T(st.dir[1]), dz = h.dir[2] - T(st.dir[2]);
            T q = mad<Fuse::Fma>(dz, dz, mad<Fuse::Fma>(dy, dy, dx * dx)) * inv_r2;  // (chord / radius)^2
            if (q >= T(1)) continue;
            T kern = (T(1) - q) * (T(1) - q);
            T amp = T(st.amplitude) * kern;
            for (uint32_t k = 0; k < nb; ++k) out[k] += clamp(amp * planck<T>(z * lambda[k], T(st.temperature)) * z5);
        }
    }
}

// Sampled spectral mode (MGK_SPECTRAL_SAMPLED, the reference's stochastic
// sensor): the ray's wavelength from the inverse CDF table icdf (256 entries)
// with u = rng(seed, sample, pixel, 2) as device_sensor_utilities.cuh:25-33
// draws it, throughput 1/pdf = 255 (t[k+1] - t[k]); the boosted blackbody of
// every emitter there (planck above, independent of the library's a / (exp - 1)
// form); sampled irradiance = radiance * throughput * sensor gain
// (device_color_utilities.cuh:22-29); spread over the bins by the
// differences of the Gaussian CDF at the bin edges
// (kernel_redistribute_radiance.cu:55-92, internal_math.h:2019-2024).
// spec (n_bins values) receives the per-bin irradiance.
template <class T>
inline void sampled_spectrum(const mgk_scene& s, const StarIndex* stars, const Hit<T>& h, uint64_t ray_id,
                             const float* icdf, T* spec) {
    const uint32_t nb = s.n_bins;
    for (uint32_t k = 0; k < nb; ++k) spec[k] = T(0);
    const uint32_t pixel = uint32_t(ray_id / s.spp), sample = uint32_t(ray_id % s.spp) + s.sample_offset;
    const float x = rng_unit(s.seed, sample, pixel, 2) * float(MGK_CMF_ICDF_ENTRIES - 1);
    const uint32_t k0 = uint32_t(std::fmin(x, float(MGK_CMF_ICDF_ENTRIES) - 2.0f));
    const float f = x - float(k0);
    const float t0 = icdf[k0], t1 = icdf[k0 + 1];
    const T lam = T((t0 * (1.0f - f)) + (t1 * f));
    const T tput = T(float(MGK_CMF_ICDF_ENTRIES - 1) * (t1 - t0));
    T z = h.z;
    T z2 = z * z;
    T z5 = z2 * z2 * z;
    auto clamp = [](T v) { return (std::isnan(v) || std::isinf(v) || v < T(0)) ? T(0) : v; };
    T rad = T(0);
    if (h.cls == MGK_RAY_DISK) {
        T temp = T(s.disk_T_in) * T(std::pow(double(h.r_hit / T(s.disk_r_in)), -0.75));
        rad = clamp(planck<T>(z * lam, temp) * z5);
    } else if (h.cls == MGK_RAY_LIGHT) {
        rad = clamp(white_led<T>(z * lam) * T(s.light_scale) * z5);
    } else if (h.cls == MGK_RAY_ESCAPED && stars && stars->n) {
        double th = std::acos(std::max(-1.0, std::min(1.0, double(h.dir[1]))));
        double radius = s.star_radius_rad;
        long lo = long((th - radius) / stars->band) - 1, hi = long((th + radius) / stars->band) + 1;
        std::vector<uint32_t> hits;
        T inv_r2 = T(1) / (T(radius) * T(radius));
        for (long b = std::max(0L, lo); b <= std::min(long(stars->bands.size()) - 1, hi); ++b)
            for (uint32_t i : stars->bands[size_t(b)]) hits.push_back(i);
        std::sort(hits.begin(), hits.end());
        for (uint32_t i : hits) {
            const mgk_star& st = stars->stars[i];
            T dx = h.dir[0] - T(st.dir[0]), dy = h.dir[1] - T(st.dir[1]), dz = h.dir[2] - T(st.dir[2]);
            T q = mad<Fuse::Fma>(dz, dz, mad<Fuse::Fma>(dy, dy, dx * dx)) * inv_r2;
            if (q >= T(1)) continue;
            T kern = (T(1) - q) * (T(1) - q);
            rad += clamp(T(st.amplitude) * kern * planck<T>(z * lam, T(st.temperature)) * z5);
        }
    }
    const double W = s.width, H = s.height;
    const double inv_b = s.sensor_diag_mm / std::sqrt(W * W + H * H);
    const double area_m2 = (W * inv_b) * (H * inv_b) / 1e6;
    const T gain = T((area_m2 / (W * H)) * s.iso * 2.0 * M_PI / ((360.0 * s.fps) / s.shutter_angle_deg));
    const T irr = (rad * tput) * gain;
    if (!(irr > T(0))) return;
    const T lo = T(s.lambda_min_nm), dl = T((s.lambda_max_nm - s.lambda_min_nm) / s.n_bins);
    const T inv_s2 = T(1.0 / (s.redistribution_sigma_nm * std::sqrt(2.0)));
    T phi0 = T(0.5) * (T(1) + std::erf((lo - lam) * inv_s2));
    for (uint32_t k = 0; k < nb; ++k) {
        const T e1 = lo + T(k + 1) * dl;
        const T phi1 = T(0.5) * (T(1) + std::erf((e1 - lam) * inv_s2));
        spec[k] = irr * (phi1 - phi0);
        phi0 = phi1;
    }
}

// XYZ of a spectrum with per-bin weights w[3*k + c].
template <class T> inline void spectrum_xyz(uint32_t nb, const T* spec, const float* w, T xyz[3]) {
    T X = 0, Y = 0, Z = 0;
    for (uint32_t k = 0; k < nb; ++k) {
        X = mad<Fuse::Fma>(spec[k], T(w[3 * k + 0]), X);
        Y = mad<Fuse::Fma>(spec[k], T(w[3 * k + 1]), Y);
        Z = mad<Fuse::Fma>(spec[k], T(w[3 * k + 2]), Z);
    }
    xyz[0] = X; xyz[1] = Y; xyz[2] = Z;
}

}  // namespace orc
