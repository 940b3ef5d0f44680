// metric<MGK_METRIC_SCHWARZSCHILD>: Schwarzschild in Kerr-Schild Cartesian
// coordinates, M = 1, with the reference's negative-mass option
// (metric_schwarzschild.cuh:8-171).  Included by metric.cuh.
#pragma once

namespace mgk {

template <> struct metric<MGK_METRIC_SCHWARZSCHILD> {
    static constexpr int tag = MGK_METRIC_SCHWARZSCHILD;
    static constexpr bool explicit_euler = false;
    static constexpr bool has_horizon = true;
    static constexpr bool ks_radius_bound = true;

    // make_params (metric_schwarzschild.cuh:79-120): capture at 2 M times the
    // horizon scalar; the mass sign flips the attraction.
    template <class T> static void make_params(const mgk_scene& s, MP<T>& m) {
        m.spin = T(0.0);
        m.mass_sign = T(s.mass_sign < 0 ? -1.0 : 1.0);
        m.horizon = T(2) * T(s.horizon_scalar);
        m.spin_abs_gt1 = T(0);
    }
    static MGK_HD double initial_h_step() { return 1.0; }
    static double length_scale(double mass_kg) {
        return 6.67430e-11 * std::fabs(mass_kg) / (299792458.0 * 299792458.0);
    }
    static double spin(const mgk_scene&) { return 0.0; }
    static double outer_horizon(const mgk_scene&) { return 2.0; }

    template <Fuse F, class T>
    static __device__ __forceinline__ void geodesic_rhs(const S7<T>& y, T pt, const MP<T>& m, S7<T>& dy) {
        if constexpr (F == Fuse::Fma) rhs_schwarzschild_fused<T>(y, pt, m.mass_sign, dy);
        else rhs_schwarzschild<F, T>(y, pt, m.mass_sign, dy);
    }
    // metric_schwarzschild.cuh:136-141: NaN radii do not capture; a negative
    // mass captures only at the origin.
    template <class T> static __device__ __forceinline__ bool in_domain(T x, T y, T z, const MP<T>& m) {
        T r = sqrt(x * x + y * y + z * z);
        if (m.mass_sign < T(0)) return r < T(1e-3);
        return r <= m.horizon;
    }
    // metric_schwarzschild.cuh:143-153.
    template <class T> static MGK_HD Sym4<T> compute_g(T x, T y, T z, const MP<T>& m) {
        const T r = sqrt(x * x + y * y + z * z);
        const T f = T(2) * m.mass_sign / r;
        const T kx = x / r, ky = y / r, kz = z / r;
        return Sym4<T>{T(-1) + f, f * kx, f * ky, f * kz, T(1) + f * kx * kx, f * kx * ky, f * kx * kz,
                       T(1) + f * ky * ky, f * ky * kz, T(1) + f * kz * kz};
    }
    template <class T> static MGK_HD Sym4<T> compute_inv_g(T x, T y, T z, const MP<T>& m) {
        const T r = sqrt(x * x + y * y + z * z);
        const T f = T(2) * m.mass_sign / r;
        const T kx = x / r, ky = y / r, kz = z / r;
        return Sym4<T>{T(-1) - f, f * kx, f * ky, f * kz, T(1) - f * kx * kx, -f * kx * ky, -f * kx * kz,
                       T(1) - f * ky * ky, -f * ky * kz, T(1) - f * kz * kz};
    }
    // The static observer (metric_schwarzschild.cuh:167-171).
    template <class T> static MGK_HD V4<T> reference_observer(T x, T y, T z, const MP<T>& m) {
        const Sym4<T> g = compute_g<T>(x, y, z, m);
        return V4<T>{0, 0, 0, T(1) / sqrt(-g.tt)};
    }
};

}  // namespace mgk
