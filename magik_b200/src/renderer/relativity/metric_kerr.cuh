// metric<MGK_METRIC_KERR>: the Kerr metric in Kerr-Schild Cartesian
// coordinates, spin axis +y, M = 1 (metric_kerr.cuh:8-226).  Included by
// metric.cuh.
#pragma once

namespace mgk {

template <> struct metric<MGK_METRIC_KERR> {
    static constexpr int tag = MGK_METRIC_KERR;
    static constexpr bool explicit_euler = false;
    static constexpr bool has_horizon = true;
    static constexpr bool ks_radius_bound = true;

    // make_params (metric_kerr.cuh:125-147): the spin flipped when time
    // reversed; the capture radius (1 + sqrt(1 - a^2)) * horizon_scalar and
    // the |a| > 1 flag evaluated in T, as in_domain evaluates them.
    template <class T> static void make_params(const mgk_scene& s, MP<T>& m) {
        const double a_t = s.time_reversed ? -s.spin : s.spin;
        m.spin = T(a_t);
        m.mass_sign = T(s.mass_sign < 0 ? -1.0 : 1.0);
        const T a = T(a_t);
        m.horizon = (T(1) + std::sqrt(T(1) - a * a)) * T(s.horizon_scalar);
        m.spin_abs_gt1 = (a > T(1) || a < T(-1)) ? T(1) : T(0);
    }
    static MGK_HD double initial_h_step() { return 1.0; }
    static double length_scale(double mass_kg) {
        return 6.67430e-11 * mass_kg / (299792458.0 * 299792458.0);
    }
    static double spin(const mgk_scene& s) { return s.spin; }
    static double outer_horizon(const mgk_scene& s) {
        const double d = 1.0 - s.spin * s.spin;
        return 1.0 + std::sqrt(d > 0.0 ? d : 0.0);
    }

    // The fused right-hand side (MIXED / F64) or the reference's tree (REF32).
    template <Fuse F, class T>
    static __device__ __forceinline__ void geodesic_rhs(const S7<T>& y, T pt, const MP<T>& m, S7<T>& dy) {
        if constexpr (F == Fuse::Fma) rhs_kerr_fused<T>(y, pt, m, dy);
        else rhs_kerr<F, T>(y, pt, m.spin, dy);
    }
    // metric_kerr.cuh:169-175: NaN radii capture, |a| > 1 never does.
    template <class T> static __device__ __forceinline__ bool in_domain(T x, T y, T z, const MP<T>& m) {
        if (m.spin_abs_gt1 != T(0)) return false;
        T r = kerr_schild_r(x, y, z, m.spin);
        if (m.horizon < r) return false;
        return true;
    }
    // g = eta + f k k (metric_kerr.cuh:177-190).
    template <class T> static MGK_HD Sym4<T> compute_g(T x, T y, T z, const MP<T>& m) {
        const T a = m.spin;
        const T r = kerr_schild_r(x, y, z, a);
        const T f = T(2) * r * r * r / (r * r * r * r + a * a * y * y);
        const T kx = (r * x - a * z) / (r * r + a * a);
        const T ky = y / r;
        const T kz = (r * z + a * x) / (r * r + a * a);
        return Sym4<T>{T(-1) + f, f * kx, f * ky, f * kz, T(1) + f * kx * kx, f * kx * ky, f * kx * kz,
                       T(1) + f * ky * ky, f * ky * kz, T(1) + f * kz * kz};
    }
    // g^-1 = eta - f k^ k^ with k^ = eta k (k is null) (metric_kerr.cuh:192-205).
    template <class T> static MGK_HD Sym4<T> compute_inv_g(T x, T y, T z, const MP<T>& m) {
        const T a = m.spin;
        const T r = kerr_schild_r(x, y, z, a);
        const T f = T(2) * r * r * r / (r * r * r * r + a * a * y * y);
        const T kx = (r * x - a * z) / (r * r + a * a);
        const T ky = y / r;
        const T kz = (r * z + a * x) / (r * r + a * a);
        return Sym4<T>{T(-1) - f, f * kx, f * ky, f * kz, T(1) - f * kx * kx, -f * kx * ky, -f * kx * kz,
                       T(1) - f * ky * ky, -f * ky * kz, T(1) - f * kz * kz};
    }
    // The zero-angular-momentum observer (metric_kerr.cuh:207-226).
    template <class T> static MGK_HD V4<T> reference_observer(T x, T y, T z, const MP<T>& m) {
        const T a = m.spin;
        T r = kerr_schild_r(x, y, z, a);
        T r_sq = r * r;
        T a_sq = a * a;
        T cos_theta = y / r;
        T sin2_theta = T(1) - cos_theta * cos_theta;
        T sigma = r_sq + a_sq * cos_theta * cos_theta;
        T delta = r_sq - T(2) * r + a_sq;
        T Lambda = (r_sq + a_sq) * (r_sq + a_sq) - a_sq * delta * sin2_theta;
        T u_t = sqrt(Lambda / (delta * sigma));
        T u_phi = T(2) * a * r / sqrt(Lambda * delta * sigma);
        return V4<T>{z * u_phi, T(0), -x * u_phi, u_t};
    }
};

}  // namespace mgk
