// metric<MGK_METRIC_MINKOWSKI>: flat space, straight rays stepped with
// explicit Euler at h = 1000, never captured (metric_minkowski.cuh:8-84).
// Included by metric.cuh.
#pragma once

namespace mgk {

template <> struct metric<MGK_METRIC_MINKOWSKI> {
    static constexpr int tag = MGK_METRIC_MINKOWSKI;
    static constexpr bool explicit_euler = true;
    static constexpr bool has_horizon = false;
    static constexpr bool ks_radius_bound = false;

    template <class T> static void make_params(const mgk_scene& s, MP<T>& m) {
        m.spin = T(0.0);
        m.mass_sign = T(s.mass_sign < 0 ? -1.0 : 1.0);
        m.horizon = T(2) * T(s.horizon_scalar);
        m.spin_abs_gt1 = T(0);
    }
    static MGK_HD double initial_h_step() { return 1000.0; }  // metric_minkowski.cuh:25-28
    static double length_scale(double) { return 1.0; }
    static double spin(const mgk_scene&) { return 0.0; }
    static double outer_horizon(const mgk_scene&) { return 0.0; }

    template <Fuse F, class T>
    static __device__ __forceinline__ void geodesic_rhs(const S7<T>& y, T pt, const MP<T>&, S7<T>& dy) {
        rhs_minkowski<T>(y, pt, dy);
    }
    template <class T> static __device__ __forceinline__ bool in_domain(T, T, T, const MP<T>&) { return false; }
    template <class T> static MGK_HD Sym4<T> compute_g(T, T, T, const MP<T>&) {
        return Sym4<T>{T(-1), 0, 0, 0, T(1), 0, 0, T(1), 0, T(1)};
    }
    template <class T> static MGK_HD Sym4<T> compute_inv_g(T, T, T, const MP<T>&) {
        return Sym4<T>{T(-1), 0, 0, 0, T(1), 0, 0, T(1), 0, T(1)};
    }
    template <class T> static MGK_HD V4<T> reference_observer(T, T, T, const MP<T>&) {
        return V4<T>{0, 0, 0, T(1)};
    }
};

}  // namespace mgk
