// A test-only metric plugin: Schwarzschild (M = 1, Kerr-Schild Cartesian)
// written against the metric<TAG> contract of
// magik_b200/src/renderer/relativity/metric.cuh under the user tag 16, the
// way a reference-side metric<T> specialisation is dropped into a build.
//
// Built into a variant library with
//   -DMGK_USER_METRIC_HEADER="<path of this file>"
// (magik_b200/build.py user_metric_build).  Everything but the Hamiltonian
// right-hand side is restated here; the right-hand side is the library's
// Schwarzschild arithmetic (rhs_schwarzschild_fused for the fused MIXED / F64
// modes, rhs_schwarzschild for the reference's separate roundings), so that
// tests/test_gpu_plugin.py can ask for records bit-identical to the built-in
// metric<MGK_METRIC_SCHWARZSCHILD>.
#pragma once

namespace mgk {

constexpr int kUserSchwarzschild = 16;

template <> struct metric<kUserSchwarzschild> {
    static constexpr int tag = kUserSchwarzschild;
    static constexpr bool explicit_euler = false;
    static constexpr bool has_horizon = true;
    static constexpr bool ks_radius_bound = true;

    template <class T> static void make_params(const mgk_scene& s, MP<T>& m) {
        m.spin = T(0.0);
        m.mass_sign = s.mass_sign < 0 ? T(-1) : T(1);
        m.horizon = T(s.horizon_scalar) * T(2);
        m.spin_abs_gt1 = T(0);
    }
    static MGK_HD double initial_h_step() { return 1.0; }
    static double length_scale(double mass_kg) {
        const double G = 6.67430e-11, c = 299792458.0;
        return G * std::fabs(mass_kg) / (c * c);
    }
    static double spin(const mgk_scene&) { return 0.0; }
    static double outer_horizon(const mgk_scene&) { return 2.0; }

    template <Fuse F, class T>
    static __device__ __forceinline__ void geodesic_rhs(const S7<T>& y, T pt, const MP<T>& m, S7<T>& dy) {
        if constexpr (F == Fuse::Fma) rhs_schwarzschild_fused<T>(y, pt, m.mass_sign, dy);
        else rhs_schwarzschild<F, T>(y, pt, m.mass_sign, dy);
    }
    template <class T> static __device__ __forceinline__ bool in_domain(T x, T y, T z, const MP<T>& m) {
        const T r = sqrt(x * x + y * y + z * z);
        return m.mass_sign < T(0) ? r < T(1e-3) : r <= m.horizon;
    }
    // g = eta + (2 m / r) k k with k = x / r (the Kerr-Schild form at a = 0)
    template <class T> static MGK_HD Sym4<T> compute_g(T x, T y, T z, const MP<T>& m) {
        const T r = sqrt(x * x + y * y + z * z);
        const T f = T(2) * m.mass_sign / r;
        const T k[3] = {x / r, y / r, z / r};
        Sym4<T> g;
        g.tt = T(-1) + f;
        g.tx = f * k[0]; g.ty = f * k[1]; g.tz = f * k[2];
        g.xx = T(1) + f * k[0] * k[0]; g.xy = f * k[0] * k[1]; g.xz = f * k[0] * k[2];
        g.yy = T(1) + f * k[1] * k[1]; g.yz = f * k[1] * k[2];
        g.zz = T(1) + f * k[2] * k[2];
        return g;
    }
    // g^-1 = eta - f k^ k^, k^ = (k, -1)
    template <class T> static MGK_HD Sym4<T> compute_inv_g(T x, T y, T z, const MP<T>& m) {
        const T r = sqrt(x * x + y * y + z * z);
        const T f = T(2) * m.mass_sign / r;
        const T k[3] = {x / r, y / r, z / r};
        Sym4<T> gi;
        gi.tt = T(-1) - f;
        gi.tx = f * k[0]; gi.ty = f * k[1]; gi.tz = f * k[2];
        gi.xx = T(1) - f * k[0] * k[0]; gi.xy = -f * k[0] * k[1]; gi.xz = -f * k[0] * k[2];
        gi.yy = T(1) - f * k[1] * k[1]; gi.yz = -f * k[1] * k[2];
        gi.zz = T(1) - f * k[2] * k[2];
        return gi;
    }
    // the static observer u = (0, 0, 0, 1 / sqrt(-g_tt))
    template <class T> static MGK_HD V4<T> reference_observer(T x, T y, T z, const MP<T>& m) {
        const T gtt = compute_g<T>(x, y, z, m).tt;
        return V4<T>{T(0), T(0), T(0), T(1) / sqrt(-gtt)};
    }
};

using user_metrics = metric_list<kUserSchwarzschild>;

}  // namespace mgk
