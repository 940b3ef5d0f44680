// The device metric plugin contract of the geodesic path.
//
// This is the B200 build's counterpart of the reference's metric<T> contract
// (src/renderer/relativity/relativity_utilities.cuh:97-120) with its
// supported_metrics list (:197-202) and the value_list / dispatch_list that
// turn the runtime metric enum into a template instantiation
// (src/utility/cuda/cuda_host_device_utilities.h:17-27).  Every kernel of the
// path (k_generate, k_integrate, k_refine, k_tail, the reference trace) is
// templated on an int metric tag and reaches the metric only through
// metric<TAG>.  A metric is added the way the reference adds one: write a
// specialisation, list its tag, rebuild.
//
// A specialisation metric<TAG> provides (T = float or double; F = the FMA
// policy, Fuse::None for the reference's separate roundings, Fuse::Fma for
// the fused MIXED / F64 arithmetic):
//
//   static constexpr int tag = TAG;
//   static constexpr bool explicit_euler;  // steps with explicit Euler at a
//       fixed h instead of RKF45 (Minkowski, metric_minkowski.cuh:49-53)
//   static constexpr bool has_horizon;     // captures rays: in_domain is
//       tested, and MIXED takes FP64 attempts within MGK_WIDE_BAND of the
//       outer horizon
//   static constexpr bool ks_radius_bound; // the capture test may be skipped
//       while |x|^2 - a^2 > 4 horizon^2 (Kerr-Schild radius, a = m.spin)
//   template <class T> static void make_params(const mgk_scene&, MP<T>&);
//       params_t / make_params (metric_kerr.cuh:112-147): fills spin (as
//       integrated: flipped when time reversed), mass_sign, horizon (the
//       capture radius in T) and spin_abs_gt1; the integrator fields (h_max,
//       tolerances, n_max) are filled by the caller
//   static MGK_HD double initial_h_step();             (metric_kerr.cuh:149-152)
//   static double length_scale(double mass_kg);       (metric_kerr.cuh:154-157)
//       metres per unit length of the scene
//   static double spin(const mgk_scene&);   // physical spin of the oblate
//       radius used by the disk and the FP64 band (0: spherical)
//   static double outer_horizon(const mgk_scene&);    // r_+ (0: none)
//   template <Fuse F, class T> static __device__ void geodesic_rhs(
//       const S7<T>& y, T pt, const MP<T>& m, S7<T>& dy);
//       the Hamiltonian right-hand side (metric_kerr.cuh:38-105); p_t is
//       constant along the ray and passed apart
//   template <class T> static __device__ bool in_domain(T x, T y, T z, const MP<T>& m);
//       true = captured (metric_kerr.cuh:169-175)
//   template <class T> static MGK_HD Sym4<T> compute_g(T x, T y, T z, const MP<T>& m);
//   template <class T> static MGK_HD Sym4<T> compute_inv_g(T x, T y, T z, const MP<T>& m);
//   template <class T> static MGK_HD V4<T> reference_observer(T x, T y, T z, const MP<T>& m);
//       (metric_kerr.cuh:177-226)
//
// The built-in specialisations are in metric_minkowski.cuh,
// metric_schwarzschild.cuh and metric_kerr.cuh.  A build may add its own: a
// header named by -DMGK_USER_METRIC_HEADER="path" that defines
// specialisations under unused tags (16 and up) and lists them as
// `using user_metrics = metric_list<TAG, ...>;` in namespace mgk.
#pragma once

#include <cmath>

#include "../../../csrc/dev_physics.cuh"
#include "../../../../include/mgk.h"

namespace mgk {

template <int... TAGS> struct metric_list {};

}  // namespace mgk

#include "metric_minkowski.cuh"
#include "metric_schwarzschild.cuh"
#include "metric_kerr.cuh"

#ifdef MGK_USER_METRIC_HEADER
#include MGK_USER_METRIC_HEADER
#else
namespace mgk {
using user_metrics = metric_list<>;
}
#endif

namespace mgk {

template <class A, class B> struct metric_list_cat;
template <int... A, int... B> struct metric_list_cat<metric_list<A...>, metric_list<B...>> {
    using type = metric_list<A..., B...>;
};

// The reference's supported_metrics: the three built-in metrics and the
// build's own.
using builtin_metrics = metric_list<MGK_METRIC_MINKOWSKI, MGK_METRIC_SCHWARZSCHILD, MGK_METRIC_KERR>;
using supported_metrics = typename metric_list_cat<builtin_metrics, user_metrics>::type;

// Calls fn(metric<TAG>{}) for the listed TAG equal to `tag`; false when the
// tag is not listed.  Host or device.
#pragma nv_exec_check_disable
template <class Fn, int... TAGS>
MGK_HD bool dispatch_metric(metric_list<TAGS...>, int tag, Fn&& fn) {
    bool found = false;
    ((tag == TAGS ? (fn(metric<TAGS>{}), found = true) : false), ...);
    return found;
}

#pragma nv_exec_check_disable
template <class Fn> MGK_HD bool with_metric(int tag, Fn&& fn) {
    return dispatch_metric(supported_metrics{}, tag, static_cast<Fn&&>(fn));
}

inline bool metric_supported(int tag) {
    return with_metric(tag, [](auto) {});
}

// The integrator parameters of a scene in T: the metric's make_params plus
// the integrator fields (h_max is the reference's 1000, metric_kerr.cuh:131,
// unless the scene sets another).
template <class MT, class T> inline MP<T> scene_params(const mgk_scene& s) {
    MP<T> m{};
    MT::template make_params<T>(s, m);
    m.h_max = T(s.h_max);
    m.abs_tol = T(s.abs_tol);
    m.rel_tol = T(s.rel_tol);
    m.n_max = s.n_max_substep;
    set_spin_consts(m);
    return m;
}

}  // namespace mgk
