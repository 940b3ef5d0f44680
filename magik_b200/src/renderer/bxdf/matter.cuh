// The matter plugin contract of the geodesic path.
//
// The counterpart of the reference's registered_matter
// (src/renderer/kernels/kernel_bxdf.cu:105-107), whose types each provide
// local_proper_velocity_function (the emitter's motion) and
// material_function (what the matter does to the ray: emit, absorb,
// reflect) (src/renderer/bxdf/matter_examples.cuh:12-31).  Here a ray's
// termination class names the matter it ended on, and matter<CLASS> gives:
//
//   static constexpr bool at_infinity;   // the emitter is static at infinity:
//       the redshift is c0 / p_t (no four-velocity needed)
//   template <int METRIC, class T> static __device__ V4<T> four_velocity(
//       const DevScene<T>&, T x, T y, T z, T r);
//       the emitter's four-velocity at the located hit (the reference's
//       local_proper_velocity_function turned into a four-velocity by
//       rest_frame_four_velocity, bxdf_utilities.cuh:53-87); the redshift is
//       g = c0 / (u . p) (compute_redshift_factor,
//       relativity_utilities.cuh:175-195)
//   emission (material_function's emitted part, in the emitter's frame), one of
//     template <class T, class Hit, class Add> static __device__ void blackbodies(
//         const DevScene<T>&, const Hit&, const mgk_star*, const Grid&, Add&& add);
//         calls add(amplitude, temperature) for each blackbody it emits
//     template <class T> static __device__ T radiance(const DevScene<T>&, T lambda_nm);
//         spectral radiance at the emitted wavelength
//   The shading boosts the emission by g^5 and clamps NaN / negative values
//   to zero (apply_absorbed, bxdf_utilities.cuh:156-163).
//
// Implemented by the thin Keplerian disk (MGK_RAY_DISK), the star field of
// the celestial sphere (MGK_RAY_ESCAPED), the room's white-LED light
// (MGK_RAY_LIGHT) and the horizon, which is black (MGK_RAY_HORIZON), as the
// reference's horizon and celestial-sphere matter are
// (matter_examples.cuh:79-96).  Included by dev_scene.cuh.
#pragma once

namespace mgk {

template <int CLASS> struct matter;

// The thin disk in y = 0: circular Keplerian orbits
// Omega = +-1 / (r^(3/2) + a) (Bardeen, Press and Teukolsky 1972), the
// sign following the time reversal; a Novikov-Thorne-like temperature
// T(r) = T_in (r / r_in)^(-3/4).
template <> struct matter<MGK_RAY_DISK> {
    static constexpr bool at_infinity = false;
    template <int METRIC, class T>
    static __device__ __forceinline__ V4<T> four_velocity(const DevScene<T>& P, T x, T, T z, T r) {
        return disk_velocity<METRIC, T>(x, z, r, P);
    }
    template <class T, class Hit, class Grid, class Add>
    static __device__ __forceinline__ void blackbodies(const DevScene<T>& P, const Hit& h, const mgk_star*,
                                                       const Grid&, Add&& add) {
        add(T(1), P.disk_T_in * exp2(T(-0.75) * log2(h.r_hit / P.disk_r_in)));
    }
};

// The celestial sphere: static emitters at infinity (u . p = p_t); each
// star a blackbody disc of angular radius R with profile (1 - (d / R)^2)^2,
// found through the cube-map grid of the escape direction.
template <> struct matter<MGK_RAY_ESCAPED> {
    static constexpr bool at_infinity = true;
    template <class T, class Hit, class Grid, class Add>
    static __device__ __forceinline__ void blackbodies(const DevScene<T>& P, const Hit& h, const mgk_star* stars,
                                                       const Grid& grid, Add&& add) {
        if (grid.n == 0u) return;
        const uint32_t cell = cube_cell(float(h.d0), float(h.d1), float(h.d2), grid.n);
        const uint32_t j1 = grid.cell_start[cell + 1];
        for (uint32_t j = grid.cell_start[cell]; j < j1; ++j) {
            const mgk_star st = stars[grid.cell_stars[j]];
            T dx = h.d0 - T(st.dir[0]), dy = h.d1 - T(st.dir[1]), dz = h.d2 - T(st.dir[2]);
            T q = mad<Fuse::Fma>(dz, dz, mad<Fuse::Fma>(dy, dy, dx * dx)) * P.star_inv_r2;
            if (q >= T(1)) continue;
            add(T(st.amplitude) * ((T(1) - q) * (T(1) - q)), T(st.temperature));
        }
    }
};

// The room's light box: at rest with the metric's reference observer
// (matter_examples.cuh:60-77), emitting the white-LED spectrum scaled by
// light_scale.
template <> struct matter<MGK_RAY_LIGHT> {
    static constexpr bool at_infinity = false;
    template <int METRIC, class T>
    static __device__ __forceinline__ V4<T> four_velocity(const DevScene<T>& P, T x, T y, T z, T) {
        return metric<METRIC>::template reference_observer<T>(x, y, z, P.m);
    }
    template <class T> static __device__ __forceinline__ T radiance(const DevScene<T>& P, T lambda_nm) {
        return white_led<T>(lambda_nm) * P.light_scale;
    }
};

// The horizon absorbs and emits nothing.
template <> struct matter<MGK_RAY_HORIZON> {
    static constexpr bool at_infinity = false;
};

}  // namespace mgk
