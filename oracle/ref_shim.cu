// Thin C entry points over the reference's own code, compiled together with
// the reference sources into oracle/_ref (test and baseline infrastructure,
// never shipped).  Mirrors the argument checks of magik_trace_geodesic
// (src/magik.cpp:196-207), exposes the reference's colour-weight routine
// (host_color_utilities.cuh:145-178), and renders pixels with the reference's
// own RKF45 step (metric<T>::solve_step, metric_kerr.cuh:159-162 /
// metric_schwarzschild.cuh) inside the CPU oracle's camera, termination and
// spectral stages, which the reference's CPU tracer lacks.
#include <algorithm>
#include <atomic>
#include <functional>
#include <thread>
#include <vector>

#include "host_trace_geodesic.h"
#include "host_color_utilities.cuh"
#include "cuda_host_utilities.h"
#include "magik.h"
#include "kernel_advance_geodesic.cuh"
#include "relativity_utilities.cuh"
#include "metric_minkowski.cuh"
#include "metric_schwarzschild.cuh"
#include "metric_kerr.cuh"

#include "oracle_scene.hpp"

extern "C" __attribute__((visibility("default"))) int ref_trace_geodesic(
    magik_trace_geodesic_container_t* container, magik_trace_geodesic_inital_conditions_t ic,
    magik_trace_geodesic_metric_parameters_t mp, magik_trace_geodesic_integrator_parameters_t ip) {
    if (!container || !container->steps) return MAGIK_ERROR_INVALID_POINTER;
    if (container->capacity != (sizeof(magik_trace_geodesic_step_t) * container->n_allocated_step))
        return MAGIK_ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH;
    return magik::host_trace_geodesic(container, ic, mp, ip) ? MAGIK_SUCCESS : MAGIK_ERROR_UNKNOWN;
}

extern "C" __attribute__((visibility("default"))) int ref_cmf_weights(unsigned n_bins, float lmin, float lmax,
                                                                      float* out) {
    magik::vec3f w[MAGIK_N_MAX_SPECTRAL_BIN];
    if (n_bins == 0 || n_bins > MAGIK_N_MAX_SPECTRAL_BIN) return 1;
    magik::compute_normalized_isi_cmf_weights(w, n_bins, lmin, lmax, magik::fetch_cmf_info(MAGIK_CMF_CIE_1931));
    for (unsigned i = 0; i < n_bins; ++i) {
        out[3 * i + 0] = w[i].x;
        out[3 * i + 1] = w[i].y;
        out[3 * i + 2] = w[i].z;
    }
    return 0;
}

// The reference's inverse CDF table of the CIE 1931 colour-matching
// functions (compute_tabulated_cmf_inverse_cdf, floor 0.05 as
// color_pipeline.cuh:36 calls it): MAGIK_N_CMF_INVERSE_CDF_BIN wavelengths.
extern "C" __attribute__((visibility("default"))) int ref_cmf_inverse_cdf(float lmin, float lmax, float* out) {
    magik::compute_tabulated_cmf_inverse_cdf(out, 0.05f, lmin, lmax, magik::fetch_cmf_info(MAGIK_CMF_CIE_1931));
    return MAGIK_N_CMF_INVERSE_CDF_BIN;
}

namespace {

void ref_parallel_for(uint64_t n, int nthreads, const std::function<void(uint64_t)>& fn) {
    if (nthreads <= 1 || n < 64) {
        for (uint64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&] {
            for (;;) {
                uint64_t b = next.fetch_add(64);
                if (b >= n) break;
                uint64_t e = std::min(n, b + 64);
                for (uint64_t i = b; i < e; ++i) fn(i);
            }
        });
    for (auto& t : th) t.join();
}

// One camera ray: the oracle's REF32 initial conditions, then per accepted
// step the reference's own solve_step (float, its op order and its powf) and
// the oracle's disk / escape / horizon / step-cap tests.
template <e_magik_spacetime_metric_types MT>
orc::RayResult trace_ref(const mgk_scene& s, const orc::SceneConsts& c, uint64_t ray_id,
                         typename magik::metric<MT>::params_t p) {
    using namespace orc;
    MetricParams<float> m = metric_params<float>(s);
    RayInit<float> ri = camera_ray<Fuse::None, float>(s, c, ray_id);
    GState<float> y = ri.y;
    float h = ri.h0;
    uint32_t steps = 0, attempts = 0, evals = 0;
    Resolved<float> rs;
    const float spin = float(s.metric == MGK_METRIC_KERR ? s.spin : 0.0);
    for (;;) {
        magik::geodesic_step_values_t y0{magik::vec4f{y.x.x, y.x.y, y.x.z, y.x.t},
                                          magik::vec4f{y.p.x, y.p.y, y.p.z, y.p.t}};
        float h_step = h, h_taken = 0.0f;
        magik::geodesic_step_values_t y1r = magik::metric<MT>::solve_step(y0, p, &h_step, &h_taken);
        GState<float> y1;
        y1.x = V4<float>{y1r.four_position.x, y1r.four_position.y, y1r.four_position.z, y1r.four_position.t};
        y1.p = V4<float>{y1r.four_momentum.x, y1r.four_momentum.y, y1r.four_momentum.z, y1r.four_momentum.t};
        ++attempts;  // the reference does not report its retries
        ++steps;
        rs = resolve<Fuse::None, float>(s, m, y, y1, h_taken, ri.c0, steps, spin, float(c.omega_sign));
        evals += rs.evals;
        y = rs.y_end;
        h = h_step;
        if (rs.hit.cls != MGK_RAY_ALIVE) break;
    }
    RayResult res{};
    store_result(&res, y, rs.hit, steps, attempts, 0u, evals);
    return res;
}

}  // namespace

// Pixels [first, first + n*stride) of the scene (stride apart) rendered with
// the reference's RKF45 step: mean XYZ per pixel into xyz_out (3 doubles per
// pixel).  Kerr and Schwarzschild scenes; returns nonzero otherwise.
extern "C" __attribute__((visibility("default"))) int ref_render_pixels(
    const mgk_scene* s, const mgk_star* stars, uint32_t n_stars, const float* w, uint64_t first_pixel,
    uint32_t n_pixels, uint64_t pixel_stride, double* xyz_out, int nthreads) {
    using namespace orc;
    if (!s || !xyz_out || (n_stars && !stars) || !w) return 2;
    if (s->metric != MGK_METRIC_KERR && s->metric != MGK_METRIC_SCHWARZSCHILD) return 1;
    SceneConsts c = scene_consts(*s);
    StarIndex idx;
    idx.build(stars, n_stars, s->star_radius_rad);
    const uint32_t nb = s->n_bins, spp = s->spp;
    const double dl = (s->lambda_max_nm - s->lambda_min_nm) / nb;
    const bool tr = s->time_reversed != 0;
    magik::kerr_metric::params_t pk{tr, 1.0f, float(tr ? -s->spin : s->spin), float(s->horizon_scalar),
                                    float(s->h_max), float(s->abs_tol), float(s->rel_tol), s->n_max_substep};
    magik::metric<e_magik_spacetime_metric_types::SCHWARZSCHILD>::params_t ps{};
    ps.time_reversed = tr;
    ps.mass_parameter = 1.0f;  // only sets the length scale, which the dimensionless step does not use
    ps.mass_sign = float(s->mass_sign < 0 ? -1.0 : 1.0);
    ps.event_horizon_scalar = float(s->horizon_scalar);
    ps.h_max = float(s->h_max);
    ps.abs_tol = float(s->abs_tol);
    ps.rel_tol = float(s->rel_tol);
    ps.n_max = s->n_max_substep;
    ref_parallel_for(n_pixels, nthreads, [&](uint64_t i) {
        const uint64_t pix = first_pixel + i * pixel_stride;
        float acc[3] = {0, 0, 0};
        for (uint32_t smp = 0; smp < spp; ++smp) {
            RayResult r = s->metric == MGK_METRIC_KERR
                              ? trace_ref<e_magik_spacetime_metric_types::KERR>(*s, c, pix * spp + smp, pk)
                              : trace_ref<e_magik_spacetime_metric_types::SCHWARZSCHILD>(*s, c, pix * spp + smp, ps);
            float lam[MGK_MAX_BINS], spec[MGK_MAX_BINS], o[3];
            for (uint32_t k = 0; k < nb; ++k) lam[k] = float(s->lambda_min_nm + (k + 0.5) * dl);
            Hit<float> h;
            h.cls = r.cls; h.z = float(r.z); h.r_hit = float(r.r_hit);
            h.dir[0] = float(r.dir[0]); h.dir[1] = float(r.dir[1]); h.dir[2] = float(r.dir[2]);
            ray_spectrum<float>(*s, &idx, h, lam, spec);
            spectrum_xyz<float>(nb, spec, w, o);
            for (int k = 0; k < 3; ++k) acc[k] += o[k];
        }
        for (int k = 0; k < 3; ++k) xyz_out[3 * i + k] = double(acc[k] / float(spp));
    });
    return 0;
}
