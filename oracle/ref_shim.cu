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
#include "color_pipeline.cuh"
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

// The reference's colour resolve (color_pipeline.cuh:21-48 with the view
// transforms' make_params / apply and the display colourspaces' encode,
// composed as scene_to_display_referred_color composes them,
// device_color_utilities.cuh:56-70), for the library's display tests.
namespace {
magik::color_settings_t ref_color_settings(const mgk_display_settings* ds) {
    magik::color_settings_t cs;
    cs.scene_colorspace_type = e_magik_scene_colorspace_types(ds->scene_colorspace);
    cs.view_transform_type = e_magik_view_transform_types(ds->view_transform);
    cs.display_colorspace_type = e_magik_display_colorspace_types(ds->display_colorspace);
    cs.vt_gt7_mode = e_magik_gran_turismo_7_mode_types(ds->gt7_mode);
    cs.vt_agx_look = e_magik_agx_look_types(ds->agx_look);
    cs.white_point = float(ds->white_point_K);
    cs.tint = float(ds->tint);
    cs.vt_reinhard_extended_white_luminance = float(ds->reinhard_white_luminance);
    cs.vt_khronos_pbr_neutral_start_compression = float(ds->khronos_start_compression);
    cs.vt_khronos_pbr_neutral_desaturation = float(ds->khronos_desaturation);
    cs.vt_gt7_sdr_paper_white = float(ds->gt7_sdr_paper_white);
    cs.vt_gt7_reference_luminance = float(ds->gt7_reference_luminance);
    cs.vt_gt7_jzazbz_exponent_scale_factor = float(ds->gt7_jzazbz_exponent_scale);
    return cs;
}
void put_m(float* d, const magik::mat3f& m) {
    const float v[9] = {m.m11, m.m12, m.m13, m.m21, m.m22, m.m23, m.m31, m.m32, m.m33};
    for (int i = 0; i < 9; ++i) d[i] = v[i];
}
magik::mat3f ref_xyz_to_scene(const magik::color_settings_t& cs) {
    auto sc = magik::fetch_scene_colorspace(cs.scene_colorspace_type);
    auto cmf = magik::fetch_cmf_info(cs.cmf_type);
    magik::vec3f src = magik::compute_white_point_xyz(cs.white_point, cs.tint, cmf);
    magik::vec3f dst = magik::cie_xy_to_cie_XYZ(sc.white_point_cie_xy);
    return sc.cie_XYZ_to_colorspace * magik::chromatic_adaptation(src, dst);
}
template <e_magik_view_transform_types V>
magik::vec3f ref_display_one(const magik::color_settings_t& cs, const magik::color_pipeline_descriptor_t& d,
                             const typename magik::generic_view_transform_t<V>::params_t& vp, magik::vec3f scene) {
    magik::vec3f c = magik::generic_view_transform_t<V>::apply(scene, vp);
    c = d.scene_to_display_referred * c;
    magik::vec3f out{0, 0, 0};
    magik::dispatch_list(magik::supported_display_colorspaces{}, d.display_colorspace_type, [&](auto tag) {
        constexpr auto D = decltype(tag)::value;
        out = magik::generic_display_colorspace_t<D>::encode(c);
    });
    return out;
}
}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_display_pipeline(const mgk_display_settings* ds,
                                                                           mgk_display_pipeline* out) {
    using namespace magik;
    color_settings_t cs = ref_color_settings(ds);
    color_pipeline_descriptor_t d = color_pipeline_descriptor_t::create(cs);
    *out = mgk_display_pipeline{};
    out->view_transform = ds->view_transform;
    out->display_colorspace = ds->display_colorspace;
    out->gt7_mode = ds->gt7_mode;
    out->agx_look = ds->agx_look;
    put_m(out->xyz_to_scene, ref_xyz_to_scene(cs));
    put_m(out->scene_to_display, d.scene_to_display_referred);
    auto re = generic_view_transform_t<MAGIK_VIEW_TRANSFORM_REINHARD_EXTENDED>::make_params(cs);
    out->luminance_weights[0] = re.luminance_weights.x;
    out->luminance_weights[1] = re.luminance_weights.y;
    out->luminance_weights[2] = re.luminance_weights.z;
    out->reinhard_white_luminance = re.white_luminance;
    auto kh = generic_view_transform_t<MAGIK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL>::make_params(cs);
    out->khronos_start_compression = kh.start_compression;
    out->khronos_desaturation = kh.desaturation;
    auto gt = generic_view_transform_t<MAGIK_VIEW_TRANSFORM_GRAN_TURISMO_7>::make_params(cs);
    auto ag = generic_view_transform_t<MAGIK_VIEW_TRANSFORM_AGX>::make_params(cs);
    if (ds->view_transform == MAGIK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL) {
        put_m(out->vt_to_working, kh.to_linear_rec_709);
        put_m(out->vt_from_working, kh.to_scene_colorspace);
    } else {
        put_m(out->vt_to_working, gt.to_linear_rec_2020);
        put_m(out->vt_from_working, gt.to_scene_colorspace);
    }
    put_m(out->agx_inset, ag.agx_inset_matrix);
    put_m(out->agx_outset, ag.agx_outset_matrix);
    out->gt7_reference_luminance = gt.reference_luminance;
    out->gt7_jzazbz_exponent_scale = gt.jzazbz_exponent_scale_factor;
    out->gt7_peak_intensity = gt.peak_intensity_;
    out->gt7_alpha = gt.alpha_;
    out->gt7_mid_point = gt.mid_point_;
    out->gt7_linear_section = gt.linear_section_;
    out->gt7_toe_strength = gt.toe_strength_;
    out->gt7_kA = gt.kA_;
    out->gt7_kB = gt.kB_;
    out->gt7_kC = gt.kC_;
    out->gt7_sdr_correction = gt.sdr_correction_factor_;
    out->gt7_fb_luminance_target = gt.framebuffer_luminance_target_;
    out->gt7_fb_luminance_target_ucs = gt.framebuffer_luminance_target_ucs;
    out->gt7_blend_ratio = gt.blend_ratio_;
    out->gt7_fade_start = gt.fade_start_;
    out->gt7_fade_end = gt.fade_end_;
    return 0;
}

// Display RGB of n XYZ triples with the reference's own functions: the
// white-balanced XYZ -> scene matrix, the view transform, the scene ->
// display matrix and the display's transfer function.
extern "C" __attribute__((visibility("default"))) int ref_display_pixels(const mgk_display_settings* ds,
                                                                         const float* xyz, uint32_t n, float* out) {
    using namespace magik;
    color_settings_t cs = ref_color_settings(ds);
    color_pipeline_descriptor_t d = color_pipeline_descriptor_t::create(cs);
    const mat3f m = ref_xyz_to_scene(cs);
    bool ok = dispatch_list(supported_view_transforms{}, cs.view_transform_type, [&](auto tag) {
        constexpr auto V = decltype(tag)::value;
        auto vp = generic_view_transform_t<V>::make_params(cs);
        for (uint32_t i = 0; i < n; ++i) {
            vec3f scene = m * vec3f{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
            vec3f o = ref_display_one<V>(cs, d, vp, scene);
            out[3 * i] = o.x;
            out[3 * i + 1] = o.y;
            out[3 * i + 2] = o.z;
        }
    });
    return ok ? 0 : 1;
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

// The reference's mirror reflection at a wall (bxdf_diffuse_matter_t on a
// wall normal to x, matter_examples.cuh:40-48) composed from its own frame
// code as generate_velocity_context / generate_material_context /
// apply_reflected do (bxdf_utilities.cuh:53-109,139-154), for a covariant
// momentum p at x and the global facing normal n: the outgoing covariant
// momentum and the new initial contraction.
template <e_magik_spacetime_metric_types MT>
void reflect_mirror_ref(typename magik::metric<MT>::params_t mp, const float* x, const float* p, const float* n,
                        float c0, float* p_out, float* c0_out) {
    using namespace magik;
    contravariant_seed_vectors_t seeds;
    const vec4f X{x[0], x[1], x[2], x[3]}, P{p[0], p[1], p[2], p[3]};
    const vec4f u = rest_frame_four_velocity<MT>(X, seeds, vec3f{0.0f, 0.0f, 0.0f}, mp);
    const sym4_t g_inv = metric<MT>::compute_inv_g(X, mp);
    const vec4f rest = global_to_observer_rest_frame<MT>(X, seeds, contract(g_inv, P), u, mp);
    const vec3f incoming = vec3f{rest.x, rest.y, rest.z}.norm();
    const float z = compute_redshift_factor(c0, u, P);
    const vec4f n_rest4 = global_to_observer_rest_frame<MT>(X, seeds, contract(g_inv, vec4f{n[0], n[1], n[2], 0.0f}), u, mp);
    const vec3f n_rest = vec3f{n_rest4.x, n_rest4.y, n_rest4.z}.norm();
    const vec3f facing = vector_dot_product(n_rest, incoming) > 0.0f ? -n_rest : n_rest;
    const vec3f out = vector_reflect(incoming, facing).make_norm();
    const vec4f po = rest_frame_direction_to_global_four_momentum<MT>(X, seeds, out, u, 0.0f, mp);
    p_out[0] = po.x; p_out[1] = po.y; p_out[2] = po.z; p_out[3] = po.t;
    *c0_out = vector_dot_product(u, po) * z;
}

// One camera ray: the oracle's REF32 initial conditions, then per accepted
// step the reference's own solve_step (float, its op order and its powf) and
// the oracle's disk / room / escape / horizon / step-cap tests.
template <e_magik_spacetime_metric_types MT>
orc::RayResult trace_ref(const mgk_scene& s, const orc::SceneConsts& c, uint64_t ray_id,
                         typename magik::metric<MT>::params_t p) {
    using namespace orc;
    MetricParams<float> m = metric_params<float>(s);
    RayInit<float> ri = camera_ray<Fuse::None, float>(s, c, ray_id);
    GState<float> y = ri.y;
    float h = ri.h0;
    uint32_t steps = 0, attempts = 0, evals = 0;
    float c0 = ri.c0;
    Bounce bn;
    bn.ray_id = ray_id;
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
        rs = resolve<Fuse::None, float>(s, m, y, y1, h_taken, &c0, steps, spin, float(c.omega_sign), &bn);
        evals += rs.evals;
        y = rs.y_end;
        h = bn.reflected ? ri.h0 : h_step;
        if (rs.hit.cls != MGK_RAY_ALIVE) break;
    }
    RayResult res{};
    store_result(&res, y, rs.hit, steps, attempts, 0u, evals, bn.count);
    return res;
}

}  // namespace

// evaluate_white_led_spectrum (internal_math.h:2501-2509) in float.
extern "C" __attribute__((visibility("default"))) float ref_white_led(float lambda_nm) {
    return magik::evaluate_white_led_spectrum(lambda_nm);
}

// reflect_mirror_ref for a Kerr (spin a, time-reversed) or Schwarzschild scene.
extern "C" __attribute__((visibility("default"))) int ref_reflect_mirror(const mgk_scene* s, const float* x,
                                                                         const float* p, const float* n, float c0,
                                                                         float* p_out, float* c0_out) {
    const bool tr = s->time_reversed != 0;
    if (s->metric == MGK_METRIC_KERR) {
        magik::kerr_metric::params_t pk{tr, 1.0f, float(tr ? -s->spin : s->spin), float(s->horizon_scalar),
                                        float(s->h_max), float(s->abs_tol), float(s->rel_tol), s->n_max_substep};
        reflect_mirror_ref<e_magik_spacetime_metric_types::KERR>(pk, x, p, n, c0, p_out, c0_out);
        return 0;
    }
    if (s->metric == MGK_METRIC_SCHWARZSCHILD) {
        magik::metric<e_magik_spacetime_metric_types::SCHWARZSCHILD>::params_t ps{};
        ps.time_reversed = tr;
        ps.mass_parameter = 1.0f;
        ps.mass_sign = float(s->mass_sign < 0 ? -1.0 : 1.0);
        ps.event_horizon_scalar = float(s->horizon_scalar);
        reflect_mirror_ref<e_magik_spacetime_metric_types::SCHWARZSCHILD>(ps, x, p, n, c0, p_out, c0_out);
        return 0;
    }
    return 1;
}

// Pixels [first, first + n*stride) of the scene (stride apart) rendered with
// the reference's RKF45 step: mean XYZ per pixel into xyz_out (3 doubles per
// pixel); steps_out (may be NULL) receives the accepted-step total.  Kerr and
// Schwarzschild scenes; returns nonzero otherwise.
extern "C" __attribute__((visibility("default"))) int ref_render_pixels(
    const mgk_scene* s, const mgk_star* stars, uint32_t n_stars, const float* w, uint64_t first_pixel,
    uint32_t n_pixels, uint64_t pixel_stride, double* xyz_out, uint64_t* steps_out, int nthreads) {
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
    std::atomic<uint64_t> stp{0};
    ref_parallel_for(n_pixels, nthreads, [&](uint64_t i) {
        const uint64_t pix = first_pixel + i * pixel_stride;
        float acc[3] = {0, 0, 0};
        uint64_t n = 0;
        for (uint32_t smp = 0; smp < spp; ++smp) {
            RayResult r = s->metric == MGK_METRIC_KERR
                              ? trace_ref<e_magik_spacetime_metric_types::KERR>(*s, c, pix * spp + smp, pk)
                              : trace_ref<e_magik_spacetime_metric_types::SCHWARZSCHILD>(*s, c, pix * spp + smp, ps);
            n += r.steps;
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
        stp += n;
    });
    if (steps_out) *steps_out = stp.load();
    return 0;
}
