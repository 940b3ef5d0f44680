// C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY: loaded by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg through
// ctypes; never by the product).
#include <algorithm>
#include <atomic>
#include <functional>
#include <thread>
#include <vector>

#include "oracle.hpp"
#include "oracle_scene.hpp"

namespace orc {

// ---------------------------------------------- reference trace semantics
// 3x3 matrices with the reference's row-major layout and products
// (internal_math.h:1611-1700, rotate at :1784-1811).
struct M3 { float m[9]; };
inline M3 mat_mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i + 0] * b.m[0 + j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
inline V3<float> mat_vec(const M3& a, V3<float> v) {
    return V3<float>{a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
                     a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z};
}
// mat3f::rotate(alpha, beta, gamma) = R_x(gamma) * R_y(beta) * R_z(alpha).
inline M3 rotate(float alpha, float beta, float gamma) {
    float sa, ca, sb, cb, sg, cg;
    ::sincosf(alpha, &sa, &ca);
    ::sincosf(beta, &sb, &cb);
    ::sincosf(gamma, &sg, &cg);
    M3 mz{{ca, -sa, 0.f, sa, ca, 0.f, 0.f, 0.f, 1.f}};
    M3 my{{cb, 0.f, sb, 0.f, 1.f, 0.f, -sb, 0.f, cb}};
    M3 mx{{1.f, 0.f, 0.f, 0.f, cg, -sg, 0.f, sg, cg}};
    return mat_mul(mat_mul(mx, my), mz);
}

template <class T> inline T length2_3(V3<T> v) { return v.x * v.x + v.y * v.y + v.z * v.z; }

// Float metric params of magik_trace_geodesic (metric_kerr.cuh:137-147,
// metric_schwarzschild.cuh:104-114, metric_minkowski.cuh:42-47).
inline bool make_ref_params(const magik_trace_geodesic_metric_parameters_t& mp,
                            const magik_trace_geodesic_integrator_parameters_t& ip, MetricParams<float>* m,
                            float* length_scale) {
    const float G = 6.67430E-11f, c = 299792458.0f;
    MetricParams<float> p{};
    p.metric = mp.metric_type;
    p.time_reversed = mp.time_reversed;
    p.h_max = 1000.0f;
    p.abs_tol = ip.integrator_absolute_error_tolerance;
    p.rel_tol = ip.integrator_relative_error_tolerance;
    p.n_max = ip.n_integrator_max_substep;
    p.horizon_scalar = mp.event_horizon_scalar;
    if (mp.metric_type == KERR) {
        p.spin = mp.time_reversed ? -mp.kerr_spin : mp.kerr_spin;
        p.mass_sign = 1.0f;
        *length_scale = G * mp.kerr_mass / (c * c);
    } else if (mp.metric_type == SCHWARZSCHILD) {
        p.spin = 0.0f;
        p.mass_sign = mp.schwarzschild_mass > 0.0f ? 1.0f : -1.0f;
        *length_scale = G * std::fabs(mp.schwarzschild_mass) / (c * c);
    } else if (mp.metric_type == MINKOWSKI) {
        p.spin = 0.0f;
        p.mass_sign = 1.0f;
        *length_scale = 1.0f;
    } else {
        return false;
    }
    *m = p;
    return true;
}

// host_trace_geodesic.cu:13-130 restated; K selects how pow() is rounded.
template <Ctl K>
int trace_geodesic_ref(magik_trace_geodesic_container_t* c, const magik_trace_geodesic_inital_conditions_t& ic,
                       const magik_trace_geodesic_metric_parameters_t& mp,
                       const magik_trace_geodesic_integrator_parameters_t& ip) {
    MetricParams<float> m;
    float L;
    if (!make_ref_params(mp, ip, &m, &L)) return MGK_ERROR_UNKNOWN;
    const float cl = 299792458.0f;
    M3 rot = rotate(ic.x_rotation, ic.y_rotation, ic.z_rotation);
    V3<float> dir = mat_vec(rot, V3<float>{0.f, 0.f, -1.f});
    V3<float> bx = mat_vec(rot, V3<float>{1.f, 0.f, 0.f});
    V3<float> by = mat_vec(rot, V3<float>{0.f, 1.f, 0.f});
    V3<float> bz = mat_vec(rot, V3<float>{0.f, 0.f, 1.f});
    V4<float> X{bx.x, bx.y, bx.z, 0.f}, Y{by.x, by.y, by.z, 0.f}, Z{bz.x, bz.y, bz.z, 0.f};
    float squared_norm;
    V3<float> lpv{ic.local_proper_velocity_x, ic.local_proper_velocity_y, ic.local_proper_velocity_z};
    if (ic.test_particle_type == MGK_MASSIVE) {
        squared_norm = -1.0f;
        float s = ic.massive_particle_speed / cl;
        dir = V3<float>{dir.x * s, dir.y * s, dir.z * s};
    } else {
        squared_norm = 0.0f;
    }
    V4<float> x0{ic.spatial_position_x / L, ic.spatial_position_y / L, ic.spatial_position_z / L, 0.0f / (L / cl)};
    // rest_frame_four_velocity (relativity_utilities.cuh:163-173)
    Sym4<float> g = compute_g(x0, m);
    V4<float> u_ref = reference_observer(x0, m);
    Tetrad<float> e = build_tetrad(g, X, Y, Z, u_ref);
    V3<float> w{lpv.x / cl, lpv.y / cl, lpv.z / cl};
    if (m.time_reversed) w = V3<float>{-w.x, -w.y, -w.z};
    V4<float> u = local_to_global(e, V4<float>{w.x, w.y, w.z, std::sqrt(length2_3(w) - -1.0f)});
    // rest_frame_direction_to_global_four_momentum (relativity_utilities.cuh:186-195), identity seeds
    V4<float> IX{1, 0, 0, 0}, IY{0, 1, 0, 0}, IZ{0, 0, 1, 0};
    Tetrad<float> e2 = build_tetrad(g, IX, IY, IZ, u);
    V3<float> d{dir.x / L, dir.y / L, dir.z / L};
    V4<float> p_up = local_to_global(e2, V4<float>{d.x, d.y, d.z, std::sqrt(length2_3(d) - squared_norm)});
    V4<float> p0 = contract(g, p_up);

    GState<float> y{x0, p0};
    GState<float> ys = rhs<Fuse::None>(y, m);
    auto put = [&](uint32_t i, const GState<float>& s, const GState<float>& ds, float contraction, float aff,
                   float dh) {
        magik_trace_geodesic_step_t& st = c->steps[i];
        st.four_position[0] = s.x.x; st.four_position[1] = s.x.y; st.four_position[2] = s.x.z; st.four_position[3] = s.x.t;
        st.four_momentum[0] = s.p.x; st.four_momentum[1] = s.p.y; st.four_momentum[2] = s.p.z; st.four_momentum[3] = s.p.t;
        st.moment_derivative[0] = ds.p.x; st.moment_derivative[1] = ds.p.y;
        st.moment_derivative[2] = ds.p.z; st.moment_derivative[3] = ds.p.t;
        st.four_vector_contraction = contraction;
        st.affine_parameter = aff;
        st.delta_affine_parameter = dh;
    };
    float contraction = dot4(u, p0);
    float h = m.metric == MINKOWSKI ? 1000.0f : 1.0f;
    float aff = 0.0f;
    c->n_written = 0;
    put(0, y, ys, contraction, aff, h);
    c->n_written = 1;
    while (c->n_written < c->n_allocated_step) {
        StepOut<float> so = solve_step<Fuse::None, K, float>(y, h, m);
        ys = rhs<Fuse::None>(so.y1, m);
        aff = aff + so.h_taken;
        h = so.h_next;
        y = so.y1;
        put(c->n_written, y, ys, contraction, aff, h);
        c->n_written++;
        if (in_domain(y.x, m)) break;
    }
    for (uint32_t i = 0; i < c->n_written; ++i)
        for (int k = 0; k < 4; ++k) c->steps[i].four_position[k] *= L;
    return MGK_SUCCESS;
}

// ------------------------------------------------------- op counting
// A scalar that counts source-level operations (+, -, *, / and sqrt = 1,
// fma = 2), used to freeze the FLOP-per-attempt figures of the roofline.
struct CF {
    double v;
    CF() = default;
    constexpr CF(double x) : v(x) {}
};
static thread_local uint64_t g_ops = 0;
inline CF operator+(CF a, CF b) { ++g_ops; return CF{a.v + b.v}; }
inline CF operator-(CF a, CF b) { ++g_ops; return CF{a.v - b.v}; }
inline CF operator*(CF a, CF b) { ++g_ops; return CF{a.v * b.v}; }
inline CF operator/(CF a, CF b) { ++g_ops; return CF{a.v / b.v}; }
inline CF operator-(CF a) { return CF{-a.v}; }
inline bool operator>(CF a, CF b) { return a.v > b.v; }
inline bool operator<(CF a, CF b) { return a.v < b.v; }
inline CF sqrt(CF a) { ++g_ops; return CF{std::sqrt(a.v)}; }
inline CF fma(CF a, CF b, CF c) { g_ops += 2; return CF{std::fma(a.v, b.v, c.v)}; }
inline CF fmax(CF a, CF b) { return CF{std::fmax(a.v, b.v)}; }
inline CF fabs(CF a) { return CF{std::fabs(a.v)}; }
// Fehlberg coefficients as plain constants (their evaluation is not counted).
template <> struct Fehlberg<CF> {
    static constexpr CF a21 = CF(1.0 / 4), a31 = CF(3.0 / 32), a32 = CF(9.0 / 32);
    static constexpr CF a41 = CF(1932.0 / 2197), a42 = CF(7200.0 / 2197), a43 = CF(7296.0 / 2197);
    static constexpr CF a51 = CF(439.0 / 216), a52 = CF(8.0), a53 = CF(3680.0 / 513), a54 = CF(845.0 / 4104);
    static constexpr CF a61 = CF(8.0 / 27), a62 = CF(2.0), a63 = CF(3544.0 / 2565), a64 = CF(1859.0 / 4104),
                        a65 = CF(11.0 / 40);
    static constexpr CF b1 = CF(16.0 / 135), b3 = CF(6656.0 / 12825), b4 = CF(28561.0 / 56430), b5 = CF(9.0 / 50),
                        b6 = CF(2.0 / 55);
    static constexpr CF e1 = CF(-1.0 / 360), e3 = CF(128.0 / 4275), e4 = CF(2197.0 / 75240), e5 = CF(1.0 / 50),
                        e6 = CF(2.0 / 55);
};
}  // namespace orc

using namespace orc;

extern "C" {

int orc_trace_geodesic(magik_trace_geodesic_container_t* c, magik_trace_geodesic_inital_conditions_t ic,
                       magik_trace_geodesic_metric_parameters_t mp,
                       magik_trace_geodesic_integrator_parameters_t ip, int pow_in_double) {
    if (!c || !c->steps) return MGK_ERROR_INVALID_POINTER;
    if (c->capacity != sizeof(magik_trace_geodesic_step_t) * uint64_t(c->n_allocated_step))
        return MGK_ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH;
    if (c->n_allocated_step == 0) return MGK_ERROR_INVALID_ARGUMENT;
    return pow_in_double ? trace_geodesic_ref<Ctl::RefD>(c, ic, mp, ip) : trace_geodesic_ref<Ctl::Ref>(c, ic, mp, ip);
}

// The benchmark workload's scene: the Kerr a = 0.9 view at r = 50 M and
// 75 degrees, 1920x1080x16, 32 bins, rtol = atol = 1e-7, MIXED.  A
// restatement of the library's defaults for the CPU legs that must not load
// the library; tests check that both fill the same bytes.
double orc_isco_radius(double a) {
    // Bardeen, Press and Teukolsky (1972), prograde orbits, M = 1.
    const double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
    const double z2 = std::sqrt(3.0 * a * a + z1 * z1);
    return 3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

void orc_scene_defaults(mgk_scene* s) {
    std::memset(s, 0, sizeof(*s));
    s->metric = MGK_METRIC_KERR;
    s->precision = MGK_PRECISION_MIXED;
    s->time_reversed = 1;
    s->n_max_substep = 56;
    s->spin = 0.9;
    s->mass_sign = 1.0;
    s->horizon_scalar = 1.01;
    s->abs_tol = 1e-7;
    s->rel_tol = 1e-7;
    s->h_max = 1000.0;
    s->max_steps = 10000;
    s->n_bins = 32;
    s->escape_radius = 1000.0;
    s->disk_r_in = orc_isco_radius(0.9);
    s->disk_r_out = 20.0;
    s->disk_T_in = 1.0e4;
    s->cam_r = 50.0;
    s->cam_incl_rad = 75.0 * M_PI / 180.0;
    s->sensor_diag_mm = 24.0;
    s->focal_length_mm = 12.0 / std::tan(30.0 * M_PI / 180.0);
    s->width = 1920;
    s->height = 1080;
    s->spp = 16;
    s->seed = 0x5EEDull;
    s->lambda_min_nm = 380.0;
    s->lambda_max_nm = 780.0;
    s->star_radius_rad = 2.0e-3;
    s->spectral_mode = MGK_SPECTRAL_BINS;
    s->iso = 500.0;
    s->fps = 24.0;
    s->shutter_angle_deg = 180.0;
    s->redistribution_sigma_nm = 10.0;
    s->room_on = 0;
    s->room_reflection_limit = 10;
    const double lo[3] = {-40.0, -20.0, -40.0}, hi[3] = {40.0, 20.0, 40.0};
    const double llo[3] = {-20.0, 19.0, -20.0}, lhi[3] = {20.0, 21.0, 20.0};
    for (int a = 0; a < 3; ++a) {
        s->room_min[a] = lo[a]; s->room_max[a] = hi[a];
        s->light_min[a] = llo[a]; s->light_max[a] = lhi[a];
    }
    s->light_scale = 7.0e5;
}

// The seeded star catalogue (a restatement of the library's): directions
// uniform on the sphere, magnitudes uniform in [0, 10] relative to a 1e4 K
// blackbody at 550 nm, temperatures uniform in 3000-30000 K.
void orc_star_catalog(uint64_t seed, uint32_t n, mgk_star* out) {
    auto planck = [](double nm, double T) {
        const double h = 6.62607015E-34, c = 299792458.0, kb = 1.380649E-23;
        const double wl = nm * 1e-9;
        return (2.0 * h * c * c / std::pow(wl, 5)) / std::expm1(h * c / (wl * kb * T));
    };
    const double ref = planck(550.0, 1.0e4);
    for (uint32_t i = 0; i < n; ++i) {
        const double u0 = rng_unit(seed, 0x57A2u, i, 0), u1 = rng_unit(seed, 0x57A2u, i, 1);
        const double u2 = rng_unit(seed, 0x57A2u, i, 2), u3 = rng_unit(seed, 0x57A2u, i, 3);
        const double y = 2.0 * u0 - 1.0, ph = 2.0 * M_PI * u1, r = std::sqrt(std::max(0.0, 1.0 - y * y));
        const double T = 3000.0 + 27000.0 * u3;
        mgk_star& st = out[i];
        std::memset(&st, 0, sizeof(st));
        st.dir[0] = float(r * std::cos(ph));
        st.dir[1] = float(y);
        st.dir[2] = float(r * std::sin(ph));
        st.amplitude = float(std::pow(10.0, -0.4 * (10.0 * u2)) * ref / planck(550.0, T));
        st.temperature = float(T);
    }
}

int orc_scene_constants(const mgk_scene* s, double* out) {
    SceneConsts c = scene_consts(*s);
    int k = 0;
    for (int i = 0; i < 4; ++i) out[k++] = c.cam_pos[i];
    for (int i = 0; i < 4; ++i) out[k++] = c.u_obs[i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[k++] = c.M[i][j];
    out[k++] = c.pix_a; out[k++] = c.pix_b; out[k++] = c.pix_c; out[k++] = c.pix_d;
    out[k++] = c.r_plus; out[k++] = c.spin_t; out[k++] = c.omega_sign;
    while (k < 32) out[k++] = 0.0;
    return 0;
}

static void parallel_for(uint64_t n, int nthreads, const std::function<void(uint64_t)>& fn) {
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

int orc_trace_rays(const mgk_scene* s, uint64_t first, uint32_t n, mgk_ray_result* out, int nthreads) {
    SceneConsts c = scene_consts(*s);
    parallel_for(n, nthreads, [&](uint64_t i) {
        RayResult r = trace_ray(*s, c, first + i);
        static_assert(sizeof(RayResult) == sizeof(mgk_ray_result), "layout");
        std::memcpy(&out[i], &r, sizeof(r));
    });
    return 0;
}

// Spectrum -> XYZ of given ray results (shading stage alone).
int orc_shade_rays(const mgk_scene* s, const mgk_star* stars, uint32_t n_stars, const float* w, uint32_t n,
                   const mgk_ray_result* in, uint64_t first_ray, const float* icdf, double* xyz_out, int nthreads) {
    if (s->spectral_mode == MGK_SPECTRAL_SAMPLED && !icdf) return 1;
    StarIndex idx;
    idx.build(stars, n_stars, s->star_radius_rad);
    const uint32_t nb = s->n_bins;
    double dl = (s->lambda_max_nm - s->lambda_min_nm) / nb;
    parallel_for(n, nthreads, [&](uint64_t i) {
        const mgk_ray_result& r = in[i];
        double out3[3];
        if (s->precision == MGK_PRECISION_F64) {
            double lam[MGK_MAX_BINS], spec[MGK_MAX_BINS];
            for (uint32_t k = 0; k < nb; ++k) lam[k] = s->lambda_min_nm + (k + 0.5) * dl;
            Hit<double> h; h.cls = r.cls; h.z = r.z; h.r_hit = r.r_hit;
            h.dir[0] = r.dir[0]; h.dir[1] = r.dir[1]; h.dir[2] = r.dir[2];
            if (s->spectral_mode == MGK_SPECTRAL_SAMPLED) sampled_spectrum<double>(*s, &idx, h, first_ray + i, icdf, spec);
            else ray_spectrum<double>(*s, &idx, h, lam, spec);
            spectrum_xyz<double>(nb, spec, w, out3);
        } else {
            float lam[MGK_MAX_BINS], spec[MGK_MAX_BINS], o[3];
            for (uint32_t k = 0; k < nb; ++k) lam[k] = float(s->lambda_min_nm + (k + 0.5) * dl);
            Hit<float> h; h.cls = r.cls; h.z = float(r.z); h.r_hit = float(r.r_hit);
            h.dir[0] = float(r.dir[0]); h.dir[1] = float(r.dir[1]); h.dir[2] = float(r.dir[2]);
            if (s->spectral_mode == MGK_SPECTRAL_SAMPLED) sampled_spectrum<float>(*s, &idx, h, first_ray + i, icdf, spec);
            else ray_spectrum<float>(*s, &idx, h, lam, spec);
            spectrum_xyz<float>(nb, spec, w, o);
            out3[0] = o[0]; out3[1] = o[1]; out3[2] = o[2];
        }
        xyz_out[3 * i + 0] = out3[0]; xyz_out[3 * i + 1] = out3[1]; xyz_out[3 * i + 2] = out3[2];
    });
    return 0;
}

// Full pipeline for pixels first_pixel + i * pixel_stride, i < n_pixels:
// trace every sample, shade, average.  xyz_out: 3 doubles per pixel.
// attempts_out / steps_out (may be NULL) receive the RKF45 attempt and
// accepted-step totals.
int orc_render_pixels(const mgk_scene* s, const mgk_star* stars, uint32_t n_stars, const float* w,
                      uint64_t first_pixel, uint32_t n_pixels, uint64_t pixel_stride, const float* icdf,
                      double* xyz_out, uint64_t* attempts_out, uint64_t* steps_out, int nthreads) {
    if (s->spectral_mode == MGK_SPECTRAL_SAMPLED && !icdf) return 1;
    SceneConsts c = scene_consts(*s);
    StarIndex idx;
    idx.build(stars, n_stars, s->star_radius_rad);
    const uint32_t nb = s->n_bins, spp = s->spp;
    const double dl = (s->lambda_max_nm - s->lambda_min_nm) / nb;
    std::atomic<uint64_t> att{0}, stp{0};
    parallel_for(n_pixels, nthreads, [&](uint64_t i) {
        uint64_t pix = first_pixel + i * pixel_stride;
        double acc[3] = {0, 0, 0};
        float accf[3] = {0, 0, 0};
        uint64_t a = 0, n = 0;
        for (uint32_t smp = 0; smp < spp; ++smp) {
            RayResult r = trace_ray(*s, c, pix * spp + smp);
            a += r.attempts;
            n += r.steps;
            if (s->precision == MGK_PRECISION_F64) {
                double lam[MGK_MAX_BINS], spec[MGK_MAX_BINS], o[3];
                for (uint32_t k = 0; k < nb; ++k) lam[k] = s->lambda_min_nm + (k + 0.5) * dl;
                Hit<double> h; h.cls = r.cls; h.z = r.z; h.r_hit = r.r_hit;
                h.dir[0] = r.dir[0]; h.dir[1] = r.dir[1]; h.dir[2] = r.dir[2];
                if (s->spectral_mode == MGK_SPECTRAL_SAMPLED)
                    sampled_spectrum<double>(*s, &idx, h, pix * spp + smp, icdf, spec);
                else ray_spectrum<double>(*s, &idx, h, lam, spec);
                spectrum_xyz<double>(nb, spec, w, o);
                for (int k = 0; k < 3; ++k) acc[k] += o[k];
            } else {
                float lam[MGK_MAX_BINS], spec[MGK_MAX_BINS], o[3];
                for (uint32_t k = 0; k < nb; ++k) lam[k] = float(s->lambda_min_nm + (k + 0.5) * dl);
                Hit<float> h; h.cls = r.cls; h.z = float(r.z); h.r_hit = float(r.r_hit);
                h.dir[0] = float(r.dir[0]); h.dir[1] = float(r.dir[1]); h.dir[2] = float(r.dir[2]);
                if (s->spectral_mode == MGK_SPECTRAL_SAMPLED)
                    sampled_spectrum<float>(*s, &idx, h, pix * spp + smp, icdf, spec);
                else ray_spectrum<float>(*s, &idx, h, lam, spec);
                spectrum_xyz<float>(nb, spec, w, o);
                for (int k = 0; k < 3; ++k) accf[k] += o[k];
            }
        }
        att += a;
        stp += n;
        for (int k = 0; k < 3; ++k)
            xyz_out[3 * i + k] = s->precision == MGK_PRECISION_F64 ? acc[k] / spp : double(accf[k] / float(spp));
    });
    if (attempts_out) *attempts_out = att.load();
    if (steps_out) *steps_out = stp.load();
    return 0;
}

// Source-level operation counts: out[0] = RHS, out[1] = one RKF45 attempt
// (6 RHS + stage combinations + error + norm + proposal).
int orc_count_ops(int metric, int fused, uint64_t* out) {
    MetricParams<CF> m{};
    m.metric = metric; m.spin = CF{0.5}; m.mass_sign = CF{1.0}; m.horizon_scalar = CF{1.01};
    m.h_max = CF{1000.0}; m.abs_tol = CF{1e-7}; m.rel_tol = CF{1e-7}; m.n_max = 1;
    GState<CF> y{V4<CF>{CF{3}, CF{4}, CF{5}, CF{0}}, V4<CF>{CF{0.1}, CF{0.2}, CF{0.3}, CF{-1}}};
    g_ops = 0;
    if (fused) (void)rhs<Fuse::Fma, CF>(y, m); else (void)rhs<Fuse::None, CF>(y, m);
    out[0] = g_ops;
    g_ops = 0;
    GState<CF> y1, k[6];
    if (fused) {
        rkf45_attempt<Fuse::Fma, CF>(y, CF{1}, m, &y1, k);
        GState<CF> e = rkf45_error<Fuse::Fma, CF>(CF{1}, k);
        CF err = rms_error<Fuse::Fma, CF>(e, y, y1, m.abs_tol, m.rel_tol);
        (void)(CF{0.9} * CF{1} * (CF{1} / err));  // proposal: 0.9*h*pow(1/err, 0.2) with pow = 1
        ++g_ops;
    } else {
        rkf45_attempt<Fuse::None, CF>(y, CF{1}, m, &y1, k);
        GState<CF> e = rkf45_error<Fuse::None, CF>(CF{1}, k);
        CF err = rms_error<Fuse::None, CF>(e, y, y1, m.abs_tol, m.rel_tol);
        (void)(CF{0.9} * CF{1} * (CF{1} / err));
        ++g_ops;
    }
    out[1] = g_ops;
    return 0;
}

// Room scene parts, for the CPU tests: the chord event (double), the
// white-LED spectrum (double) and one wall reflection of a float state.
int orc_room_event(const mgk_scene* s, const double* p0, const double* p1, double* t, int* axis_side_light) {
    RoomEvent<double> ev = room_event<double>(*s, V4<double>{p0[0], p0[1], p0[2], 0.0},
                                              V4<double>{p1[0], p1[1], p1[2], 0.0});
    *t = ev.t;
    axis_side_light[0] = ev.axis; axis_side_light[1] = ev.side; axis_side_light[2] = ev.light ? 1 : 0;
    return 0;
}

double orc_white_led(double lambda_nm) { return white_led<double>(lambda_nm); }

int orc_reflect_wall(const mgk_scene* s, const float* x, const float* p, int axis, int side, float c0,
                     uint32_t bounce, uint64_t ray_id, float* x_out, float* p_out, float* c0_out) {
    MetricParams<float> m = metric_params<float>(*s);
    GState<float> ys;
    ys.x = V4<float>{x[0], x[1], x[2], x[3]};
    ys.p = V4<float>{p[0], p[1], p[2], p[3]};
    float c = c0;
    GState<float> o = reflect_wall<float>(*s, m, axis, side, ys, &c, bounce, ray_id);
    x_out[0] = o.x.x; x_out[1] = o.x.y; x_out[2] = o.x.z; x_out[3] = o.x.t;
    p_out[0] = o.p.x; p_out[1] = o.p.y; p_out[2] = o.p.z; p_out[3] = o.p.t;
    *c0_out = c;
    return 0;
}

}  // extern "C"
