// C ABI of libmgk.so: context and arena, scene validation, host utilities,
// the chunked render pipeline and the reference-compatible trace entry point.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "dev_scene.cuh"
#include "internal.h"

using namespace mgk;

struct mgk_context {
    int device = 0;
    int sm_count = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    void* stage = nullptr;            // device staging of mgk_render_host's inputs and film
    size_t stage_bytes = 0;
    std::vector<cudaEvent_t> events;  // pairs around the integrator launches
    std::string last_error = "no error";
};

namespace {

constexpr uint32_t kMaxChunkRays = 1u << 25;

mgk_result cuda_fail(mgk_context* ctx, cudaError_t e, const char* what) {
    if (ctx) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
        ctx->last_error = buf;
    }
    return MGK_ERROR_CUDA;
}
#define MGK_CUDA(ctx, call)                                         \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_fail((ctx), _e, #call);  \
    } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

mgk_result ensure_arena(mgk_context* ctx, size_t bytes) {
    if (ctx->arena_bytes >= bytes) return MGK_SUCCESS;
    if (ctx->arena) {
        cudaError_t e = cudaFree(ctx->arena);
        ctx->arena = nullptr;
        ctx->arena_bytes = 0;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaFree(arena)");
    }
    cudaError_t e = cudaMalloc(&ctx->arena, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->arena = nullptr;
        cuda_fail(ctx, e, "cudaMalloc(arena)");
        return MGK_ERROR_DEVICE_OUT_OF_MEMORY;
    }
    ctx->arena_bytes = bytes;
    return MGK_SUCCESS;
}

mgk_result validate(const mgk_scene* s) {
    if (!s) return MGK_ERROR_INVALID_POINTER;
    if (!metric_supported(s->metric)) return MGK_ERROR_UNKNOWN_METRIC;
    if (s->precision < 0 || s->precision > 2) return MGK_UNKNOWN_ENUM_TYPE;
    if (s->n_max_substep < 1 || !(s->abs_tol > 0.0) || !(s->rel_tol >= 0.0) || !(s->h_max > 0.0))
        return MGK_ERROR_INVALID_ARGUMENT;
    if (s->max_steps < 1 || s->n_bins < 1 || s->n_bins > MGK_MAX_BINS) return MGK_ERROR_INVALID_ARGUMENT;
    if (s->width < 1 || s->height < 1 || s->spp < 1) return MGK_ERROR_INVALID_ARGUMENT;
    if (uint64_t(s->sample_offset) + s->spp > (1ull << 32)) return MGK_ERROR_INVALID_ARGUMENT;
    if (uint64_t(s->width) * s->height >= (1ull << 32)) return MGK_ERROR_INVALID_ARGUMENT;
    if (!(s->escape_radius > 0.0) || !(s->lambda_max_nm > s->lambda_min_nm) || !(s->lambda_min_nm > 0.0))
        return MGK_ERROR_INVALID_ARGUMENT;
    if (s->disk_r_out > 0.0 && !(s->disk_r_in > 0.0 && s->disk_r_in < s->disk_r_out)) return MGK_ERROR_INVALID_ARGUMENT;
    if (!(s->focal_length_mm > 0.0) || !(s->sensor_diag_mm > 0.0) || !(s->cam_explicit || s->cam_r > 0.0))
        return MGK_ERROR_INVALID_ARGUMENT;
    if (s->cam_explicit > 1u) return MGK_ERROR_INVALID_ARGUMENT;
    // the camera position (M)
    double cam[3] = {0.0, s->cam_r * std::cos(s->cam_incl_rad), s->cam_r * std::sin(s->cam_incl_rad)};
    if (s->cam_explicit) {
        // finite position and velocity, orthonormal axes, outside the capture radius
        const double* A = s->cam_axes;
        for (int i = 0; i < 3; ++i) {
            cam[i] = s->cam_pos[i];
            if (!std::isfinite(cam[i]) || !std::isfinite(s->cam_velocity[i])) return MGK_ERROR_INVALID_ARGUMENT;
            for (int j = 0; j < 3; ++j) {
                const double d = A[3 * i] * A[3 * j] + A[3 * i + 1] * A[3 * j + 1] + A[3 * i + 2] * A[3 * j + 2];
                if (!(std::fabs(d - (i == j ? 1.0 : 0.0)) <= 1e-6)) return MGK_ERROR_INVALID_ARGUMENT;
            }
        }
        bool outside = true;
        with_metric(s->metric, [&](auto mt) {
            using MT = decltype(mt);
            if (!MT::has_horizon) return;
            const double a = MT::spin(*s);
            const double R = cam[0] * cam[0] + cam[1] * cam[1] + cam[2] * cam[2] - a * a;
            const double r = std::sqrt(0.5 * R + 0.5 * std::sqrt(R * R + 4.0 * a * a * cam[1] * cam[1]));
            outside = r > MT::outer_horizon(*s) * s->horizon_scalar;
        });
        if (!outside) return MGK_ERROR_INVALID_ARGUMENT;
    }
    if (!(s->star_radius_rad > 0.0 && s->star_radius_rad <= 0.02)) return MGK_ERROR_INVALID_ARGUMENT;
    if (s->spectral_mode > MGK_SPECTRAL_SAMPLED) return MGK_UNKNOWN_ENUM_TYPE;
    if (s->spectral_mode == MGK_SPECTRAL_SAMPLED &&
        !(s->iso > 0.0 && s->fps > 0.0 && s->shutter_angle_deg > 0.0 && s->redistribution_sigma_nm > 0.0))
        return MGK_ERROR_INVALID_ARGUMENT;
    if (s->room_on) {
        // both boxes proper, the camera inside the room and outside the light
        // (rays start inside the room: kernel_intersect.cu:81-100 takes the
        // room's far face)
        for (int a = 0; a < 3; ++a)
            if (!(s->room_min[a] < s->room_max[a] && s->light_min[a] < s->light_max[a]) ||
                !std::isfinite(s->room_min[a]) || !std::isfinite(s->room_max[a]) ||
                !std::isfinite(s->light_min[a]) || !std::isfinite(s->light_max[a]))
                return MGK_ERROR_INVALID_ARGUMENT;
        if (!(s->light_scale >= 0.0 && std::isfinite(s->light_scale)) || s->room_reflection_limit > 1024u)
            return MGK_ERROR_INVALID_ARGUMENT;
        const double* q = cam;
        bool in_room = true, in_light = true;
        for (int a = 0; a < 3; ++a) {
            in_room = in_room && q[a] > s->room_min[a] && q[a] < s->room_max[a];
            in_light = in_light && q[a] >= s->light_min[a] && q[a] <= s->light_max[a];
        }
        if (!in_room || in_light) return MGK_ERROR_INVALID_ARGUMENT;
    }
    // MIXED evaluates the RHS with one float reciprocal of ~r^9, finite below
    // r ~ 1.9e4; a ray moves at most about h_max past the escape radius
    if (s->precision == MGK_PRECISION_MIXED && s->escape_radius + 2.0 * s->h_max > 1.5e4)
        return MGK_ERROR_INVALID_ARGUMENT;
    return MGK_SUCCESS;
}

// --------------------------------------------------------- CIE 1931 data
// The CIE 1931 2-degree standard observer at 1 nm over 360-830 nm, the
// published standard data the reference tabulates
// (color_matching_functions.cuh:22-28).
const float kCie1931[471][3] = {
#include "cie1931_2deg.inc"
};
constexpr uint32_t kCieEntries = 471;
constexpr float kCieMinNm = 360.0f, kCieMaxNm = 830.0f;

// ------------------------------------------- CIE 1931 (analytic, opt-in)
// Multi-lobe piecewise-Gaussian fit of the CIE 1931 2-degree observer from
// Wyman, Sloan and Shirley, "Simple Analytic Approximations to the CIE XYZ
// Color Matching Functions", JCGT 2(2), 2013.
double lobe(double l, double mu, double s1, double s2) {
    double t = (l - mu) / (l < mu ? s1 : s2);
    return std::exp(-0.5 * t * t);
}
void cmf_1931_fit(double l, double out[3]) {
    out[0] = 1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) - 0.065 * lobe(l, 501.1, 20.4, 26.2);
    out[1] = 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1);
    out[2] = 1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8);
}

double planck_d(double nm, double T) {
    const double h = 6.62607015E-34, c = 299792458.0, kb = 1.380649E-23;
    double wl = nm * 1e-9;
    return (2.0 * h * c * c / std::pow(wl, 5)) / std::expm1(h * c / (wl * kb * T));
}

// ------------------------------------------------------------- star grid
uint32_t grid_n(double radius) {
    // A cell spans 4 star radii at a face centre and 4/3 at a corner, so the
    // box of a star (2.5 radii across) covers at most 3 x 3 cells per face.
    double n = 0.125 * M_PI / radius;
    if (n > 256.0) n = 256.0;
    if (n < 8.0) n = 8.0;
    return uint32_t(n);
}

}  // namespace

namespace mgk {
// The tabulated CIE 1931 functions at `nm`, interpolated linearly between
// the 1 nm entries in float and clamped to the table's ends, in the order of
// operations of sample_equidistant_spectral_data and lerp
// (color_matching_functions.cuh:35-44, internal_math.h:2040-2043).
void cie1931_sample(float nm, float out[3]) {
    const float spacing = (kCieMaxNm - kCieMinNm) / float(kCieEntries - 1);
    const float fi = std::fmin(std::fmax((nm - kCieMinNm) / spacing, 0.0f), float(kCieEntries - 1));
    const uint32_t lower = uint32_t(std::fmin(float(uint32_t(fi)), float(kCieEntries - 2)));
    const float t = fi - float(lower);
    for (int c = 0; c < 3; ++c) out[c] = (kCie1931[lower][c] * (1.0f - t)) + (kCie1931[lower + 1][c] * t);
}

// CIE inverse CDF table of the sampled spectral mode, as the reference builds
// it (host_color_utilities.cuh:188-233) in float: the tabulated functions
// resampled at 471 points over [lmin, lmax], s = x + y + z, a trapezoid CDF
// with a floor of 5 % of the mean of s per unit wavelength, normalised,
// inverted at 256 equidistant probabilities by linear interpolation.  With
// `fit` the analytic functions stand in for the table.
void cmf_inverse_cdf_table(double lmin_d, double lmax_d, float* out, bool fit) {
    const uint32_t n = kCieEntries - 1;
    const float lmin = float(lmin_d), lmax = float(lmax_d);
    const float dl = (lmax - lmin) / float(n);
    std::vector<float> s(kCieEntries);
    for (uint32_t i = 0; i < kCieEntries; ++i) {
        const float nm = lmin + float(i) * dl;
        float c[3];
        if (fit) {
            double d[3];
            cmf_1931_fit(double(nm), d);
            c[0] = float(d[0]); c[1] = float(d[1]); c[2] = float(d[2]);
        } else {
            cie1931_sample(nm, c);
        }
        s[i] = (c[0] + c[1]) + c[2];
    }
    float mean = 0.0f;
    for (uint32_t i = 0; i < kCieEntries; ++i) mean += s[i];
    mean /= float(kCieEntries);
    const float floor = 0.05f * mean;
    std::vector<float> cdf(n + 1, 0.0f);
    for (uint32_t i = 0; i < n; ++i) cdf[i + 1] = cdf[i] + (0.5f * (s[i] + s[i + 1]) + floor) * dl;
    const float total = cdf[n];
    for (uint32_t j = 0; j <= n; ++j) cdf[j] /= total;
    uint32_t j = 0;
    for (uint32_t k = 0; k < MGK_CMF_ICDF_ENTRIES; ++k) {
        const float u = float(k) / float(MGK_CMF_ICDF_ENTRIES - 1);
        while (j < n - 1 && cdf[j + 1] < u) ++j;
        const float tt = (u - cdf[j]) / std::fmax(cdf[j + 1] - cdf[j], 1e-12f);
        out[k] = lmin + (float(j) + tt) * dl;
    }
}

}  // namespace mgk

constexpr int kStarBox = 4;

// Cells whose area the disc of a star can reach: the bounding box, per cube
// face, of 16 points on a circle of 1.25 star radii around the star (plus the
// centre), each projected onto every face it lies in front of.
__device__ __forceinline__ void star_faces_box(const mgk_star& st, float rad, uint32_t n, int box[6][4], unsigned& faces) {
    float d[3] = {st.dir[0], st.dir[1], st.dir[2]};
    // tangent basis at the star
    float a[3] = {fabsf(d[0]) < 0.9f ? 1.f : 0.f, fabsf(d[0]) < 0.9f ? 0.f : 1.f, 0.f};
    float t1[3] = {d[1] * a[2] - d[2] * a[1], d[2] * a[0] - d[0] * a[2], d[0] * a[1] - d[1] * a[0]};
    float l1 = sqrtf(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (int i = 0; i < 3; ++i) t1[i] /= l1;
    float t2[3] = {d[1] * t1[2] - d[2] * t1[1], d[2] * t1[0] - d[0] * t1[2], d[0] * t1[1] - d[1] * t1[0]};
    faces = 0;
    for (int f = 0; f < 6; ++f) { box[f][0] = box[f][1] = 1 << 30; box[f][2] = box[f][3] = -1; }
    float ang = 1.25f * rad;
    for (int k = 0; k <= 16; ++k) {
        float p[3];
        if (k == 16) { p[0] = d[0]; p[1] = d[1]; p[2] = d[2]; }
        else {
            float ph = 6.2831853f * float(k) / 16.f, c = cosf(ang), s = sinf(ang);
            float cp = cosf(ph), sp = sinf(ph);
            for (int i = 0; i < 3; ++i) p[i] = c * d[i] + s * (cp * t1[i] + sp * t2[i]);
        }
        uint32_t cell = cube_cell(p[0], p[1], p[2], n);
        faces |= 1u << (cell / (n * n));
    }
    for (int k = 0; k <= 16; ++k) {
        float p[3];
        if (k == 16) { p[0] = d[0]; p[1] = d[1]; p[2] = d[2]; }
        else {
            float ph = 6.2831853f * float(k) / 16.f, c = cosf(ang), s = sinf(ang);
            float cp = cosf(ph), sp = sinf(ph);
            for (int i = 0; i < 3; ++i) p[i] = c * d[i] + s * (cp * t1[i] + sp * t2[i]);
        }
        for (int f = 0; f < 6; ++f) {
            if (!(faces & (1u << f))) continue;
            int axis = f >> 1;
            float sgn = (f & 1) ? -1.f : 1.f;
            float m = sgn * p[axis];
            if (m <= 0.f) continue;
            float u = axis == 0 ? p[1] : p[0];
            float v = axis == 2 ? p[1] : p[2];
            int iu = int(floorf((u / m + 1.f) * 0.5f * float(n)));
            int iv = int(floorf((v / m + 1.f) * 0.5f * float(n)));
            iu = iu < 0 ? 0 : (iu >= int(n) ? int(n) - 1 : iu);
            iv = iv < 0 ? 0 : (iv >= int(n) ? int(n) - 1 : iv);
            box[f][0] = min(box[f][0], iu); box[f][1] = min(box[f][1], iv);
            box[f][2] = max(box[f][2], iu); box[f][3] = max(box[f][3], iv);
        }
    }
    // memory guard: at most kStarBox x kStarBox cells per face (the grid size
    // keeps real boxes at 3 x 3)
    for (int f = 0; f < 6; ++f) {
        if (box[f][2] - box[f][0] >= kStarBox) box[f][2] = box[f][0] + kStarBox - 1;
        if (box[f][3] - box[f][1] >= kStarBox) box[f][3] = box[f][1] + kStarBox - 1;
    }
}

__global__ void k_grid_count(const mgk_star* stars, uint32_t n_stars, float rad, uint32_t n, uint32_t* counts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_stars) return;
    int box[6][4];
    unsigned faces;
    star_faces_box(stars[i], rad, n, box, faces);
    for (int f = 0; f < 6; ++f) {
        if (!(faces & (1u << f)) || box[f][2] < 0) continue;
        for (int v = box[f][1]; v <= box[f][3]; ++v)
            for (int u = box[f][0]; u <= box[f][2]; ++u) atomicAdd(&counts[(f * n + v) * n + u], 1u);
    }
}

__global__ void k_grid_fill(const mgk_star* stars, uint32_t n_stars, float rad, uint32_t n, const uint32_t* start,
                            uint32_t* cursor, uint32_t* list) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_stars) return;
    int box[6][4];
    unsigned faces;
    star_faces_box(stars[i], rad, n, box, faces);
    for (int f = 0; f < 6; ++f) {
        if (!(faces & (1u << f)) || box[f][2] < 0) continue;
        for (int v = box[f][1]; v <= box[f][3]; ++v)
            for (int u = box[f][0]; u <= box[f][2]; ++u) {
                uint32_t c = (f * n + v) * n + u;
                list[start[c] + atomicAdd(&cursor[c], 1u)] = i;
            }
    }
}

// Exclusive scan of counts[0..m) into start[0..m] by one block.
__global__ void __launch_bounds__(1024) k_grid_scan(const uint32_t* counts, uint32_t m, uint32_t* start) {
    __shared__ uint32_t part[1024];
    uint32_t per = (m + 1023) / 1024;
    uint32_t b = threadIdx.x * per, e = min(m, b + per);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (uint32_t i = b; i < e; ++i) {
        start[i] = run;
        run += counts[i];
    }
    if (threadIdx.x == 1023) start[m] = part[1023];
}

// Sorts each cell's list by star index (lists hold a handful of entries).
__global__ void k_grid_sort(const uint32_t* start, uint32_t m, uint32_t* list) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    uint32_t b = start[c], e = start[c + 1];
    for (uint32_t i = b + 1; i < e; ++i) {
        uint32_t v = list[i];
        uint32_t j = i;
        while (j > b && list[j - 1] > v) { list[j] = list[j - 1]; --j; }
        list[j] = v;
    }
}

namespace {

struct Layout {
    size_t qx, qp, qc, hits, refine, resume, cont0, cont1, xyz, counters, g_counts, g_start, g_cursor, g_list, total;
    bool cont;
};

// Adds one chunk's per-pass record (m rays) to the render statistics: the
// passes k_next_pass recorded, then the last pass from the final counts (its
// hits include the tail kernel's).
void add_pass_history(mgk_render_stats* st, const Counters& k, uint32_t m) {
    const uint32_t recorded = std::min<uint32_t>(k.n_hist, MGK_PASS_HISTORY);
    const uint32_t last = std::min<uint32_t>(k.n_hist, MGK_PASS_HISTORY - 1);
    uint64_t cross[MGK_PASS_HISTORY] = {}, cont[MGK_PASS_HISTORY] = {}, hit[MGK_PASS_HISTORY] = {},
             res[MGK_PASS_HISTORY] = {};
    for (uint32_t e = 0; e < recorded; ++e) {
        cross[e] = k.hist[e][0];
        cont[e] = k.hist[e][1];
        hit[e] = k.hist[e][2];
        res[e] = k.hist[e][3];
    }
    cross[last] += uint64_t(k.refine_count) + k.escape_count;
    hit[last] = k.hit_count;
    res[last] = k.resume_count;
    for (uint32_t e = 0; e <= last; ++e) {
        st->pass_rays[e] += e == 0 ? m : cont[e - 1];
        st->pass_crossings[e] += cross[e];
        st->pass_hits[e] += hit[e] - (e ? hit[e - 1] : 0);
        st->pass_continued[e] += cont[e];
        st->pass_to_tail[e] += res[e] - (e ? res[e - 1] : 0);
    }
    st->n_passes = std::max<uint32_t>(st->n_passes, k.n_hist + 1u);
}

Layout make_layout(const mgk_scene& s, uint32_t chunk, uint32_t n_chunks, uint32_t n_stars, uint32_t gn) {
    const size_t T = s.precision == MGK_PRECISION_F64 ? 8 : 4;
    const bool f64 = s.precision == MGK_PRECISION_F64;
    const size_t hit = f64 ? sizeof(HitEntry<double>) : sizeof(HitEntry<float>);
    const size_t ref = f64 ? sizeof(RefineEntry<double>) : sizeof(RefineEntry<float>);
    const size_t rsm = f64 ? sizeof(ResumeEntry<double>) : sizeof(ResumeEntry<float>);
    Layout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = align_up(o + bytes, 256); return at; };
    L.qx = take(size_t(chunk) * 4 * T);
    L.qp = take(size_t(chunk) * 4 * T);
    L.qc = take(size_t(chunk) * T);
    L.hits = take(size_t(chunk) * hit);
    L.refine = take(size_t(chunk) * ref);
    L.resume = take(size_t(chunk) * rsm);
    // continuation queues of the integrator's extra passes: two in room
    // scenes (one pass per reflection), one otherwise (the disk misses)
    L.cont = s.room_on != 0;
    L.cont0 = take(L.cont ? size_t(chunk) * rsm : 0);
    L.cont1 = take(size_t(chunk) * rsm);
    L.xyz = take(size_t(chunk) * 12);
    L.counters = take(size_t(n_chunks) * sizeof(Counters));
    size_t cells = n_stars ? size_t(6) * gn * gn : 0;
    L.g_counts = take(cells * 4);
    L.g_start = take(cells ? (cells + 1) * 4 : 0);
    L.g_cursor = take(cells * 4);
    L.g_list = take(size_t(n_stars) * 6 * kStarBox * kStarBox * 4);
    L.total = o;
    return L;
}

template <class P> P* at(void* base, size_t off) { return reinterpret_cast<P*>(static_cast<char*>(base) + off); }

// Runs the path over rays [first, first + n) of the scene in chunks.
//  results (device, may be NULL): per-ray records
//  ray_xyz (device, may be NULL): per-ray XYZ (3 floats per ray)
//  film / film_spec (device, may be NULL): per-pixel outputs (first must be pixel aligned then)
mgk_result run(mgk_context* ctx, const mgk_scene& s, const mgk_star* d_stars, uint32_t n_stars, const float* d_w,
               uint64_t first, uint64_t n, mgk_ray_result* results, float* ray_xyz, float* film, float* film_spec,
               mgk_render_stats* stats, cudaStream_t st, bool shade) {
    mgk_result rc = validate(&s);
    if (rc != MGK_SUCCESS) return rc;
    if (n_stars && !d_stars) return MGK_ERROR_INVALID_POINTER;
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t spp = s.spp;
    uint32_t chunk = kMaxChunkRays;
    if (film) chunk = kMaxChunkRays / spp * spp;
    if (chunk == 0) return MGK_ERROR_INVALID_ARGUMENT;
    if (n < chunk) chunk = uint32_t(n);
    const uint32_t n_chunks = n ? uint32_t((n + chunk - 1) / chunk) : 0;
    const uint32_t gn = grid_n(s.star_radius_rad);
    Layout L = make_layout(s, chunk ? chunk : 1, n_chunks ? n_chunks : 1, n_stars, gn);
    rc = ensure_arena(ctx, L.total);
    if (rc != MGK_SUCCESS) return rc;
    void* A = ctx->arena;

    // weights and the device scene table
    std::vector<float> w(3 * MGK_MAX_BINS, 0.f);
    if (!d_w) mgk_xyz_weights(s.n_bins, s.lambda_min_nm, s.lambda_max_nm, w.data());
    alignas(16) unsigned char table[sizeof(DevScene<double>)];
    fill_dev_scene(s, w.data(), table);

    // star grid
    StarGridDev grid{nullptr, nullptr, 0};
    if (shade && n_stars) {
        const uint32_t cells = 6 * gn * gn;
        uint32_t* counts = at<uint32_t>(A, L.g_counts);
        uint32_t* start = at<uint32_t>(A, L.g_start);
        uint32_t* cursor = at<uint32_t>(A, L.g_cursor);
        uint32_t* list = at<uint32_t>(A, L.g_list);
        MGK_CUDA(ctx, cudaMemsetAsync(counts, 0, size_t(cells) * 4, st));
        MGK_CUDA(ctx, cudaMemsetAsync(cursor, 0, size_t(cells) * 4, st));
        float rad = float(s.star_radius_rad);
        k_grid_count<<<(n_stars + 255) / 256, 256, 0, st>>>(d_stars, n_stars, rad, gn, counts);
        k_grid_scan<<<1, 1024, 0, st>>>(counts, cells, start);
        k_grid_fill<<<(n_stars + 255) / 256, 256, 0, st>>>(d_stars, n_stars, rad, gn, start, cursor, list);
        k_grid_sort<<<(cells + 255) / 256, 256, 0, st>>>(start, cells, list);
        MGK_CUDA(ctx, cudaGetLastError());
        grid = StarGridDev{start, list, gn};
    }
    if (film_spec) {
        MGK_CUDA(ctx, cudaMemsetAsync(film_spec, 0, size_t(s.width) * s.height * s.n_bins * 4, st));
    }
    while (ctx->events.size() < 2 * size_t(n_chunks) + 2) {
        cudaEvent_t e;
        MGK_CUDA(ctx, cudaEventCreate(&e));
        ctx->events.push_back(e);
    }
    Counters* cnt_all = at<Counters>(A, L.counters);
    MGK_CUDA(ctx, cudaMemsetAsync(cnt_all, 0, size_t(n_chunks) * sizeof(Counters), st));
    MGK_CUDA(ctx, cudaEventRecord(ctx->events[0], st));
    for (uint32_t c = 0; c < n_chunks; ++c) {
        uint64_t b = first + uint64_t(c) * chunk;
        uint32_t m = uint32_t(std::min<uint64_t>(chunk, first + n - b));
        ChunkBuffers B;
        B.qx = at<void>(A, L.qx);
        B.qp = at<void>(A, L.qp);
        B.qc = at<void>(A, L.qc);
        B.hits = at<void>(A, L.hits);
        B.refine = at<void>(A, L.refine);
        B.resume = at<void>(A, L.resume);
        if (L.cont) B.cont[0] = at<void>(A, L.cont0);
        B.cont[1] = at<void>(A, L.cont1);
        B.xyz_ray = ray_xyz ? ray_xyz + 3 * (b - first) : at<float>(A, L.xyz);
        B.counters = cnt_all + c;
        MGK_CUDA(ctx, launch_generate(s, table, b, m, B, st));
        MGK_CUDA(ctx, cudaEventRecord(ctx->events[2 + 2 * c], st));
        MGK_CUDA(ctx, launch_integrate(s, table, b, m, B, results ? results + (b - first) : nullptr, ctx->sm_count,
                                       st));
        MGK_CUDA(ctx, cudaEventRecord(ctx->events[3 + 2 * c], st));
        if (shade) {
            MGK_CUDA(ctx, cudaMemsetAsync(B.xyz_ray, 0, size_t(m) * 12, st));
            MGK_CUDA(ctx, launch_shade(s, table, b, m, B, d_stars, grid, d_w, film_spec, ctx->sm_count, st));
        }
        if (film) MGK_CUDA(ctx, launch_resolve(s, b / spp, m / spp, B.xyz_ray, film, st));
    }
    MGK_CUDA(ctx, cudaEventRecord(ctx->events[1], st));
    if (stats) {
        std::vector<Counters> h(n_chunks);
        MGK_CUDA(ctx, cudaMemcpyAsync(h.data(), cnt_all, n_chunks * sizeof(Counters), cudaMemcpyDeviceToHost, st));
        MGK_CUDA(ctx, cudaStreamSynchronize(st));
        std::memset(stats, 0, sizeof(*stats));
        stats->rays = n;
        uint32_t status = 0;
        for (uint32_t c = 0; c < n_chunks; ++c)
            add_pass_history(stats, h[c], uint32_t(std::min<uint64_t>(chunk, first + n - (first + uint64_t(c) * chunk))));
        for (auto& k : h) {
            stats->attempts += k.attempts;
            stats->steps += k.steps;
            stats->wide_attempts += k.wide_attempts;
            stats->refine_evals += k.refine_evals;
            stats->crossings += k.refine_count + k.escape_count + k.crossings_prev;
            stats->resumed += k.resume_count;
            stats->reflections += k.reflections;
            for (int i = 0; i < MGK_RAY_CLASSES; ++i) stats->class_count[i] += k.class_count[i];
            status |= k.status;
        }
        float ms = 0.f;
        MGK_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
        stats->total_ms = ms;
        double im = 0.0;
        for (uint32_t c = 0; c < n_chunks; ++c) {
            MGK_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->events[2 + 2 * c], ctx->events[3 + 2 * c]));
            im += ms;
        }
        stats->integrate_ms = im;
        if (status) {
            ctx->last_error = "queue overflow reported by the integrator";
            return MGK_ERROR_DEVICE_STATUS;
        }
    }
    return MGK_SUCCESS;
}

std::mutex g_default_mu;
mgk_context* g_default[64] = {};

}  // namespace

namespace mgk {
int context_device(mgk_context* ctx) { return ctx->device; }
size_t context_device_bytes(mgk_context* ctx) { return ctx->arena_bytes + ctx->stage_bytes; }
// Scene checks shared with the allocation-free entry point (static_scratch.cu).
mgk_result validate_scene(const mgk_scene* s) { return validate(s); }
}  // namespace mgk

// ====================================================================== ABI
extern "C" {

MGK_API mgk_result mgk_context_create(int32_t device, mgk_context** out) {
    if (!out) return MGK_ERROR_INVALID_POINTER;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return MGK_ERROR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return MGK_INVALID_CUDA_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MGK_ERROR_NO_DEVICE;
    if (prop.major != 10) return MGK_ERROR_NO_DEVICE;  // the kernels are built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return MGK_INVALID_CUDA_DEVICE;
    // the fatbin holds only sm_100a code: make sure it loads on this device
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_grid_sort) != cudaSuccess) {
        cudaGetLastError();
        return MGK_ERROR_NO_DEVICE;
    }
    mgk_context* c = new (std::nothrow) mgk_context();
    if (!c) return MGK_ERROR_HOST_ALLOCATION_FAILED;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    *out = c;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_context_destroy(mgk_context* ctx) {
    if (!ctx) return MGK_ERROR_INVALID_POINTER;
    cudaSetDevice(ctx->device);
    for (auto e : ctx->events) cudaEventDestroy(e);
    if (ctx->arena) cudaFree(ctx->arena);
    if (ctx->stage) cudaFree(ctx->stage);
    delete ctx;
    return MGK_SUCCESS;
}

MGK_API const char* mgk_last_error(mgk_context* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

MGK_API double mgk_isco_radius(double a) {
    // Bardeen, Press and Teukolsky (1972), prograde orbits, M = 1.
    double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
    double z2 = std::sqrt(3.0 * a * a + z1 * z1);
    return 3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

MGK_API void mgk_scene_defaults(mgk_scene* s) {
    if (!s) return;
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
    s->disk_r_in = mgk_isco_radius(0.9);
    s->disk_r_out = 20.0;
    s->disk_T_in = 1.0e4;
    s->cam_r = 50.0;
    s->cam_incl_rad = 75.0 * M_PI / 180.0;
    s->sensor_diag_mm = 24.0;
    s->focal_length_mm = 12.0 / std::tan(30.0 * M_PI / 180.0);  // 60 degree horizontal field of view
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
    // the reference's stage (stage.h:19-22, optical_system_settings.h:33) in
    // units of M = G M / c^2 = 0.5 m (relativity_settings.h:21-24)
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

MGK_API mgk_result mgk_xyz_weights(uint32_t n_bins, double lmin_d, double lmax_d, float* w_out) {
    if (!w_out) return MGK_ERROR_INVALID_POINTER;
    if (n_bins < 1 || n_bins > MGK_MAX_BINS || !(lmax_d > lmin_d)) return MGK_ERROR_INVALID_ARGUMENT;
    // compute_normalized_isi_cmf_weights (host_color_utilities.cuh:145-178) in
    // float over the tabulated functions: each bin midpoint-sampled at the
    // table's 1 nm spacing, then normalised by sum(Y) and the bin width.
    const float lmin = float(lmin_d), lmax = float(lmax_d);
    const float bin = (lmax - lmin) / float(n_bins);
    const float cmf_bin = (kCieMaxNm - kCieMinNm) / float(kCieEntries - 1);
    const uint32_t sub = uint32_t(std::ceil(bin / cmf_bin));
    const float dsub = bin / float(sub);
    float sum_y = 0.0f;
    for (uint32_t i = 0; i < n_bins; ++i) {
        const float x0 = lmin + float(i) * bin;
        float w[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t j = 0; j < sub; ++j) {
            float c[3];
            cie1931_sample(x0 + (float(j) + 0.5f) * dsub, c);
            for (int k = 0; k < 3; ++k) w[k] += c[k] * dsub;
        }
        for (int k = 0; k < 3; ++k) w_out[3 * i + k] = w[k];
        sum_y += w[1];
    }
    const float scale = (1.0f / sum_y) * (1.0f / bin);
    for (uint32_t i = 0; i < 3 * n_bins; ++i) w_out[i] *= scale;
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_xyz_weights_analytic(uint32_t n_bins, double lmin, double lmax, float* w_out) {
    if (!w_out) return MGK_ERROR_INVALID_POINTER;
    if (n_bins < 1 || n_bins > MGK_MAX_BINS || !(lmax > lmin)) return MGK_ERROR_INVALID_ARGUMENT;
    // the same normalisation in double over the analytic functions
    const double bin = (lmax - lmin) / n_bins;
    const uint32_t sub = uint32_t(std::ceil(bin / 1.0));
    const double dsub = bin / sub;
    std::vector<double> acc(3 * n_bins, 0.0);
    double sum_y = 0.0;
    for (uint32_t i = 0; i < n_bins; ++i) {
        for (uint32_t j = 0; j < sub; ++j) {
            double c[3];
            cmf_1931_fit(lmin + i * bin + (j + 0.5) * dsub, c);
            for (int k = 0; k < 3; ++k) acc[3 * i + k] += c[k] * dsub;
        }
        sum_y += acc[3 * i + 1];
    }
    for (uint32_t i = 0; i < 3 * n_bins; ++i) w_out[i] = float(acc[i] / sum_y / bin);
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_cmf_inverse_cdf(double lmin, double lmax, float* table_out) {
    if (!table_out) return MGK_ERROR_INVALID_POINTER;
    if (!(lmax > lmin) || !(lmin > 0.0)) return MGK_ERROR_INVALID_ARGUMENT;
    cmf_inverse_cdf_table(lmin, lmax, table_out, false);
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_cmf_inverse_cdf_analytic(double lmin, double lmax, float* table_out) {
    if (!table_out) return MGK_ERROR_INVALID_POINTER;
    if (!(lmax > lmin) || !(lmin > 0.0)) return MGK_ERROR_INVALID_ARGUMENT;
    cmf_inverse_cdf_table(lmin, lmax, table_out, true);
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_star_catalog(uint64_t seed, uint32_t n, mgk_star* out) {
    if (!out && n) return MGK_ERROR_INVALID_POINTER;
    const double ref = planck_d(550.0, 1.0e4);
    for (uint32_t i = 0; i < n; ++i) {
        double u0 = rng_unit(seed, 0x57A2u, i, 0), u1 = rng_unit(seed, 0x57A2u, i, 1);
        double u2 = rng_unit(seed, 0x57A2u, i, 2), u3 = rng_unit(seed, 0x57A2u, i, 3);
        double y = 2.0 * u0 - 1.0, ph = 2.0 * M_PI * u1, r = std::sqrt(std::max(0.0, 1.0 - y * y));
        double mag = 10.0 * u2;
        double T = 3000.0 + 27000.0 * u3;
        mgk_star& s = out[i];
        std::memset(&s, 0, sizeof(s));
        s.dir[0] = float(r * std::cos(ph));
        s.dir[1] = float(y);
        s.dir[2] = float(r * std::sin(ph));
        s.amplitude = float(std::pow(10.0, -0.4 * mag) * ref / planck_d(550.0, T));
        s.temperature = float(T);
    }
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_scene_constants(const mgk_scene* s, double* out) {
    if (!s || !out) return MGK_ERROR_INVALID_POINTER;
    SceneConsts c = scene_consts(*s);
    int k = 0;
    for (int i = 0; i < 4; ++i) out[k++] = c.cam_pos[i];
    for (int i = 0; i < 4; ++i) out[k++] = c.u_obs[i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[k++] = c.M[i][j];
    out[k++] = c.pix_a; out[k++] = c.pix_b; out[k++] = c.pix_c; out[k++] = c.pix_d;
    out[k++] = c.r_plus; out[k++] = c.spin_t; out[k++] = c.omega_sign;
    while (k < 32) out[k++] = 0.0;
    return MGK_SUCCESS;
}

// Best of three timed launches (after one untimed) of an FMA-chain probe:
// blocks x 256 threads x iters loop trips x 16 FLOP per trip.
static mgk_result probe_peak(mgk_context* ctx, cudaError_t (*launch)(uint32_t, uint32_t, void*),
                             double* flops_per_s) {
    if (!ctx || !flops_per_s) return MGK_ERROR_INVALID_POINTER;
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    mgk_result rc = ensure_arena(ctx, 4096);
    if (rc != MGK_SUCCESS) return rc;
    const uint32_t blocks = uint32_t(ctx->sm_count) * 8u, iters = 1u << 14;
    cudaEvent_t e0, e1;
    MGK_CUDA(ctx, cudaEventCreate(&e0));
    MGK_CUDA(ctx, cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        MGK_CUDA(ctx, cudaEventRecord(e0, nullptr));
        MGK_CUDA(ctx, launch(blocks, iters, ctx->arena));
        MGK_CUDA(ctx, cudaEventRecord(e1, nullptr));
        MGK_CUDA(ctx, cudaEventSynchronize(e1));
        float ms = 0.f;
        MGK_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *flops_per_s = double(blocks) * 256.0 * iters * 32.0 * 2.0 / (best * 1e-3);
    return MGK_SUCCESS;
}

static cudaError_t fp32_probe(uint32_t blocks, uint32_t iters, void* sink) {
    return launch_fma_probe(blocks, iters, static_cast<float*>(sink), nullptr);
}
static cudaError_t fp64_probe(uint32_t blocks, uint32_t iters, void* sink) {
    return launch_dfma_probe(blocks, iters, static_cast<double*>(sink), nullptr);
}

MGK_API mgk_result mgk_fp32_peak(mgk_context* ctx, double* flops_per_s) {
    return probe_peak(ctx, fp32_probe, flops_per_s);
}

MGK_API mgk_result mgk_fp64_peak(mgk_context* ctx, double* flops_per_s) {
    return probe_peak(ctx, fp64_probe, flops_per_s);
}

MGK_API mgk_result mgk_check_rounding(mgk_context* ctx, uint64_t mismatches[2]) {
    if (!ctx || !mismatches) return MGK_ERROR_INVALID_POINTER;
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    mgk_result rc = ensure_arena(ctx, 4096);
    if (rc != MGK_SUCCESS) return rc;
    auto* out = static_cast<unsigned long long*>(ctx->arena);
    MGK_CUDA(ctx, cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), nullptr));
    MGK_CUDA(ctx, launch_check_rounding(ctx->sm_count, out, nullptr));
    unsigned long long h[2] = {0, 0};
    MGK_CUDA(ctx, cudaMemcpy(h, out, sizeof h, cudaMemcpyDeviceToHost));
    mismatches[0] = h[0];
    mismatches[1] = h[1];
    return MGK_SUCCESS;
}

MGK_API void mgk_display_defaults(mgk_display_settings* ds) {
    if (ds) display_defaults(ds);
}

MGK_API mgk_result mgk_display_prepare(const mgk_display_settings* ds, mgk_display_pipeline* out) {
    if (!ds || !out) return MGK_ERROR_INVALID_POINTER;
    return display_prepare(*ds, out);
}

MGK_API mgk_result mgk_display(mgk_context* ctx, const mgk_display_pipeline* p, const float* d_xyz, uint64_t n_pixels,
                               float* d_rgb, void* stream) {
    if (!ctx || !p || ((!d_xyz || !d_rgb) && n_pixels)) return MGK_ERROR_INVALID_POINTER;
    if (p->view_transform < 0 || p->view_transform > MGK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL ||
        p->display_colorspace < 0 || p->display_colorspace > MGK_DISPLAY_COLORSPACE_ADOBE_RGB)
        return MGK_UNKNOWN_ENUM_TYPE;
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    MGK_CUDA(ctx, launch_display(*p, d_xyz, n_pixels, d_rgb, static_cast<cudaStream_t>(stream)));
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_render(mgk_context* ctx, const mgk_scene* s, const mgk_star* d_stars, uint32_t n_stars,
                              const float* d_xyz_w, float* d_film_xyz, float* d_film_spectral,
                              mgk_render_stats* stats, void* stream) {
    if (!ctx || !s || !d_film_xyz) return MGK_ERROR_INVALID_POINTER;
    uint64_t n = uint64_t(s->width) * s->height * s->spp;
    return run(ctx, *s, d_stars, n_stars, d_xyz_w, 0, n, nullptr, nullptr, d_film_xyz, d_film_spectral, stats,
               static_cast<cudaStream_t>(stream), true);
}

MGK_API mgk_result mgk_render_host(mgk_context* ctx, const mgk_scene* s, const mgk_star* h_stars, uint32_t n_stars,
                                   const float* h_xyz_w, float* h_film_xyz, mgk_render_stats* stats, void* stream) {
    if (!ctx || !s || !h_film_xyz || (n_stars && !h_stars)) return MGK_ERROR_INVALID_POINTER;
    mgk_result rc = validate(s);
    if (rc != MGK_SUCCESS) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t film_bytes = size_t(s->width) * s->height * 12;
    const size_t star_bytes = size_t(n_stars) * sizeof(mgk_star);
    const size_t w_bytes = h_xyz_w ? size_t(s->n_bins) * 12 : 0;
    // host-side inputs and outputs travel through one device staging block,
    // kept by the context and grown when a frame needs more (a block freed
    // back to the stream-ordered pool would be unmapped at the next
    // synchronisation and mapped again by every call)
    const size_t stage_bytes = align_up(film_bytes, 256) + align_up(star_bytes, 256) + align_up(w_bytes, 256) + 256;
    if (ctx->stage_bytes < stage_bytes) {
        MGK_CUDA(ctx, cudaStreamSynchronize(st));
        if (ctx->stage) cudaFree(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
        MGK_CUDA(ctx, cudaMalloc(&ctx->stage, stage_bytes));
        ctx->stage_bytes = stage_bytes;
    }
    char* p = static_cast<char*>(ctx->stage);
    float* d_film = reinterpret_cast<float*>(p);
    mgk_star* d_stars = reinterpret_cast<mgk_star*>(p + align_up(film_bytes, 256));
    float* d_w = h_xyz_w ? reinterpret_cast<float*>(p + align_up(film_bytes, 256) + align_up(star_bytes, 256)) : nullptr;
    cudaError_t e = cudaSuccess;
    if (star_bytes) e = cudaMemcpyAsync(d_stars, h_stars, star_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && w_bytes) e = cudaMemcpyAsync(d_w, h_xyz_w, w_bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync(H2D)");
    uint64_t n = uint64_t(s->width) * s->height * s->spp;
    rc = run(ctx, *s, d_stars, n_stars, d_w, 0, n, nullptr, nullptr, d_film, nullptr, stats, st, true);
    if (rc == MGK_SUCCESS) {
        e = cudaMemcpyAsync(h_film_xyz, d_film, film_bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemcpyAsync(D2H)");
    }
    return rc;
}

MGK_API mgk_result mgk_trace_rays(mgk_context* ctx, const mgk_scene* s, uint64_t first_ray, uint32_t n_rays,
                                  mgk_ray_result* d_out, void* stream) {
    if (!ctx || !s || !d_out) return MGK_ERROR_INVALID_POINTER;
    uint64_t total = uint64_t(s->width) * s->height * s->spp;
    if (first_ray > total || n_rays > total - first_ray) return MGK_ERROR_INVALID_ARGUMENT;
    return run(ctx, *s, nullptr, 0, nullptr, first_ray, n_rays, d_out, nullptr, nullptr, nullptr, nullptr,
               static_cast<cudaStream_t>(stream), false);
}

MGK_API mgk_result mgk_shade_rays(mgk_context* ctx, const mgk_scene* s, const mgk_star* d_stars, uint32_t n_stars,
                                  const float* d_xyz_w, uint64_t first_ray, uint32_t n_rays, float* d_xyz,
                                  void* stream) {
    if (!ctx || !s || !d_xyz) return MGK_ERROR_INVALID_POINTER;
    uint64_t total = uint64_t(s->width) * s->height * s->spp;
    if (first_ray > total || n_rays > total - first_ray) return MGK_ERROR_INVALID_ARGUMENT;
    return run(ctx, *s, d_stars, n_stars, d_xyz_w, first_ray, n_rays, nullptr, d_xyz, nullptr, nullptr, nullptr,
               static_cast<cudaStream_t>(stream), true);
}

// ----------------------------------------------- reference trace entry
namespace {
struct M3f { float m[9]; };
M3f mat_mul(const M3f& a, const M3f& b) {
    M3f r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i + 0] * b.m[0 + j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
void mat_vec(const M3f& a, const float v[3], float o[3]) {
    o[0] = a.m[0] * v[0] + a.m[1] * v[1] + a.m[2] * v[2];
    o[1] = a.m[3] * v[0] + a.m[4] * v[1] + a.m[5] * v[2];
    o[2] = a.m[6] * v[0] + a.m[7] * v[1] + a.m[8] * v[2];
}

// Host part of host_trace_geodesic.cu:13-51 (rotation, seeds, SI -> M units),
// with the float arithmetic of the reference; the tetrads run on the device.
mgk_result prepare_job(const magik_trace_geodesic_inital_conditions_t& ic,
                       const magik_trace_geodesic_metric_parameters_t& mp,
                       const magik_trace_geodesic_integrator_parameters_t& ip, TraceJob* J) {
    const float G = 6.67430E-11f, c = 299792458.0f;
    std::memset(J, 0, sizeof(*J));
    float L;
    J->metric = mp.metric_type;
    if (mp.metric_type == MGK_METRIC_KERR) {
        J->spin = mp.time_reversed ? -mp.kerr_spin : mp.kerr_spin;
        J->mass_sign = 1.0f;
        L = G * mp.kerr_mass / (c * c);
        J->horizon = (1.0f + std::sqrt(1.0f - J->spin * J->spin)) * mp.event_horizon_scalar;
        J->spin_abs_gt1 = std::fabs(J->spin) > 1.0f ? 1.0f : 0.0f;
    } else if (mp.metric_type == MGK_METRIC_SCHWARZSCHILD) {
        J->mass_sign = mp.schwarzschild_mass > 0.0f ? 1.0f : -1.0f;
        L = G * std::fabs(mp.schwarzschild_mass) / (c * c);
        J->horizon = 2.0f * mp.event_horizon_scalar;
    } else if (mp.metric_type == MGK_METRIC_MINKOWSKI) {
        J->mass_sign = 1.0f;
        L = 1.0f;
    } else {
        return MGK_ERROR_UNKNOWN;
    }
    J->n_max = int32_t(ip.n_integrator_max_substep);
    J->atol = ip.integrator_absolute_error_tolerance;
    J->rtol = ip.integrator_relative_error_tolerance;
    J->length_scale = L;
    float sa, ca, sb, cb, sg, cg;
    ::sincosf(ic.x_rotation, &sa, &ca);
    ::sincosf(ic.y_rotation, &sb, &cb);
    ::sincosf(ic.z_rotation, &sg, &cg);
    M3f mz{{ca, -sa, 0.f, sa, ca, 0.f, 0.f, 0.f, 1.f}};
    M3f my{{cb, 0.f, sb, 0.f, 1.f, 0.f, -sb, 0.f, cb}};
    M3f mx{{1.f, 0.f, 0.f, 0.f, cg, -sg, 0.f, sg, cg}};
    M3f rot = mat_mul(mat_mul(mx, my), mz);
    const float e0[3] = {0.f, 0.f, -1.f}, ex[3] = {1.f, 0.f, 0.f}, ey[3] = {0.f, 1.f, 0.f}, ez[3] = {0.f, 0.f, 1.f};
    float dir[3], bx[3], by[3], bz[3];
    mat_vec(rot, e0, dir);
    mat_vec(rot, ex, bx);
    mat_vec(rot, ey, by);
    mat_vec(rot, ez, bz);
    for (int i = 0; i < 3; ++i) {
        J->seed[0][i] = bx[i];
        J->seed[1][i] = by[i];
        J->seed[2][i] = bz[i];
    }
    if (ic.test_particle_type == MGK_MASSIVE) {
        J->squared_norm = -1.0f;
        float sp = ic.massive_particle_speed / c;
        for (int i = 0; i < 3; ++i) dir[i] = dir[i] * sp;
    } else {
        J->squared_norm = 0.0f;
    }
    J->x0[0] = ic.spatial_position_x / L;
    J->x0[1] = ic.spatial_position_y / L;
    J->x0[2] = ic.spatial_position_z / L;
    J->x0[3] = 0.0f / (L / c);
    float w[3] = {ic.local_proper_velocity_x / c, ic.local_proper_velocity_y / c, ic.local_proper_velocity_z / c};
    if (mp.time_reversed)
        for (int i = 0; i < 3; ++i) w[i] = -w[i];
    for (int i = 0; i < 3; ++i) {
        J->w[i] = w[i];
        J->dir[i] = dir[i] / L;
    }
    return MGK_SUCCESS;
}

mgk_context* default_context() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default[dev]) {
        mgk_context* c = nullptr;
        if (mgk_context_create(dev, &c) != MGK_SUCCESS) return nullptr;
        g_default[dev] = c;
    }
    return g_default[dev];
}
}  // namespace

MGK_API mgk_result mgk_trace_geodesic_batch(mgk_context* ctx, magik_trace_geodesic_container_t* cs,
                                            const magik_trace_geodesic_inital_conditions_t* ics,
                                            const magik_trace_geodesic_metric_parameters_t* mps,
                                            const magik_trace_geodesic_integrator_parameters_t* ips, uint32_t n) {
    if (!ctx || (n && (!cs || !ics || !mps || !ips))) return MGK_ERROR_INVALID_POINTER;
    if (n == 0) return MGK_SUCCESS;
    std::vector<TraceJob> jobs(n);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!cs[i].steps) return MGK_ERROR_INVALID_POINTER;
        if (cs[i].capacity != sizeof(magik_trace_geodesic_step_t) * uint64_t(cs[i].n_allocated_step))
            return MGK_ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH;
        if (cs[i].n_allocated_step == 0) return MGK_ERROR_INVALID_ARGUMENT;
        if (ips[i].n_integrator_max_substep == 0) return MGK_ERROR_INVALID_ARGUMENT;
        mgk_result rc = prepare_job(ics[i], mps[i], ips[i], &jobs[i]);
        if (rc != MGK_SUCCESS) return rc;
        jobs[i].n_steps = cs[i].n_allocated_step;
        jobs[i].step_offset = uint32_t(total);
        total += cs[i].n_allocated_step;
        if (total >= (1ull << 32)) return MGK_ERROR_INVALID_ARGUMENT;
    }
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t jb = align_up(n * sizeof(TraceJob), 256), sb = align_up(total * sizeof(magik_trace_geodesic_step_t), 256);
    size_t wb = align_up(n * 4, 256);
    mgk_result rc = ensure_arena(ctx, jb + sb + wb);
    if (rc != MGK_SUCCESS) return rc;
    char* A = static_cast<char*>(ctx->arena);
    cudaStream_t st = nullptr;
    MGK_CUDA(ctx, cudaMemcpyAsync(A, jobs.data(), n * sizeof(TraceJob), cudaMemcpyHostToDevice, st));
    MGK_CUDA(ctx, launch_trace_geodesic(A, n, A + jb, reinterpret_cast<uint32_t*>(A + jb + sb), st));
    std::vector<uint32_t> written(n);
    MGK_CUDA(ctx, cudaMemcpyAsync(written.data(), A + jb + sb, n * 4, cudaMemcpyDeviceToHost, st));
    MGK_CUDA(ctx, cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < n; ++i) {
        MGK_CUDA(ctx, cudaMemcpyAsync(cs[i].steps, A + jb + jobs[i].step_offset * sizeof(magik_trace_geodesic_step_t),
                                      written[i] * sizeof(magik_trace_geodesic_step_t), cudaMemcpyDeviceToHost, st));
        cs[i].n_written = written[i];
    }
    MGK_CUDA(ctx, cudaStreamSynchronize(st));
    return MGK_SUCCESS;
}

MGK_API int32_t magik_trace_geodesic(magik_trace_geodesic_container_t* container,
                                     magik_trace_geodesic_inital_conditions_t ic,
                                     magik_trace_geodesic_metric_parameters_t mp,
                                     magik_trace_geodesic_integrator_parameters_t ip) {
    if (!container || !container->steps) return MGK_ERROR_INVALID_POINTER;
    if (container->capacity != sizeof(magik_trace_geodesic_step_t) * uint64_t(container->n_allocated_step))
        return MGK_ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH;
    mgk_context* ctx = default_context();
    if (!ctx) return MGK_ERROR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_default_mu);
    mgk_result rc = mgk_trace_geodesic_batch(ctx, container, &ic, &mp, &ip, 1);
    if (rc == MGK_ERROR_INVALID_ARGUMENT || rc == MGK_ERROR_UNKNOWN) return MGK_ERROR_UNKNOWN;
    return rc;
}

}  // extern "C"

// ------------------------------------------------------------- surrogate
namespace {

constexpr uint32_t kSampleChunk = 1u << 22;
constexpr uint32_t kRouteBatch = 1u << 20;

ChunkBuffers chunk_buffers(void* A, const Layout& L, Counters* cnt) {
    ChunkBuffers B;
    B.qx = at<void>(A, L.qx);
    B.qp = at<void>(A, L.qp);
    B.qc = at<void>(A, L.qc);
    B.hits = at<void>(A, L.hits);
    B.refine = at<void>(A, L.refine);
    B.resume = at<void>(A, L.resume);
    if (L.cont) B.cont[0] = at<void>(A, L.cont0);
    B.cont[1] = at<void>(A, L.cont1);
    B.xyz_ray = at<float>(A, L.xyz);
    B.counters = cnt;
    return B;
}

}  // namespace

extern "C" {

MGK_API mgk_result mgk_make_samples(mgk_context* ctx, const mgk_scene* base, uint64_t seed, uint32_t n,
                                    uint32_t n_spin_buckets, float* d_feat, mgk_sample_label* d_lab, void* stream) {
    if (!ctx || !base || !d_feat || !d_lab) return MGK_ERROR_INVALID_POINTER;
    if (n == 0) return MGK_SUCCESS;
    mgk_scene s0 = *base;
    s0.precision = MGK_PRECISION_F64;
    mgk_result rc = validate(&s0);
    if (rc != MGK_SUCCESS) return rc;
    if (n_spin_buckets > 1024 || (n_spin_buckets && s0.escape_radius < 100.0)) return MGK_ERROR_INVALID_ARGUMENT;
    // the surrogate learns sky directions seen by the orbit camera's observer
    if (s0.room_on || s0.cam_explicit) return MGK_ERROR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t chunk = std::min(n, kSampleChunk);
    Layout L = make_layout(s0, chunk, 1, 0, 8);
    const size_t res_off = align_up(L.total, 256);
    rc = ensure_arena(ctx, res_off + size_t(chunk) * sizeof(mgk_ray_result));
    if (rc != MGK_SUCCESS) return rc;
    void* A = ctx->arena;
    Counters* cnt = at<Counters>(A, L.counters);
    mgk_ray_result* res = at<mgk_ray_result>(A, res_off);
    std::vector<float> w(3 * MGK_MAX_BINS, 0.f);
    alignas(16) unsigned char table[sizeof(DevScene<double>)];
    if (!n_spin_buckets) {
        // Frames that cover the whole field of view: n / pixels samples per
        // pixel, or a coarser pixel grid over the same sensor when n is
        // smaller than the pixel count.
        const uint64_t pixels = uint64_t(s0.width) * s0.height;
        if (n >= pixels) {
            s0.spp = uint32_t(n / pixels);
        } else {
            const double f = std::sqrt(double(n) / double(pixels));
            s0.width = std::max<uint32_t>(1, uint32_t(s0.width * f));
            s0.height = std::max<uint32_t>(1, uint32_t(s0.height * f));
            s0.spp = 1;
        }
    }
    const uint64_t frame_rays = uint64_t(s0.width) * s0.height * s0.spp;
    const uint32_t nb = n_spin_buckets ? n_spin_buckets : 1;
    uint32_t status = 0;
    for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t lo = uint32_t(uint64_t(n) * k / nb), hi = uint32_t(uint64_t(n) * (k + 1) / nb);
        mgk_scene s = s0;
        if (n_spin_buckets > 1) s.spin = 0.998 * double(k) / double(nb - 1);
        if (n_spin_buckets) s.disk_r_in = mgk_isco_radius(s.spin);
        if (s.disk_r_in >= s.disk_r_out) return MGK_ERROR_INVALID_ARGUMENT;
        for (uint32_t j = lo; j < hi;) {
            uint32_t m = std::min(chunk, hi - j);
            uint64_t first = j;
            if (!n_spin_buckets) {  // camera rays of frame j / frame_rays
                s.seed = seed + j / frame_rays;
                first = j % frame_rays;
                m = uint32_t(std::min<uint64_t>(m, frame_rays - first));
            }
            fill_dev_scene(s, w.data(), table);
            ChunkBuffers B = chunk_buffers(A, L, cnt);
            MGK_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(Counters), st));
            if (n_spin_buckets) {
                MGK_CUDA(ctx, launch_generate_samples(s, table, seed, j, m, B, d_feat + size_t(j) * 7, st));
            } else {
                MGK_CUDA(ctx, launch_generate(s, table, first, m, B, st));
                MGK_CUDA(ctx, launch_camera_features(s, table, first, m, B, d_feat + size_t(j) * 7, st));
            }
            MGK_CUDA(ctx, launch_integrate(s, table, first, m, B, res, ctx->sm_count, st));
            MGK_CUDA(ctx, launch_labels(res, d_feat + size_t(j) * 7, m, d_lab + j, st));
            Counters h;
            MGK_CUDA(ctx, cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
            MGK_CUDA(ctx, cudaStreamSynchronize(st));
            status |= h.status;
            j += m;
        }
    }
    if (status) {
        ctx->last_error = "queue overflow reported by the integrator";
        return MGK_ERROR_DEVICE_STATUS;
    }
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_render_surrogate(mgk_context* ctx, mgk_surrogate* net, const mgk_scene* sp,
                                        const mgk_star* d_stars, uint32_t n_stars, const float* d_w, float conf_min,
                                        float crit_frac, float* film, mgk_render_stats* stats, void* stream) {
    if (!ctx || !net || !sp || !film) return MGK_ERROR_INVALID_POINTER;
    const mgk_scene& s = *sp;
    mgk_result rc = validate(&s);
    if (rc != MGK_SUCCESS) return rc;
    if (s.precision == MGK_PRECISION_REF32) return MGK_ERROR_INVALID_ARGUMENT;
    // the surrogate learns sky directions seen by the orbit camera's observer
    if (s.room_on || s.cam_explicit) return MGK_ERROR_INVALID_ARGUMENT;
    if (n_stars && !d_stars) return MGK_ERROR_INVALID_POINTER;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MGK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint64_t n = uint64_t(s.width) * s.height * s.spp;
    uint32_t chunk = kMaxChunkRays / s.spp * s.spp;
    if (chunk == 0) return MGK_ERROR_INVALID_ARGUMENT;
    if (n < chunk) chunk = uint32_t(n);
    const uint32_t n_chunks = uint32_t((n + chunk - 1) / chunk);
    const uint32_t gn = grid_n(s.star_radius_rad);
    Layout L = make_layout(s, chunk, n_chunks, n_stars, gn);
    const size_t T = s.precision == MGK_PRECISION_F64 ? 8 : 4;
    const size_t fq_off = align_up(L.total, 256);
    const size_t ids_off = align_up(fq_off + size_t(chunk) * 9 * T, 256);
    const size_t feat_off = align_up(ids_off + size_t(chunk) * 4, 256);
    const size_t out_off = align_up(feat_off + size_t(kRouteBatch) * 7 * 4, 256);
    rc = ensure_arena(ctx, out_off + size_t(kRouteBatch) * 16 * 4);
    if (rc != MGK_SUCCESS) return rc;
    void* A = ctx->arena;
    std::vector<float> w(3 * MGK_MAX_BINS, 0.f);
    if (!d_w) mgk_xyz_weights(s.n_bins, s.lambda_min_nm, s.lambda_max_nm, w.data());
    alignas(16) unsigned char table[sizeof(DevScene<double>)];
    fill_dev_scene(s, w.data(), table);

    StarGridDev grid{nullptr, nullptr, 0};
    if (n_stars) {
        const uint32_t cells = 6 * gn * gn;
        uint32_t* counts = at<uint32_t>(A, L.g_counts);
        uint32_t* start = at<uint32_t>(A, L.g_start);
        uint32_t* cursor = at<uint32_t>(A, L.g_cursor);
        uint32_t* list = at<uint32_t>(A, L.g_list);
        MGK_CUDA(ctx, cudaMemsetAsync(counts, 0, size_t(cells) * 4, st));
        MGK_CUDA(ctx, cudaMemsetAsync(cursor, 0, size_t(cells) * 4, st));
        float rad = float(s.star_radius_rad);
        k_grid_count<<<(n_stars + 255) / 256, 256, 0, st>>>(d_stars, n_stars, rad, gn, counts);
        k_grid_scan<<<1, 1024, 0, st>>>(counts, cells, start);
        k_grid_fill<<<(n_stars + 255) / 256, 256, 0, st>>>(d_stars, n_stars, rad, gn, start, cursor, list);
        k_grid_sort<<<(cells + 255) / 256, 256, 0, st>>>(start, cells, list);
        MGK_CUDA(ctx, cudaGetLastError());
        grid = StarGridDev{start, list, gn};
    }
    while (ctx->events.size() < 4 * size_t(n_chunks) + 2) {
        cudaEvent_t e;
        MGK_CUDA(ctx, cudaEventCreate(&e));
        ctx->events.push_back(e);
    }
    Counters* cnt_all = at<Counters>(A, L.counters);
    MGK_CUDA(ctx, cudaMemsetAsync(cnt_all, 0, size_t(n_chunks) * sizeof(Counters), st));
    MGK_CUDA(ctx, cudaEventRecord(ctx->events[0], st));
    std::vector<Counters> h(n_chunks);
    for (uint32_t c = 0; c < n_chunks; ++c) {
        const uint64_t b = uint64_t(c) * chunk;
        const uint32_t m = uint32_t(std::min<uint64_t>(chunk, n - b));
        ChunkBuffers B = chunk_buffers(A, L, cnt_all + c);
        void* fq = at<void>(A, fq_off);
        uint32_t* ids = at<uint32_t>(A, ids_off);
        float* feat = at<float>(A, feat_off);
        float* out = at<float>(A, out_off);
        cudaEvent_t* ev = &ctx->events[2 + 4 * c];
        MGK_CUDA(ctx, launch_generate(s, table, b, m, B, st));
        MGK_CUDA(ctx, cudaEventRecord(ev[0], st));
        for (uint32_t r0 = 0; r0 < m; r0 += kRouteBatch) {
            const uint32_t k = std::min(kRouteBatch, m - r0);
            MGK_CUDA(ctx, launch_camera_features(s, table, b + r0, k, B, feat, st));
            MGK_CUDA(ctx, surrogate_infer(net, feat, k, out, st));
            MGK_CUDA(ctx, launch_route(s, table, r0, k, m, out, feat, conf_min, crit_frac, B, ids, fq, st));
        }
        MGK_CUDA(ctx, cudaEventRecord(ev[1], st));
        Counters hc;
        MGK_CUDA(ctx, cudaMemcpyAsync(&hc, cnt_all + c, sizeof(hc), cudaMemcpyDeviceToHost, st));
        MGK_CUDA(ctx, cudaStreamSynchronize(st));
        const uint32_t nf = std::min(hc.fallback_count, m);
        ChunkBuffers F = B;
        F.qx = fq;
        F.qp = static_cast<char*>(fq) + size_t(m) * 4 * T;
        F.qc = static_cast<char*>(fq) + size_t(m) * 8 * T;
        F.ray_ids = ids;
        F.hit_cap = m;
        MGK_CUDA(ctx, cudaEventRecord(ev[2], st));
        MGK_CUDA(ctx, launch_integrate(s, table, b, nf, F, nullptr, ctx->sm_count, st));
        MGK_CUDA(ctx, cudaEventRecord(ev[3], st));
        MGK_CUDA(ctx, cudaMemsetAsync(B.xyz_ray, 0, size_t(m) * 12, st));
        MGK_CUDA(ctx, launch_shade(s, table, b, m, B, d_stars, grid, d_w, nullptr, ctx->sm_count, st));
        MGK_CUDA(ctx, launch_resolve(s, b / s.spp, m / s.spp, B.xyz_ray, film, st));
    }
    MGK_CUDA(ctx, cudaEventRecord(ctx->events[1], st));
    MGK_CUDA(ctx, cudaMemcpyAsync(h.data(), cnt_all, n_chunks * sizeof(Counters), cudaMemcpyDeviceToHost, st));
    MGK_CUDA(ctx, cudaStreamSynchronize(st));
    uint32_t status = surrogate_status(net);
    for (auto& k : h) status |= k.status;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->rays = n;
        for (auto& k : h) {
            stats->attempts += k.attempts;
            stats->steps += k.steps;
            stats->wide_attempts += k.wide_attempts;
            stats->refine_evals += k.refine_evals;
            stats->crossings += k.refine_count + k.escape_count + k.crossings_prev;
            stats->resumed += k.resume_count;
            stats->reflections += k.reflections;
            stats->fallback_rays += k.fallback_count;
            for (int i = 0; i < MGK_RAY_CLASSES; ++i) stats->class_count[i] += k.class_count[i];
        }
        float ms = 0.f;
        MGK_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
        stats->total_ms = ms;
        double im = 0.0, sm = 0.0;
        for (uint32_t c = 0; c < n_chunks; ++c) {
            cudaEvent_t* ev = &ctx->events[2 + 4 * c];
            MGK_CUDA(ctx, cudaEventElapsedTime(&ms, ev[0], ev[1]));
            sm += ms;
            MGK_CUDA(ctx, cudaEventElapsedTime(&ms, ev[2], ev[3]));
            im += ms;
        }
        stats->integrate_ms = im;
        stats->surrogate_ms = sm;
    }
    if (status) {
        ctx->last_error = "queue overflow or surrogate wait timeout reported on the device";
        return MGK_ERROR_DEVICE_STATUS;
    }
    return MGK_SUCCESS;
}

}  // extern "C"
