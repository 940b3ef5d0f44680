// The colour resolve after the XYZ film (the reference's colour pipeline,
// color_pipeline.cuh:21-48 and kernel_splat_to_renderbuffer.cu:37-57):
//
//   XYZ -> white-balanced scene colourspace -> view transform
//       -> display colourspace -> display transfer function.
//
// mgk_display_prepare builds the pipeline on the host; k_display applies it,
// one thread per pixel (HBM-bound: 12 bytes in and 12 out per pixel).
//
// The colourspace matrices and white points are the published colorimetry
// constants (IEC 61966-2-1 sRGB, ITU-R BT.709 / BT.2020 / BT.2100, SMPTE
// RP 431-2 DCI-P3, Display P3, Adobe RGB (1998), ACEScg, CIE RGB), with the
// values and rounding the reference uses (colorspaces.cuh), so that both
// compute the same colours.  The view transforms follow their published
// forms as the reference states them: Reinhard (simple and extended
// luminance), Khronos PBR Neutral, the Gran Turismo 7 tone mapper
// (ICtCp / Jzazbz), AgX (minimal, with the Golden and Punchy looks).
// Arithmetic is float, every product and sum rounded separately (the
// library is compiled with -fmad=false), in the reference's order.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

#include "internal.h"

namespace mgk {
namespace {

struct V3 { float x, y, z; };
struct M3 { float m[9]; };  // row-major

__host__ __device__ inline V3 mv(const float* m, V3 v) {
    return V3{m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z};
}
inline M3 mm(const M3& a, const M3& b) {
    M3 c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            c.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return c;
}
inline M3 transpose(const M3& a) {
    return M3{{a.m[0], a.m[3], a.m[6], a.m[1], a.m[4], a.m[7], a.m[2], a.m[5], a.m[8]}};
}

// ---------------------------------------------------------- colourspaces
struct Colourspace {
    M3 to_xyz, from_xyz;
    float wx, wy;  // white point, CIE xy
};
constexpr float kD65x = 0.31272f, kD65y = 0.32903f;

Colourspace scene_colourspace(int cs) {
    switch (cs) {
        case MGK_SCENE_COLORSPACE_CIE_RGB:
            return {{{0.49f, 0.31f, 0.2f, 0.1769f, 0.8124f, 0.0107f, 0.0f, 0.0099f, 0.9901f}},
                    {{2.36449012f, -0.89655263f, -0.46793749f, -0.51493525f, 1.42633279f, 0.08860245f, 0.00514883f,
                      -0.01426189f, 1.00911305f}},
                    1.0f / 3.0f, 1.0f / 3.0f};
        case MGK_SCENE_COLORSPACE_LINEAR_REC709:
            return {{{0.41238656f, 0.35759149f, 0.18045049f, 0.21263682f, 0.71518298f, 0.0721802f, 0.01933062f,
                      0.11919716f, 0.95037259f}},
                    {{3.24100326f, -1.53739899f, -0.49861587f, -0.96922426f, 1.87592999f, 0.04155422f, 0.05563942f,
                      -0.2040112f, 1.05714897f}},
                    kD65x, kD65y};
        case MGK_SCENE_COLORSPACE_LINEAR_REC2020:
            return {{{6.36953507e-01f, 1.44619185e-01f, 1.68855854e-01f, 2.62698339e-01f, 6.78008766e-01f,
                      5.92928953e-02f, 4.99407097e-17f, 2.80731358e-02f, 1.06082723e+00f}},
                    {{1.71666343f, -0.35567332f, -0.25336809f, -0.66667384f, 1.61645574f, 0.0157683f, 0.01764248f,
                      -0.04277698f, 0.94224328f}},
                    kD65x, kD65y};
        case MGK_SCENE_COLORSPACE_ACES_CG:
            return {{{0.66245418f, 0.13400421f, 0.15618769f, 0.27222872f, 0.67408177f, 0.05368952f, -0.00557465f,
                      0.00406073f, 1.0103391f}},
                    {{1.64102338f, -0.32480329f, -0.2364247f, -0.66366286f, 1.61533159f, 0.01675635f, 0.01172189f,
                      -0.00828444f, 0.98839486f}},
                    0.32168f, 0.33767f};
        case MGK_SCENE_COLORSPACE_ADOBE_RGB_1998:
            return {{{0.57667f, 0.18556f, 0.18823f, 0.29734f, 0.62736f, 0.07529f, 0.02703f, 0.07069f, 0.99134f}},
                    {{2.04159f, -0.56501f, -0.34473f, -0.96924f, 1.87597f, 0.04156f, 0.01344f, -0.11836f, 1.01517f}},
                    kD65x, kD65y};
        default:  // CIE XYZ
            return {{{1, 0, 0, 0, 1, 0, 0, 0, 1}}, {{1, 0, 0, 0, 1, 0, 0, 0, 1}}, 1.0f / 3.0f, 1.0f / 3.0f};
    }
}

Colourspace display_colourspace(int cs) {
    switch (cs) {
        case MGK_DISPLAY_COLORSPACE_REC709:
            return scene_colourspace(MGK_SCENE_COLORSPACE_LINEAR_REC709);
        case MGK_DISPLAY_COLORSPACE_REC2100_PQ:
            return {{{0.63695804830129132f, 0.14461690358620838f, 0.16888097516417205f, 0.26270021201126703f,
                      0.67799807151887104f, 0.059301716469861945f, 0.0f, 0.028072693049087508f, 1.0609850577107909f}},
                    {{1.7166511879712676f, -0.35567078377639239f, -0.2533662813736598f, -0.66668435183248898f,
                      1.616481236634939f, 0.015768545813911131f, 0.017639857445310915f, -0.042770613257808655f,
                      0.94210312123547402f}},
                    kD65x, kD65y};
        case MGK_DISPLAY_COLORSPACE_REC2100_HLG:
            return {{{0.636958063f, 0.144616902f, 0.168880969f, 0.262700200f, 0.677998066f, 0.059301715f, 0.0f,
                      0.028072693f, 1.060985090f}},
                    {{1.716651200f, -0.355670780f, -0.253366292f, -0.666684330f, 1.616481180f, 0.015768547f,
                      0.017639857f, -0.042770613f, 0.942103148f}},
                    kD65x, kD65y};
        case MGK_DISPLAY_COLORSPACE_DCI_P3_THEATRICAL_WHITE_POINT:
            return {{{0.44516982f, 0.27713441f, 0.17228267f, 0.20949168f, 0.72159525f, 0.06891307f, 0.0f, 0.04706056f,
                      0.90735539f}},
                    {{2.72539403f, -1.01800301f, -0.44016320f, -0.79516803f, 1.68973205f, 0.02264719f, 0.04124189f,
                      -0.08763902f, 1.10092938f}},
                    0.314f, 0.351f};
        case MGK_DISPLAY_COLORSPACE_DISPLAY_P3:
            return {{{0.486570954f, 0.265667707f, 0.198217288f, 0.228974566f, 0.691738546f, 0.0792869106f, 0.0f,
                      0.045113381f, 1.043944360f}},
                    {{2.493496890f, -0.9313836100f, -0.402710795f, -0.829488993f, 1.7626640800f, 0.0236246865f,
                      0.035845831f, -0.0761723891f, 0.956884503f}},
                    kD65x, kD65y};
        case MGK_DISPLAY_COLORSPACE_ADOBE_RGB:
            return {{{0.57666904f, 0.18555824f, 0.18822865f, 0.29734498f, 0.62736357f, 0.07529146f, 0.02703136f,
                      0.07068885f, 0.99133754f}},
                    {{2.04158790f, -0.56500697f, -0.34473135f, -0.96924364f, 1.87596750f, 0.04155506f, 0.01344428f,
                      -0.11836239f, 1.01517499f}},
                    kD65x, kD65y};
        default:  // sRGB
            return {{{0.4124564f, 0.3575761f, 0.1804375f, 0.2126729f, 0.7151522f, 0.0721750f, 0.0193339f, 0.1191920f,
                      0.9503041f}},
                    {{3.2406255f, -1.537208f, -0.4986286f, -0.9689307f, 1.8757561f, 0.0415175f, 0.0557101f, -0.2040211f,
                      1.0569959f}},
                    kD65x, kD65y};
    }
}

V3 xy_to_XYZ(float x, float y) { return V3{x / y, 1.0f, (1.0f - x - y) / y}; }

// Bradford chromatic adaptation from one white to another (von Kries in the
// Bradford cone space): M^-1 diag(lms_dst / lms_src) M.
M3 chromatic_adaptation(V3 src, V3 dst) {
    const M3 m{{0.8951f, 0.2664f, -0.1614f, -0.7502f, 1.7135f, 0.0367f, 0.0389f, -0.0685f, 1.0296f}};
    const M3 mi{{0.9869929f, -0.1470543f, 0.1599627f, 0.4323053f, 0.5183603f, 0.0492912f, -0.0085287f, 0.0400428f,
                 0.9684867f}};
    const V3 ls = mv(m.m, src), ld = mv(m.m, dst);
    const M3 d{{ld.x / ls.x, 0, 0, 0, ld.y / ls.y, 0, 0, 0, ld.z / ls.z}};
    return mm(mm(mi, d), m);
}

M3 convert_colourspace(const Colourspace& from, const Colourspace& to) {
    return mm(mm(to.from_xyz, chromatic_adaptation(xy_to_XYZ(from.wx, from.wy), xy_to_XYZ(to.wx, to.wy))), from.to_xyz);
}

// Planck's law in float (internal_math.h:2511-2526), wavelength in nm.
float planck_f(float nm, float temperature) {
    const float h = 6.62607015E-34f, c = 299792458.0f, kb = 1.380649E-23f;
    const float wl = nm * 1e-9f;
    const float t0 = h * c;
    const float t1 = 2.0f * t0 * c;
    const float t2 = wl * wl * wl * wl * wl;
    const float t3 = std::exp(t0 / (wl * kb * temperature)) - 1.0f;
    return (t1 / t2) * (1.0f / t3);
}

// White balance white point (host_color_utilities.cuh:24-51): the blackbody
// at `temperature` integrated against the colour-matching functions at the
// 471 wavelengths 360, 361, ... 830 nm of the CIE table, normalised to Y = 1;
// the tint moves it along the normal of the Planckian locus in CIE 1960 uv
// (the direction towards T + 1 K rotated by 90 degrees, pointing to +v).
V3 white_point_xyz(float temperature, float tint) {
    V3 b0{0, 0, 0}, b1{0, 0, 0};
    float lam = 360.0f;
    const float step = (830.0f - 360.0f) / 470.0f;
    for (int i = 0; i < 471; ++i) {
        float c[3];
        cie1931_sample(lam, c);
        const V3 cm{c[0], c[1], c[2]};
        const float p0 = planck_f(lam, temperature), p1 = planck_f(lam, temperature + 1.0f);
        b0 = V3{b0.x + cm.x * p0, b0.y + cm.y * p0, b0.z + cm.z * p0};
        b1 = V3{b1.x + cm.x * p1, b1.y + cm.y * p1, b1.z + cm.z * p1};
        lam += step;
    }
    b0 = V3{b0.x / b0.y, b0.y / b0.y, b0.z / b0.y};
    b1 = V3{b1.x / b1.y, b1.y / b1.y, b1.z / b1.y};
    auto uv = [](V3 v) {
        const float d = v.x + 15.0f * v.y + 3.0f * v.z;
        return std::pair<float, float>{4.0f * v.x / d, 6.0f * v.y / d};
    };
    const auto uv0 = uv(b0), uv1 = uv(b1);
    float nx = uv1.first - uv0.first, ny = uv1.second - uv0.second;
    const float len = std::sqrt(nx * nx + ny * ny);
    nx /= len; ny /= len;
    float rx = -ny, ry = nx;
    if (ry < 0.0f) { rx *= -1.0f; ry *= -1.0f; }
    const float u = uv0.first + rx * tint, v = uv0.second + ry * tint;
    const float den = 2.0f * u - 8.0f * v + 4.0f;
    return xy_to_XYZ(3.0f * u / den, 2.0f * v / den);
}

// ------------------------------------------------------------------ GT7
// The Gran Turismo 7 tone mapper's pieces (view_transform.cuh:115-462),
// shared by the host set-up and the kernel.
__host__ __device__ inline float gt7_smooth_step(float x, float e0, float e1) {
    const float t = (x - e0) / (e1 - e0);
    if (x < e0) return 0.0f;
    if (x > e1) return 1.0f;
    return t * t * (3.0f - 2.0f * t);
}
// SMPTE ST 2084 (PQ) with the exponent m2 scaled (Jzazbz uses 1.7 m2).
__host__ __device__ inline float gt7_eotf(float n, float ref_lum, float scale) {
    n = n < 0.0f ? 0.0f : (n > 1.0f ? 1.0f : n);
    const float m1 = 0.1593017578125f, m2 = 78.84375f * scale, c1 = 0.8359375f, c2 = 18.8515625f, c3 = 18.6875f;
    const float np = powf(n, 1.0f / m2);
    float l = np - c1;
    if (l < 0.0f) l = 0.0f;
    l = l / (c2 - c3 * np);
    l = powf(l, 1.0f / m1);
    return (l * 10000.0f) / ref_lum;
}
__host__ __device__ inline float gt7_inverse_eotf(float v, float ref_lum, float scale) {
    const float m1 = 0.1593017578125f, m2 = 78.84375f * scale, c1 = 0.8359375f, c2 = 18.8515625f, c3 = 18.6875f;
    const float y = (v * ref_lum) / 10000.0f;
    const float ym = powf(y, m1);
    return exp2f(m2 * (log2f(c1 + c2 * ym) - log2f(1.0f + c3 * ym)));
}
__host__ __device__ inline void gt7_rgb_to_ucs(const float* rgb, float* o, float ref_lum, float scale, int mode) {
    if (mode == MGK_GT7_MODE_ICTCP) {
        const float l = (rgb[0] * 1688.0f + rgb[1] * 2146.0f + rgb[2] * 262.0f) / 4096.0f;
        const float m = (rgb[0] * 683.0f + rgb[1] * 2951.0f + rgb[2] * 462.0f) / 4096.0f;
        const float s = (rgb[0] * 99.0f + rgb[1] * 309.0f + rgb[2] * 3688.0f) / 4096.0f;
        const float lp = gt7_inverse_eotf(l, ref_lum, 1.0f), mp = gt7_inverse_eotf(m, ref_lum, 1.0f),
                    sp = gt7_inverse_eotf(s, ref_lum, 1.0f);
        o[0] = (2048.0f * lp + 2048.0f * mp) / 4096.0f;
        o[1] = (6610.0f * lp - 13613.0f * mp + 7003.0f * sp) / 4096.0f;
        o[2] = (17933.0f * lp - 17390.0f * mp - 543.0f * sp) / 4096.0f;
    } else {
        const float l = rgb[0] * 0.530004f + rgb[1] * 0.355704f + rgb[2] * 0.086090f;
        const float m = rgb[0] * 0.289388f + rgb[1] * 0.525395f + rgb[2] * 0.157481f;
        const float s = rgb[0] * 0.091098f + rgb[1] * 0.147588f + rgb[2] * 0.734234f;
        const float lp = gt7_inverse_eotf(l, ref_lum, scale), mp = gt7_inverse_eotf(m, ref_lum, scale),
                    sp = gt7_inverse_eotf(s, ref_lum, scale);
        const float iz = 0.5f * lp + 0.5f * mp;
        o[0] = (0.44f * iz) / (1.0f - 0.56f * iz) - 1.6295499532821566e-11f;
        o[1] = 3.524000f * lp - 4.066708f * mp + 0.542708f * sp;
        o[2] = 0.199076f * lp + 1.096799f * mp - 1.295875f * sp;
    }
}
__host__ __device__ inline void gt7_ucs_to_rgb(const float* u, float* rgb, float ref_lum, float scale, int mode) {
    if (mode == MGK_GT7_MODE_ICTCP) {
        const float l = u[0] + 0.00860904f * u[1] + 0.11103f * u[2];
        const float m = u[0] - 0.00860904f * u[1] - 0.11103f * u[2];
        const float s = u[0] + 0.560031f * u[1] - 0.320627f * u[2];
        const float ll = gt7_eotf(l, ref_lum, 1.0f), ml = gt7_eotf(m, ref_lum, 1.0f), sl = gt7_eotf(s, ref_lum, 1.0f);
        rgb[0] = fmaxf(3.43661f * ll - 2.50645f * ml + 0.0698454f * sl, 0.0f);
        rgb[1] = fmaxf(-0.79133f * ll + 1.9836f * ml - 0.192271f * sl, 0.0f);
        rgb[2] = fmaxf(-0.0259499f * ll - 0.0989137f * ml + 1.12486f * sl, 0.0f);
    } else {
        const float jz = u[0] + 1.6295499532821566e-11f;
        const float iz = jz / (0.44f + 0.56f * jz);
        const float a = u[1], b = u[2];
        const float l = iz + a * 1.386050432715393e-1f + b * 5.804731615611869e-2f;
        const float m = iz + a * -1.386050432715393e-1f + b * -5.804731615611869e-2f;
        const float s = iz + a * -9.601924202631895e-2f + b * -8.118918960560390e-1f;
        const float ll = gt7_eotf(l, ref_lum, scale), ml = gt7_eotf(m, ref_lum, scale), sl = gt7_eotf(s, ref_lum, scale);
        rgb[0] = ll * 2.990669f + ml * -2.049742f + sl * 0.088977f;
        rgb[1] = ll * -1.634525f + ml * 3.145627f + sl * -0.483037f;
        rgb[2] = ll * -0.042505f + ml * -0.377983f + sl * 1.448019f;
    }
}

// ------------------------------------------------------------ the kernel
__device__ inline float gt7_curve(const mgk_display_pipeline& p, float x) {
    if (x < 0.0f) return 0.0f;
    const float w_lin = gt7_smooth_step(x, 0.0f, p.gt7_mid_point);
    const float w_toe = 1.0f - w_lin;
    const float shoulder = p.gt7_kA + p.gt7_kB * expf(x * p.gt7_kC);
    if (x < p.gt7_linear_section * p.gt7_peak_intensity) {
        const float toe = p.gt7_mid_point * powf(x / p.gt7_mid_point, p.gt7_toe_strength);
        return w_toe * toe + w_lin * x;
    }
    return shoulder;
}

__device__ inline V3 view_transform(const mgk_display_pipeline& p, V3 c) {
    switch (p.view_transform) {
        case MGK_VIEW_TRANSFORM_REINHARD_SIMPLE:
            return V3{c.x / (c.x + 1.0f), c.y / (c.y + 1.0f), c.z / (c.z + 1.0f)};
        case MGK_VIEW_TRANSFORM_REINHARD_EXTENDED: {
            const float L = p.luminance_weights[0] * c.x + p.luminance_weights[1] * c.y + p.luminance_weights[2] * c.z;
            const float w2 = p.reinhard_white_luminance * p.reinhard_white_luminance;
            const float L0 = L * (1.0f + L / w2) / (1.0f + L);
            if (!(L > 0.0f)) return V3{0.0f, 0.0f, 0.0f};
            const float s = L0 / L;
            return V3{c.x * s, c.y * s, c.z * s};
        }
        case MGK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL: {
            V3 col = mv(p.vt_to_working, c);
            const float start = p.khronos_start_compression - 0.04f;
            const float x = fminf(col.x, fminf(col.y, col.z));
            const float off = x < 0.08f ? x - 6.25f * x * x : 0.04f;
            col = V3{col.x - off, col.y - off, col.z - off};
            const float peak = fmaxf(col.x, fmaxf(col.y, col.z));
            if (peak < start) return mv(p.vt_from_working, col);
            const float d = 1.0f - start;
            const float new_peak = 1.0f - d * d / (peak + d - start);
            const float s = new_peak / peak;
            col = V3{col.x * s, col.y * s, col.z * s};
            const float g = 1.0f - 1.0f / (p.khronos_desaturation * (peak - new_peak) + 1.0f);
            const float ig = 1.0f - g;
            col = V3{col.x * ig + new_peak * g, col.y * ig + new_peak * g, col.z * ig + new_peak * g};
            return mv(p.vt_from_working, col);
        }
        case MGK_VIEW_TRANSFORM_GRAN_TURISMO_7: {
            // the reference clamps a copy of the Rec.2020 colour and tone-maps
            // the unclamped one (view_transform.cuh:446-460); so does this
            const V3 w = mv(p.vt_to_working, c);
            const float rgb[3] = {w.x, w.y, w.z};
            const float rl = p.gt7_reference_luminance, sc = p.gt7_jzazbz_exponent_scale;
            float ucs[3], skew_ucs[3], scaled[3];
            gt7_rgb_to_ucs(rgb, ucs, rl, sc, p.gt7_mode);
            const float skew[3] = {gt7_curve(p, rgb[0]), gt7_curve(p, rgb[1]), gt7_curve(p, rgb[2])};
            gt7_rgb_to_ucs(skew, skew_ucs, rl, sc, p.gt7_mode);
            const float chroma = 1.0f - gt7_smooth_step(ucs[0] / p.gt7_fb_luminance_target_ucs, p.gt7_fade_start,
                                                        p.gt7_fade_end);
            const float su[3] = {skew_ucs[0], ucs[1] * chroma, ucs[2] * chroma};
            gt7_ucs_to_rgb(su, scaled, rl, sc, p.gt7_mode);
            float o[3];
            for (int i = 0; i < 3; ++i) {
                const float blended = (1.0f - p.gt7_blend_ratio) * skew[i] + p.gt7_blend_ratio * scaled[i];
                o[i] = p.gt7_sdr_correction * fminf(blended, p.gt7_fb_luminance_target);
            }
            return mv(p.vt_from_working, V3{o[0], o[1], o[2]});
        }
        case MGK_VIEW_TRANSFORM_AGX: {
            const float min_ev = -12.47393f, max_ev = 4.026069f;
            V3 v = mv(p.vt_to_working, c);
            v = V3{fmaxf(0.0f, v.x), fmaxf(0.0f, v.y), fmaxf(0.0f, v.z)};
            v = mv(p.agx_inset, v);
            v = V3{fmaxf(v.x, 1e-10f), fmaxf(v.y, 1e-10f), fmaxf(v.z, 1e-10f)};
            v = V3{log2f(v.x), log2f(v.y), log2f(v.z)};
            const float span = max_ev - min_ev;
            v = V3{(v.x - min_ev) / span, (v.y - min_ev) / span, (v.z - min_ev) / span};
            auto cl = [](float a) { return fminf(fmaxf(a, 0.0f), 1.0f); };
            v = V3{cl(v.x), cl(v.y), cl(v.z)};
            // the minimal AgX contrast polynomial
            auto poly = [](float x) {
                const float x2 = x * x, x4 = x2 * x2, x6 = x4 * x2;
                return -17.86f * x6 * x + 78.01f * x6 - 126.7f * x4 * x + 92.06f * x4 - 28.72f * x2 * x + 4.361f * x2 -
                       0.1718f * x + 0.002857f;
            };
            v = V3{poly(v.x), poly(v.y), poly(v.z)};
            if (p.agx_look != MGK_AGX_LOOK_NONE) {
                const float luma = v.x * 0.2126f + v.y * 0.7152f + v.z * 0.0722f;
                V3 slope{1.0f, 1.0f, 1.0f};
                float power = 1.0f, sat = 1.0f;
                if (p.agx_look == MGK_AGX_LOOK_GOLDEN) { slope = V3{1.0f, 0.9f, 0.5f}; power = 0.8f; sat = 1.3f; }
                if (p.agx_look == MGK_AGX_LOOK_PUNCHY) { power = 1.35f; sat = 1.4f; }
                const V3 v2{powf(v.x * slope.x + 0.0f, power), powf(v.y * slope.y + 0.0f, power),
                            powf(v.z * slope.z + 0.0f, power)};
                v = V3{luma + sat * (v2.x - luma), luma + sat * (v2.y - luma), luma + sat * (v2.z - luma)};
            }
            v = mv(p.agx_outset, v);
            v = V3{powf(fmaxf(0.0f, v.x), 2.2f), powf(fmaxf(0.0f, v.y), 2.2f), powf(fmaxf(0.0f, v.z), 2.2f)};
            return mv(p.vt_from_working, v);
        }
        default:
            return c;
    }
}

__device__ inline float encode1(int display, float L) {
    switch (display) {
        case MGK_DISPLAY_COLORSPACE_REC709:
            return powf(fmaxf(L, 0.0f), 1.0f / 2.4f);
        case MGK_DISPLAY_COLORSPACE_REC2100_PQ: {
            const float m1 = 2610.0f / 16384.0f, m2 = 2523.0f / 4096.0f * 128.0f, c1 = 3424.0f / 4096.0f,
                        c2 = 2413.0f / 4096.0f * 32.0f, c3 = 2392.0f / 4096.0f * 32.0f;
            const float lc = fminf(fmaxf(L, 0.0f), 1.0f);
            const float lm = powf(lc, m1);
            return powf((c1 + c2 * lm) / (1.0f + c3 * lm), m2);
        }
        case MGK_DISPLAY_COLORSPACE_REC2100_HLG: {
            const float a = 0.17883277f, b = 0.28466892f, c = 0.55991073f;
            const float ln = fminf(fmaxf(L, 0.0f), 1.0f);
            if (ln <= 1.0f / 12.0f) return sqrtf(3.0f * ln);
            return a * logf(12.0f * ln - b) + c;
        }
        case MGK_DISPLAY_COLORSPACE_DCI_P3_THEATRICAL_WHITE_POINT:
            return powf(fmaxf(L, 0.0f), 1.0f / 2.6f);
        case MGK_DISPLAY_COLORSPACE_ADOBE_RGB:
            return powf(fminf(fmaxf(L, 0.0f), 1.0f), 256.0f / 563.0f);
        default:  // sRGB and Display P3
            if (L <= 0.0031308f) return 12.92f * L;
            return 1.055f * powf(L, 1.0f / 2.4f) - 0.055f;
    }
}

__global__ void __launch_bounds__(256) k_display(const mgk_display_pipeline p, const float* __restrict__ xyz,
                                                 uint64_t n, float* __restrict__ rgb) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 c{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    V3 v = mv(p.xyz_to_scene, c);
    v = view_transform(p, v);
    v = mv(p.scene_to_display, v);
    rgb[3 * i] = encode1(p.display_colorspace, v.x);
    rgb[3 * i + 1] = encode1(p.display_colorspace, v.y);
    rgb[3 * i + 2] = encode1(p.display_colorspace, v.z);
}

void put(float* dst, const M3& m) {
    for (int i = 0; i < 9; ++i) dst[i] = m.m[i];
}

}  // namespace

void display_defaults(mgk_display_settings* d) {
    *d = mgk_display_settings{};
    d->scene_colorspace = MGK_SCENE_COLORSPACE_LINEAR_REC709;
    d->view_transform = MGK_VIEW_TRANSFORM_GRAN_TURISMO_7;
    d->display_colorspace = MGK_DISPLAY_COLORSPACE_REC709;
    d->gt7_mode = MGK_GT7_MODE_JZAZBZ;
    d->agx_look = MGK_AGX_LOOK_GOLDEN;
    d->white_point_K = 5600.0;
    d->tint = 0.0;
    d->reinhard_white_luminance = 4.0;
    d->khronos_start_compression = 0.8;
    d->khronos_desaturation = 0.15;
    d->gt7_sdr_paper_white = 250.0;
    d->gt7_reference_luminance = 100.0;
    d->gt7_jzazbz_exponent_scale = 1.7;
}

mgk_result display_prepare(const mgk_display_settings& s, mgk_display_pipeline* out) {
    if (s.scene_colorspace < 0 || s.scene_colorspace > MGK_SCENE_COLORSPACE_ADOBE_RGB_1998 ||
        s.display_colorspace < 0 || s.display_colorspace > MGK_DISPLAY_COLORSPACE_ADOBE_RGB ||
        s.view_transform < 0 || s.view_transform > MGK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL || s.gt7_mode < 0 ||
        s.gt7_mode > MGK_GT7_MODE_JZAZBZ || s.agx_look < 0 || s.agx_look > MGK_AGX_LOOK_PUNCHY)
        return MGK_UNKNOWN_ENUM_TYPE;
    if (!(s.white_point_K > 0.0) || !(s.reinhard_white_luminance > 0.0) || !(s.gt7_sdr_paper_white > 0.0) ||
        !(s.gt7_reference_luminance > 0.0) || !(s.gt7_jzazbz_exponent_scale > 0.0))
        return MGK_ERROR_INVALID_ARGUMENT;
    mgk_display_pipeline p{};
    p.view_transform = s.view_transform;
    p.display_colorspace = s.display_colorspace;
    p.gt7_mode = s.gt7_mode;
    p.agx_look = s.agx_look;
    const Colourspace sc = scene_colourspace(s.scene_colorspace);
    const Colourspace dc = display_colourspace(s.display_colorspace);
    // color_pipeline.cuh:38-43
    const V3 wp_src = white_point_xyz(float(s.white_point_K), float(s.tint));
    const V3 wp_scene = xy_to_XYZ(sc.wx, sc.wy);
    put(p.xyz_to_scene, mm(sc.from_xyz, chromatic_adaptation(wp_src, wp_scene)));
    put(p.scene_to_display, mm(mm(dc.from_xyz, chromatic_adaptation(wp_scene, xy_to_XYZ(dc.wx, dc.wy))), sc.to_xyz));
    // view transform parameters (view_transform.cuh make_params)
    p.luminance_weights[0] = sc.to_xyz.m[3];
    p.luminance_weights[1] = sc.to_xyz.m[4];
    p.luminance_weights[2] = sc.to_xyz.m[5];
    p.reinhard_white_luminance = float(s.reinhard_white_luminance);
    p.khronos_start_compression = float(s.khronos_start_compression);
    p.khronos_desaturation = float(s.khronos_desaturation);
    const Colourspace working = scene_colourspace(s.view_transform == MGK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL
                                                      ? MGK_SCENE_COLORSPACE_LINEAR_REC709
                                                      : MGK_SCENE_COLORSPACE_LINEAR_REC2020);
    put(p.vt_to_working, convert_colourspace(sc, working));
    put(p.vt_from_working, convert_colourspace(working, sc));
    put(p.agx_inset, transpose(M3{{0.856627153315983f, 0.137318972929847f, 0.11189821299995f, 0.0951212405381588f,
                                   0.761241990602591f, 0.0767994186031903f, 0.0482516061458583f, 0.101439036467562f,
                                   0.811302368396859f}}));
    put(p.agx_outset, transpose(M3{{1.1271005818144f, -0.14132976349844f, -0.14132976349844f, -0.11060664309660f,
                                    1.1578237022163f, -0.11060664309660f, -0.016493938717835f, -0.016493938717834f,
                                    1.2519364065950f}}));
    // GT7 (SDR): the curve through the paper white, view_transform.cuh:318-393
    p.gt7_reference_luminance = float(s.gt7_reference_luminance);
    p.gt7_jzazbz_exponent_scale = float(s.gt7_jzazbz_exponent_scale);
    const float paper = float(s.gt7_sdr_paper_white);
    p.gt7_sdr_correction = 1.0f / (paper / p.gt7_reference_luminance);
    p.gt7_fb_luminance_target = paper / p.gt7_reference_luminance;
    p.gt7_peak_intensity = p.gt7_fb_luminance_target;
    p.gt7_alpha = 0.25f;
    p.gt7_mid_point = 0.538f;
    p.gt7_linear_section = 0.444f;
    p.gt7_toe_strength = 1.280f;
    const float k = (p.gt7_linear_section - 1.0f) / (p.gt7_alpha - 1.0f);
    p.gt7_kA = p.gt7_peak_intensity * p.gt7_linear_section + p.gt7_peak_intensity * k;
    p.gt7_kB = -p.gt7_peak_intensity * k * std::exp(p.gt7_linear_section / k);
    p.gt7_kC = -1.0f / (k * p.gt7_peak_intensity);
    p.gt7_blend_ratio = 0.6f;
    p.gt7_fade_start = 0.98f;
    p.gt7_fade_end = 1.16f;
    const float fb[3] = {p.gt7_fb_luminance_target, p.gt7_fb_luminance_target, p.gt7_fb_luminance_target};
    float ucs[3];
    gt7_rgb_to_ucs(fb, ucs, p.gt7_reference_luminance, p.gt7_jzazbz_exponent_scale, p.gt7_mode);
    p.gt7_fb_luminance_target_ucs = ucs[0];
    *out = p;
    return MGK_SUCCESS;
}

cudaError_t launch_display(const mgk_display_pipeline& p, const float* xyz, uint64_t n, float* rgb, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_display<<<uint32_t((n + 255) / 256), 256, 0, st>>>(p, xyz, n, rgb);
    return cudaGetLastError();
}

}  // namespace mgk
