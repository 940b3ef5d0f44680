// The reference's render-manager API (magik.h:222-313, 380-575, 660-1283)
// over libmgk's own entry points.
//
//  stage    the command semantics: mgk_stage_apply parses a command buffer
//           the way command.cpp's consume_command_buffer walks it (type,
//           size, bounds) and applies each command as apply_command does
//           (command.cpp:146-680), including its range checks; mgk_stage_scene
//           turns the stage into the mgk_scene of one sample pass.
//  manager  one worker thread per manager: it takes dispatched command
//           buffers, renders one sample per pixel per iteration with
//           mgk_render (the reference's render loop, renderer.cpp:41-128),
//           accumulates the samples on the device, resolves them with
//           mgk_display and publishes the frame to every AOV.
//  CQS      two command buffers: the host writes the front one; dispatch
//           hands it to the worker only after the worker released the
//           previous one (command.cpp:715-737), so the two never touch the
//           same buffer.
//  frames   the worker publishes under a mutex with a version number; a
//           fetch copies the newest version into the caller's collection.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/mgk_manager.h"
#include "../src/renderer/relativity/metric.cuh"
#include "internal.h"

namespace {

// ---------------------------------------------------------------- stage
uint32_t command_size(int32_t t) {
    switch (t) {
        case MAGIK_COMMAND_SET_STATE_RENDER: return sizeof(magik_command_set_state_render_t);
        case MAGIK_COMMAND_SET_STATE_PAUSE: return sizeof(magik_command_set_state_pause_t);
        case MAGIK_COMMAND_CLEAR_RENDER_BUFFER: return sizeof(magik_command_clear_render_buffer_t);
        case MAGIK_COMMAND_ADD_AOV: return sizeof(magik_command_add_aov_t);
        case MAGIK_COMMAND_REMOVE_AOV: return sizeof(magik_command_remove_aov_t);
        case MAGIK_COMMAND_PRINTF: return sizeof(magik_command_printf_t);
        case MAGIK_COMMAND_SET_METRIC_MINKOWSKI: return sizeof(magik_command_set_metric_minkowski_t);
        case MAGIK_COMMAND_SET_METRIC_SCHWARZSCHILD: return sizeof(magik_command_set_metric_schwarzschild_t);
        case MAGIK_COMMAND_SET_METRIC_KERR: return sizeof(magik_command_set_metric_kerr_t);
        case MAGIK_COMMAND_SET_ABSOLUTE_ERROR_TOLERANCE: return sizeof(magik_command_set_absolute_error_tolerance_t);
        case MAGIK_COMMAND_SET_RELATIVE_ERROR_TOLERANCE: return sizeof(magik_command_set_relative_error_tolerance_t);
        case MAGIK_COMMAND_SET_MAX_SUBSTEPS: return sizeof(magik_command_set_max_substeps_t);
        case MAGIK_COMMAND_SET_OBSERVER_LOCAL_PROPER_VELOCITY:
            return sizeof(magik_command_set_observer_local_proper_velocity_t);
        case MAGIK_COMMAND_SET_CELESTIAL_SPHERE_RADIUS: return sizeof(magik_command_set_celestial_sphere_radius_t);
        case MAGIK_COMMAND_SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR:
            return sizeof(magik_command_set_schwarzschild_event_horizon_scalar_t);
        case MAGIK_COMMAND_SET_SCHWARZSCHILD_MASS_PARAMETER:
            return sizeof(magik_command_set_schwarzschild_mass_parameter_t);
        case MAGIK_COMMAND_SET_KERR_EVENT_HORIZON_SCALAR: return sizeof(magik_command_set_kerr_event_horizon_scalar_t);
        case MAGIK_COMMAND_SET_KERR_MASS_PARAMETER: return sizeof(magik_command_set_kerr_mass_parameter_t);
        case MAGIK_COMMAND_SET_KERR_DIMENSIONLESS_SPIN_PARAMETER:
            return sizeof(magik_command_set_kerr_dimensionless_spin_parameter_t);
        case MAGIK_COMMAND_SET_ACTIVE_CAMERA: return sizeof(magik_command_set_active_camera_t);
        case MAGIK_COMMAND_SET_CAMERA_POSITION: return sizeof(magik_command_set_camera_position_t);
        case MAGIK_COMMAND_SET_CAMERA_ORIENTATION: return sizeof(magik_command_set_camera_orientation_t);
        case MAGIK_COMMAND_SET_CAMERA_RESOLUTION: return sizeof(magik_command_set_camera_resolution_t);
        case MAGIK_COMMAND_SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN:
            return sizeof(magik_command_set_n_intrinsic_spectral_irradiance_bin_t);
        case MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MAXIMUM_WAVELENGTH_NM:
            return sizeof(magik_command_set_sample_domain_maximum_wavelength_nm_t);
        case MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MINIMUM_WAVELENGTH_NM:
            return sizeof(magik_command_set_sample_domain_minimum_wavelength_nm_t);
        case MAGIK_COMMAND_SET_REDISTRIBUTION_STANDARD_DEVIATION_NM:
            return sizeof(magik_command_set_redistribution_standard_deviation_nm_t);
        case MAGIK_COMMAND_SET_COLOR_MATCHING_FUNCTION: return sizeof(magik_command_set_color_matching_function_t);
        case MAGIK_COMMAND_SET_SCENE_COLORSPACE: return sizeof(magik_command_set_scene_colorspace_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM: return sizeof(magik_command_set_view_transform_t);
        case MAGIK_COMMAND_SET_DISPLAY_COLORSPACE: return sizeof(magik_command_set_display_colorspace_t);
        case MAGIK_COMMAND_SET_OUTPUT_FORMAT: return sizeof(magik_command_set_output_format_t);
        case MAGIK_COMMAND_SET_WHITE_BALANCE_WHITE_POINT: return sizeof(magik_command_set_white_balance_white_point_t);
        case MAGIK_COMMAND_SET_WHITE_BALANCE_TINT: return sizeof(magik_command_set_white_balance_tint_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_REINHARD_EXTENDED_WHITE_LUMINANCE:
            return sizeof(magik_command_set_view_transform_reinhard_extended_white_luminance_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_START_COMPRESSION:
            return sizeof(magik_command_set_view_transform_khronos_pbr_neutral_start_compression_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_DESATURATION:
            return sizeof(magik_command_set_view_transform_khronos_pbr_neutral_desaturation_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_MODE: return sizeof(magik_command_set_view_transform_gt7_mode_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_SDR_PAPER_WHITE_BALANCE:
            return sizeof(magik_command_set_view_transform_gt7_sdr_paper_white_balance_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_REFERENCE_LUMINANCE:
            return sizeof(magik_command_set_view_transform_gt7_reference_luminance_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR:
            return sizeof(magik_command_set_view_transform_gt7_jzazbz_exponent_scale_factor_t);
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_AGX_LOOK: return sizeof(magik_command_set_view_transform_agx_look_t);
        case MAGIK_COMMAND_SET_N_GEODESIC_STEP_LIMIT: return sizeof(magik_command_set_n_geodesic_step_limit_t);
        case MAGIK_COMMAND_SET_N_REFLECTED_LIMIT: return sizeof(magik_command_set_n_reflected_limit_t);
        default: return 0;
    }
}

// Rx(x) Ry(y) Rz(z), row-major (mat3f::rotate, internal_math.h:1784-1810, as
// command.cpp:380-391 calls it).
void rotation(double x, double y, double z, float* out) {
    const double cx = std::cos(x), sx = std::sin(x), cy = std::cos(y), sy = std::sin(y), cz = std::cos(z),
                 sz = std::sin(z);
    const double Rx[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
    const double Ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    const double Rz[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
    double t[9], m[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            t[3 * i + j] = Rx[3 * i] * Ry[j] + Rx[3 * i + 1] * Ry[3 + j] + Rx[3 * i + 2] * Ry[6 + j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[3 * i + j] = t[3 * i] * Rz[j] + t[3 * i + 1] * Rz[3 + j] + t[3 * i + 2] * Rz[6 + j];
    for (int k = 0; k < 9; ++k) out[k] = float(m[k]);
}

int find_aov(const mgk_stage& s, const char* name, uint32_t len) {
    for (uint32_t i = 0; i < s.n_aov; ++i)
        if (s.aov[i].name_length == len && std::memcmp(s.aov[i].name, name, len) == 0) return int(i);
    return -1;
}

template <class C> C as(const uint32_t* p) {
    C c;
    std::memcpy(&c, p, sizeof(C));
    return c;
}

void apply_one(mgk_stage& s, int32_t type, const uint32_t* p) {
    bool clear = true;  // the settings commands invalidate the accumulated samples
    switch (type) {
        case MAGIK_COMMAND_SET_STATE_RENDER: s.rendering = 1; clear = false; break;
        case MAGIK_COMMAND_SET_STATE_PAUSE: s.rendering = 0; clear = false; break;
        case MAGIK_COMMAND_CLEAR_RENDER_BUFFER: break;
        case MAGIK_COMMAND_ADD_AOV: {
            const auto c = as<magik_command_add_aov_t>(p);
            const uint32_t len = c.length_of_name < MGK_AOV_NAME_BYTES ? c.length_of_name : MGK_AOV_NAME_BYTES;
            // an existing name keeps its buffer (the reference's emplace)
            if (find_aov(s, c.name, len) < 0 && s.n_aov < MGK_MAX_AOV) {
                mgk_aov& a = s.aov[s.n_aov++];
                std::memset(&a, 0, sizeof(a));
                a.channels = c.channels;
                a.name_length = len;
                std::memcpy(a.name, c.name, len);
            }
            clear = false;
            break;
        }
        case MAGIK_COMMAND_REMOVE_AOV: {
            const auto c = as<magik_command_remove_aov_t>(p);
            const uint32_t len = c.length_of_name < MGK_AOV_NAME_BYTES ? c.length_of_name : MGK_AOV_NAME_BYTES;
            const int i = find_aov(s, c.name, len);
            if (i >= 0) {
                for (uint32_t k = uint32_t(i) + 1; k < s.n_aov; ++k) s.aov[k - 1] = s.aov[k];
                --s.n_aov;
            }
            clear = false;
            break;
        }
        case MAGIK_COMMAND_PRINTF: {
            const auto c = as<magik_command_printf_t>(p);
            if (c.length_of_text < 512) std::printf("%.*s \n", int(c.length_of_text), c.text);
            clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_METRIC_MINKOWSKI: s.metric_type = MGK_METRIC_MINKOWSKI; break;
        case MAGIK_COMMAND_SET_METRIC_SCHWARZSCHILD: s.metric_type = MGK_METRIC_SCHWARZSCHILD; break;
        case MAGIK_COMMAND_SET_METRIC_KERR: s.metric_type = MGK_METRIC_KERR; break;
        case MAGIK_COMMAND_SET_ABSOLUTE_ERROR_TOLERANCE: {
            const float v = as<magik_command_set_absolute_error_tolerance_t>(p).absolute_error_tolerance;
            if (v > 0.0f) s.abs_tol = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_RELATIVE_ERROR_TOLERANCE: {
            const float v = as<magik_command_set_relative_error_tolerance_t>(p).relative_error_tolerance;
            if (v > 0.0f) s.rel_tol = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_MAX_SUBSTEPS: {
            const uint32_t v = as<magik_command_set_max_substeps_t>(p).max_substeps;
            if (v > 0) s.n_max_substep = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_OBSERVER_LOCAL_PROPER_VELOCITY: {
            const auto c = as<magik_command_set_observer_local_proper_velocity_t>(p);
            s.observer_velocity[0] = c.velocity_x;
            s.observer_velocity[1] = c.velocity_y;
            s.observer_velocity[2] = c.velocity_z;
            break;
        }
        case MAGIK_COMMAND_SET_CELESTIAL_SPHERE_RADIUS: {
            const float v = as<magik_command_set_celestial_sphere_radius_t>(p).celestial_sphere_radius;
            if (v > 0.0f) s.celestial_sphere_radius = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR: {
            const float v = as<magik_command_set_schwarzschild_event_horizon_scalar_t>(p).scalar;
            if (v > 1.0f) s.schwarzschild_horizon_scalar = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_SCHWARZSCHILD_MASS_PARAMETER:
            s.schwarzschild_mass = as<magik_command_set_schwarzschild_mass_parameter_t>(p).mass_parameter;
            break;
        case MAGIK_COMMAND_SET_KERR_EVENT_HORIZON_SCALAR: {
            const float v = as<magik_command_set_kerr_event_horizon_scalar_t>(p).scalar;
            if (v > 1.0f) s.kerr_horizon_scalar = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_KERR_MASS_PARAMETER:
            s.kerr_mass = as<magik_command_set_kerr_mass_parameter_t>(p).mass_parameter;
            break;
        case MAGIK_COMMAND_SET_KERR_DIMENSIONLESS_SPIN_PARAMETER:
            s.kerr_spin = as<magik_command_set_kerr_dimensionless_spin_parameter_t>(p).dimensionless_spin_parameter;
            break;
        case MAGIK_COMMAND_SET_ACTIVE_CAMERA: clear = false; break;  // one camera
        case MAGIK_COMMAND_SET_CAMERA_POSITION: {
            const auto c = as<magik_command_set_camera_position_t>(p);
            s.position[0] = c.position_x;
            s.position[1] = c.position_y;
            s.position[2] = c.position_z;
            break;
        }
        case MAGIK_COMMAND_SET_CAMERA_ORIENTATION: {
            const auto c = as<magik_command_set_camera_orientation_t>(p);
            rotation(c.rotation_x, c.rotation_y, c.rotation_z, s.orientation);
            break;
        }
        case MAGIK_COMMAND_SET_CAMERA_RESOLUTION: {
            const auto c = as<magik_command_set_camera_resolution_t>(p);
            s.x_resolution = c.x_resolution ? c.x_resolution : 2u;
            s.y_resolution = c.y_resolution ? c.y_resolution : 2u;
            break;
        }
        case MAGIK_COMMAND_SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN: {
            const uint32_t v = as<magik_command_set_n_intrinsic_spectral_irradiance_bin_t>(p).n_isi_bin;
            if (v > 0 && v <= 64) s.n_isi_bin = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MAXIMUM_WAVELENGTH_NM: {
            const float v = as<magik_command_set_sample_domain_maximum_wavelength_nm_t>(p).maximum_wavelength_nm;
            if (v > 0.0f) s.isi_max_nm = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MINIMUM_WAVELENGTH_NM: {
            const float v = as<magik_command_set_sample_domain_minimum_wavelength_nm_t>(p).minimum_wavelength_nm;
            if (v > 0.0f) s.isi_min_nm = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_REDISTRIBUTION_STANDARD_DEVIATION_NM: {
            const float v = as<magik_command_set_redistribution_standard_deviation_nm_t>(p).standard_deviation_nm;
            if (v > 0.0f) s.redistribution_sigma_nm = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_COLOR_MATCHING_FUNCTION:
            s.cmf_type = as<magik_command_set_color_matching_function_t>(p).cmf_type;
            break;
        case MAGIK_COMMAND_SET_SCENE_COLORSPACE:
            s.scene_colorspace = as<magik_command_set_scene_colorspace_t>(p).scene_colorspace;
            break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM:
            s.view_transform = as<magik_command_set_view_transform_t>(p).view_transform;
            break;
        case MAGIK_COMMAND_SET_DISPLAY_COLORSPACE:
            s.display_colorspace = as<magik_command_set_display_colorspace_t>(p).display_colorspace;
            break;
        case MAGIK_COMMAND_SET_OUTPUT_FORMAT:
            s.output_format = as<magik_command_set_output_format_t>(p).output_format;
            break;
        case MAGIK_COMMAND_SET_WHITE_BALANCE_WHITE_POINT:
            s.white_point = as<magik_command_set_white_balance_white_point_t>(p).white_point_kelvin;
            break;
        case MAGIK_COMMAND_SET_WHITE_BALANCE_TINT: s.tint = as<magik_command_set_white_balance_tint_t>(p).tint; break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_REINHARD_EXTENDED_WHITE_LUMINANCE:
            s.reinhard_white_luminance =
                as<magik_command_set_view_transform_reinhard_extended_white_luminance_t>(p).white_luminance;
            break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_START_COMPRESSION:
            s.khronos_start_compression =
                as<magik_command_set_view_transform_khronos_pbr_neutral_start_compression_t>(p).start_compression;
            break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_DESATURATION:
            s.khronos_desaturation =
                as<magik_command_set_view_transform_khronos_pbr_neutral_desaturation_t>(p).desaturation;
            break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_MODE:
            s.gt7_mode = as<magik_command_set_view_transform_gt7_mode_t>(p).mode;
            break;
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_SDR_PAPER_WHITE_BALANCE: {
            const float v = as<magik_command_set_view_transform_gt7_sdr_paper_white_balance_t>(p).sdr_paper_white_balance;
            if (v > 0.0f) s.gt7_sdr_paper_white = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_REFERENCE_LUMINANCE: {
            const float v = as<magik_command_set_view_transform_gt7_reference_luminance_t>(p).reference_luminance;
            if (v > 0.0f) s.gt7_reference_luminance = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR: {
            const float v =
                as<magik_command_set_view_transform_gt7_jzazbz_exponent_scale_factor_t>(p).jzazbz_exponent_scale_factor;
            if (v > 1.0f) s.gt7_jzazbz_exponent_scale = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_VIEW_TRANSFORM_AGX_LOOK:
            s.agx_look = as<magik_command_set_view_transform_agx_look_t>(p).look;
            break;
        case MAGIK_COMMAND_SET_N_GEODESIC_STEP_LIMIT: {
            const uint32_t v = as<magik_command_set_n_geodesic_step_limit_t>(p).n_geodesic_step_limit;
            if (v > 0) s.n_geodesic_step_limit = v; else clear = false;
            break;
        }
        case MAGIK_COMMAND_SET_N_REFLECTED_LIMIT: {
            const uint32_t v = as<magik_command_set_n_reflected_limit_t>(p).n_reflected_limit;
            if (v > 0) s.n_reflected_limit = v; else clear = false;
            break;
        }
        default: clear = false; break;
    }
    if (clear) s.clear_requested = 1;
}

// ---------------------------------------------------------------- manager
struct AovFrame {
    std::string name;
    uint32_t channels = 0;
    std::vector<float> data;  // x * y * channels
};

struct Frame {
    uint32_t x = 0, y = 0;
    std::vector<AovFrame> aovs;
};

// One sample's queue history, per integrator pass.
struct History {
    std::vector<uint32_t> a, b, isect, bxdf, redis, splat;
};

// acc += sample (acc = sample for the first), mean = acc / count.
__global__ void k_accumulate(float* __restrict__ acc, const float* __restrict__ sample, float* __restrict__ mean,
                             uint64_t n, float count, bool first) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float v = first ? sample[i] : acc[i] + sample[i];
        acc[i] = v;
        mean[i] = v / count;
    }
}

}  // namespace

struct magik_render_manager {
    int device = 0;
    int display_type = MAGIK_DISPLAY_SWAPCHAIN;
    void* user_stream = nullptr;
    uint64_t seed = 0x5EEDull;

    // command queue system
    uint32_t n_chunk = 0;
    bool drop_overflow = false;
    std::unique_ptr<uint32_t[]> cq[2];
    uint32_t occupied[2] = {0, 0};
    std::atomic<int> front{0};             // the buffer the host writes
    std::atomic<bool> back_released{true};  // the worker is done with the other one

    std::atomic<bool> running{true};
    std::atomic<int32_t> last_error{MAGIK_SUCCESS};
    std::thread worker;

    // published frame
    std::mutex frame_mutex;
    Frame frame;
    uint64_t frame_version = 0;

    // statistics (worker writes, host fetches)
    std::mutex stats_mutex;
    magik_renderer_statistics_t stats{};
    History history;
    uint64_t stats_version = 0;
    uint64_t stats_fetched = 0;
    History fetched;  // the arrays the last fetch handed out

    void fail(int32_t code) {
        int32_t expected = MAGIK_SUCCESS;
        last_error.compare_exchange_strong(expected, code);
    }
    void run();
};

struct magik_framebuffer_collection_external {
    int32_t config_type = MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_HOST;
    uint64_t version = 0;
    std::map<std::string, AovFrame> collection;
    uint32_t x = 0, y = 0;
};

void magik_render_manager::run() {
    using clock = std::chrono::steady_clock;
    const auto t_start = clock::now();
    if (cudaSetDevice(device) != cudaSuccess) {
        fail(MAGIK_INVALID_CUDA_DEVICE);
        running.store(false);
        return;
    }
    cudaStream_t st = static_cast<cudaStream_t>(user_stream);
    bool own_stream = false;
    if (!st) {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            fail(MAGIK_ERROR_UNKNOWN);
            running.store(false);
            return;
        }
        own_stream = true;
    }
    mgk_context* ctx = nullptr;
    if (mgk_context_create(device, &ctx) != MGK_SUCCESS) {
        fail(MAGIK_INVALID_CUDA_DEVICE);
        if (own_stream) cudaStreamDestroy(st);
        running.store(false);
        return;
    }
    mgk_stage stage;
    mgk_stage_defaults(&stage);
    float *d_sample = nullptr, *d_acc = nullptr, *d_mean = nullptr, *d_rgb = nullptr, *h_rgb = nullptr;
    size_t n_alloc = 0;
    uint64_t x_sample = 0;
    double total_sample_s = 0.0;

    while (running.load(std::memory_order_acquire)) {
        const auto t0 = clock::now();
        // commands: the buffer the host dispatched
        if (!back_released.load(std::memory_order_acquire)) {
            const int b = 1 - front.load(std::memory_order_relaxed);
            const mgk_result rc = mgk_stage_apply(&stage, cq[b].get(), occupied[b]);
            if (rc != MGK_SUCCESS) fail(rc);
            occupied[b] = 0;
            back_released.store(true, std::memory_order_release);
        }
        if (stage.clear_requested) {
            x_sample = 0;
            stage.clear_requested = 0;
            std::lock_guard<std::mutex> lk(stats_mutex);
            stats.x_sample = 0;
            ++stats_version;
        }
        if (!stage.rendering || stage.n_aov == 0) {
            std::this_thread::sleep_for(std::chrono::milliseconds(2));
            continue;
        }
        mgk_scene sc;
        mgk_display_settings ds;
        mgk_result rc = mgk_stage_scene(&stage, seed + x_sample, &sc, &ds);
        mgk_display_pipeline pipe;
        if (rc == MGK_SUCCESS) rc = mgk_display_prepare(&ds, &pipe);
        if (rc != MGK_SUCCESS) {
            fail(rc);
            std::this_thread::sleep_for(std::chrono::milliseconds(10));
            continue;
        }
        const uint64_t npix = uint64_t(sc.width) * sc.height, n3 = 3 * npix;
        if (n3 != n_alloc) {
            cudaFree(d_sample);
            cudaFree(d_acc);
            cudaFree(d_mean);
            cudaFree(d_rgb);
            cudaFreeHost(h_rgb);
            d_sample = d_acc = d_mean = d_rgb = h_rgb = nullptr;
            n_alloc = 0;
            if (cudaMalloc(&d_sample, n3 * 4) != cudaSuccess || cudaMalloc(&d_acc, n3 * 4) != cudaSuccess ||
                cudaMalloc(&d_mean, n3 * 4) != cudaSuccess || cudaMalloc(&d_rgb, n3 * 4) != cudaSuccess ||
                cudaMallocHost(&h_rgb, n3 * 4) != cudaSuccess) {
                fail(MAGIK_ERROR_DEVICE_OUT_OF_MEMORY);
                running.store(false);
                break;
            }
            n_alloc = n3;
            x_sample = 0;
        }
        mgk_render_stats rs;
        rc = mgk_render(ctx, &sc, nullptr, 0, nullptr, d_sample, nullptr, &rs, st);
        if (rc != MGK_SUCCESS) {
            fail(rc);
            std::this_thread::sleep_for(std::chrono::milliseconds(10));
            continue;
        }
        // running sum over the samples in order, then the mean, as one
        // render with that many samples per pixel averages them
        const uint32_t blocks = uint32_t(std::min<uint64_t>((n3 + 255) / 256, 4096));
        k_accumulate<<<blocks, 256, 0, st>>>(d_acc, d_sample, d_mean, n3, float(x_sample + 1), x_sample == 0);
        rc = mgk_display(ctx, &pipe, d_mean, npix, d_rgb, st);
        if (rc != MGK_SUCCESS || cudaMemcpyAsync(h_rgb, d_rgb, n3 * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            fail(rc != MGK_SUCCESS ? rc : MAGIK_ERROR_UNKNOWN);
            running.store(false);
            break;
        }
        ++x_sample;
        // the AOVs: RGB in the first three channels, alpha 1 in the fourth
        Frame f;
        f.x = sc.width;
        f.y = sc.height;
        for (uint32_t a = 0; a < stage.n_aov; ++a) {
            AovFrame af;
            af.name.assign(stage.aov[a].name, stage.aov[a].name_length);
            af.channels = stage.aov[a].channels;
            af.data.assign(npix * af.channels, 0.0f);
            for (uint64_t i = 0; i < npix; ++i)
                for (uint32_t c = 0; c < af.channels; ++c)
                    af.data[i * af.channels + c] = c < 3 ? h_rgb[3 * i + c] : (c == 3 ? 1.0f : 0.0f);
            f.aovs.push_back(std::move(af));
        }
        size_t fb_bytes = 0;
        for (auto& a : f.aovs) fb_bytes += a.data.size() * sizeof(float);
        {
            std::lock_guard<std::mutex> lk(frame_mutex);
            frame = std::move(f);
            ++frame_version;
        }
        // statistics of this iteration
        const auto t1 = clock::now();
        total_sample_s += rs.total_ms * 1e-3;
        History h;
        for (uint32_t p = 0; p < std::min<uint32_t>(rs.n_passes, MGK_PASS_HISTORY); ++p) {
            const uint64_t finished = rs.pass_rays[p] - rs.pass_continued[p] - rs.pass_to_tail[p];
            h.a.push_back(uint32_t(rs.pass_rays[p]));
            h.b.push_back(uint32_t(rs.pass_continued[p]));
            h.isect.push_back(uint32_t(rs.pass_crossings[p]));
            h.bxdf.push_back(uint32_t(rs.pass_hits[p] + (p + 1 < rs.n_passes ? rs.pass_continued[p] : 0)));
            h.redis.push_back(uint32_t(rs.pass_hits[p]));
            h.splat.push_back(uint32_t(finished));
        }
        {
            std::lock_guard<std::mutex> lk(stats_mutex);
            stats.x_sample = size_t(x_sample);
            stats.total_render_time_seconds = std::chrono::duration<double>(t1 - t_start).count();
            stats.latest_render_loop_iteration_time_seconds = std::chrono::duration<double>(t1 - t0).count();
            stats.total_wavefront_sample_time_seconds = total_sample_s;
            stats.latest_wavefront_sample_time_seconds = rs.total_ms * 1e-3;
            stats.latest_wavefront_history_length = h.a.size();
            stats.total_framebuffer_swapchain_size = 2 * fb_bytes;
            stats.total_wavefront_buffer_size = mgk::context_device_bytes(ctx) + 4 * n3 * 4;
            history = std::move(h);
            ++stats_version;
        }
    }
    cudaStreamSynchronize(st);
    cudaFree(d_sample);
    cudaFree(d_acc);
    cudaFree(d_mean);
    cudaFree(d_rgb);
    cudaFreeHost(h_rgb);
    mgk_context_destroy(ctx);
    if (own_stream) cudaStreamDestroy(st);
}

extern "C" {

MGK_API void mgk_stage_defaults(mgk_stage* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->metric_type = MGK_METRIC_KERR;
    s->abs_tol = 1e-3f;
    s->rel_tol = 1e-10f;
    s->n_max_substep = 56;
    s->celestial_sphere_radius = 1000.0f;
    s->schwarzschild_horizon_scalar = 1.01f;
    s->schwarzschild_mass = 6.7329546075E26f;
    s->kerr_horizon_scalar = 1.01f;
    s->kerr_mass = 6.7329546075E26f;
    s->kerr_spin = 0.999f;
    s->focal_length_mm = 12.0f;
    s->iso = 500.0f;
    s->fps = 24.0f;
    s->shutter_angle = 180.0f;
    s->sensor_diagonal_mm = 24.0f;
    s->x_resolution = 2195;
    s->y_resolution = 1860;
    s->position[0] = 2.0f; s->position[1] = 0.0f; s->position[2] = 9.0f;
    s->orientation[0] = s->orientation[4] = s->orientation[8] = 1.0f;
    s->n_isi_bin = 24;
    s->isi_max_nm = 830.0f;
    s->isi_min_nm = 360.0f;
    s->redistribution_sigma_nm = 10.0f;
    s->cmf_type = 0;
    s->scene_colorspace = MGK_SCENE_COLORSPACE_LINEAR_REC709;
    s->view_transform = MGK_VIEW_TRANSFORM_GRAN_TURISMO_7;
    s->display_colorspace = MGK_DISPLAY_COLORSPACE_REC709;
    s->output_format = 5;  // float32
    s->white_point = 5600.0f;
    s->tint = 0.0f;
    s->reinhard_white_luminance = 4.0f;
    s->khronos_start_compression = 0.8f;
    s->khronos_desaturation = 0.15f;
    s->gt7_mode = MGK_GT7_MODE_JZAZBZ;
    s->gt7_sdr_paper_white = 250.0f;
    s->gt7_reference_luminance = 100.0f;
    s->gt7_jzazbz_exponent_scale = 1.7f;
    s->agx_look = MGK_AGX_LOOK_GOLDEN;
    s->n_geodesic_step_limit = 512;
    s->n_reflected_limit = 10;
    const float bmin[3] = {-20.0f, -10.0f, -20.0f}, bmax[3] = {20.0f, 10.0f, 20.0f};
    const float lmin[3] = {-10.0f, 9.5f, -10.0f}, lmax[3] = {10.0f, 10.5f, 10.0f};
    for (int a = 0; a < 3; ++a) {
        s->box_min[a] = bmin[a]; s->box_max[a] = bmax[a];
        s->light_min[a] = lmin[a]; s->light_max[a] = lmax[a];
    }
    s->rendering = 1;
}

MGK_API uint32_t mgk_command_size(int32_t type) { return command_size(type); }

MGK_API mgk_result mgk_stage_apply(mgk_stage* s, const uint32_t* chunks, uint32_t n_chunks) {
    if (!s || (n_chunks && !chunks)) return MGK_ERROR_INVALID_POINTER;
    uint32_t off = 0;
    while (off < n_chunks) {
        int32_t type;
        std::memcpy(&type, chunks + off, sizeof(type));
        const uint32_t size = command_size(type);
        if (size == 0 || size % 4u != 0) return MAGIK_ERROR_INVALID_COMMAND;
        if (uint64_t(off) + size / 4u > n_chunks) return MAGIK_ERROR_OUT_OF_BOUNDS_COMMAND_BUFFER_READ;
        uint32_t local[sizeof(magik_command_add_aov_t) / 4 + 1];
        std::memcpy(local, chunks + off, size);
        apply_one(*s, type, local);
        off += size / 4u;
    }
    return MGK_SUCCESS;
}

MGK_API mgk_result mgk_stage_scene(const mgk_stage* st, uint64_t seed, mgk_scene* out, mgk_display_settings* ds) {
    if (!st || !out || !ds) return MGK_ERROR_INVALID_POINTER;
    if (st->metric_type < 0 || st->metric_type > 2) return MGK_ERROR_UNKNOWN_METRIC;
    const double c = 299792458.0;
    const bool kerr = st->metric_type == MGK_METRIC_KERR, schw = st->metric_type == MGK_METRIC_SCHWARZSCHILD;
    const double mass = kerr ? st->kerr_mass : st->schwarzschild_mass;
    // the metric's length scale (metric<TAG>::length_scale): M in metres
    double L = 0.0;
    mgk::with_metric(st->metric_type, [&](auto mt) { L = decltype(mt)::length_scale(std::fabs(mass)); });
    if (!(L > 0.0) || !std::isfinite(L)) return MGK_ERROR_INVALID_ARGUMENT;
    mgk_scene s;
    mgk_scene_defaults(&s);
    s.metric = st->metric_type;
    s.spin = kerr ? st->kerr_spin : 0.0;
    s.mass_sign = (schw && mass < 0.0) ? -1.0 : 1.0;
    s.horizon_scalar = kerr ? st->kerr_horizon_scalar : st->schwarzschild_horizon_scalar;
    s.abs_tol = st->abs_tol;
    s.rel_tol = st->rel_tol;
    s.n_max_substep = st->n_max_substep;
    s.h_max = 1000.0;  // metric_kerr.cuh:131
    s.max_steps = st->n_geodesic_step_limit;
    s.escape_radius = st->celestial_sphere_radius / L;
    s.cam_explicit = 1;
    for (int a = 0; a < 3; ++a) {
        s.cam_pos[a] = st->position[a] / L;
        s.cam_velocity[a] = st->observer_velocity[a] / c;
        // the orientation's columns: the camera's x, y, z axes in the world
        s.cam_axes[a] = st->orientation[3 * a];
        s.cam_axes[3 + a] = st->orientation[3 * a + 1];
        s.cam_axes[6 + a] = st->orientation[3 * a + 2];
        s.room_min[a] = st->box_min[a] / L;
        s.room_max[a] = st->box_max[a] / L;
        s.light_min[a] = st->light_min[a] / L;
        s.light_max[a] = st->light_max[a] / L;
    }
    s.focal_length_mm = st->focal_length_mm;
    s.sensor_diag_mm = st->sensor_diagonal_mm;
    s.width = st->x_resolution;
    s.height = st->y_resolution;
    s.spp = 1;
    s.seed = seed;
    s.spectral_mode = MGK_SPECTRAL_SAMPLED;
    s.n_bins = st->n_isi_bin;
    s.lambda_min_nm = st->isi_min_nm;
    s.lambda_max_nm = st->isi_max_nm;
    s.iso = st->iso;
    s.fps = st->fps;
    s.shutter_angle_deg = st->shutter_angle;
    s.redistribution_sigma_nm = st->redistribution_sigma_nm;
    s.disk_r_out = 0.0;  // the reference's stage has no disk
    s.room_on = 1;
    s.room_reflection_limit = st->n_reflected_limit;
    s.light_scale = 7.0e5;
    // MIXED where its float range allows the sphere, else F64
    s.precision = MGK_PRECISION_MIXED;
    mgk_result rc = mgk::validate_scene(&s);
    if (rc != MGK_SUCCESS) {
        s.precision = MGK_PRECISION_F64;
        if (mgk::validate_scene(&s) != MGK_SUCCESS) s.precision = MGK_PRECISION_MIXED;
        else rc = MGK_SUCCESS;
    }
    *out = s;
    mgk_display_defaults(ds);
    ds->scene_colorspace = st->scene_colorspace;
    ds->view_transform = st->view_transform;
    ds->display_colorspace = st->display_colorspace;
    ds->gt7_mode = st->gt7_mode;
    ds->agx_look = st->agx_look;
    ds->white_point_K = st->white_point;
    ds->tint = st->tint;
    ds->reinhard_white_luminance = st->reinhard_white_luminance;
    ds->khronos_start_compression = st->khronos_start_compression;
    ds->khronos_desaturation = st->khronos_desaturation;
    ds->gt7_sdr_paper_white = st->gt7_sdr_paper_white;
    ds->gt7_reference_luminance = st->gt7_reference_luminance;
    ds->gt7_jzazbz_exponent_scale = st->gt7_jzazbz_exponent_scale;
    return rc;
}

MGK_API e_magik_result_types magik_render_manager_create(magik_render_manager_t* manager,
                                                         magik_manager_descriptor_t d) {
    if (!manager) return MAGIK_ERROR_INVALID_POINTER;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    if (int64_t(d.user_device_id) >= int64_t(n)) return MAGIK_INVALID_CUDA_DEVICE;
    if (d.display_type != MAGIK_DISPLAY_SWAPCHAIN && d.display_type != MAGIK_DISPLAY_HEADLESS)
        return MAGIK_UNKNOWN_ENUM_TYPE;
    auto* m = new (std::nothrow) magik_render_manager();
    if (!m) return MAGIK_ERROR_COMMAND_BUFFER_ALLOCATION_FAILED;
    m->device = int(d.user_device_id);
    m->display_type = d.display_type;
    m->user_stream = d.user_stream;
    m->n_chunk = d.cqs_n_reserved_chunk;
    m->drop_overflow = d.cqs_drop_overflow;
    m->cq[0].reset(new (std::nothrow) uint32_t[m->n_chunk ? m->n_chunk : 1]);
    m->cq[1].reset(new (std::nothrow) uint32_t[m->n_chunk ? m->n_chunk : 1]);
    if (!m->cq[0] || !m->cq[1]) {
        delete m;
        return MAGIK_ERROR_COMMAND_BUFFER_ALLOCATION_FAILED;
    }
    m->worker = std::thread([m] { m->run(); });
    *manager = m;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_render_manager_destroy(magik_render_manager_t m) {
    if (!m) return MAGIK_ERROR_INVALID_POINTER;
    m->running.store(false, std::memory_order_release);
    if (m->worker.joinable()) m->worker.join();
    delete m;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_render_manager_fetch_error(magik_render_manager_t m) {
    if (!m) return MAGIK_ERROR_INVALID_POINTER;
    return m->last_error.load(std::memory_order_acquire);
}

MGK_API e_magik_result_types magik_cqs_push_command(magik_render_manager_t m, const void* command) {
    if (!m || !command) return MAGIK_ERROR_INVALID_POINTER;
    if (reinterpret_cast<uintptr_t>(command) % 4u != 0) return MAGIK_ERROR_PACKED_COMMAND_NOT_ALLIGNED;
    int32_t type;
    std::memcpy(&type, command, sizeof(type));
    const uint32_t size = command_size(type);
    if (size == 0) return MAGIK_ERROR_INVALID_COMMAND;
    if (size % 4u != 0) return MAGIK_ERROR_COMMAND_SIZE_NOT_A_MULTIPLE_OF_4;
    const int f = m->front.load(std::memory_order_relaxed);
    if (uint64_t(m->occupied[f]) * 4u + size > uint64_t(m->n_chunk) * 4u)
        return m->drop_overflow ? MAGIK_SUCCESS : MAGIK_ERROR_COMMAND_BUFFER_OVERFLOW;
    std::memcpy(m->cq[f].get() + m->occupied[f], command, size);
    m->occupied[f] += size / 4u;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_cqs_dispatch_command_buffer(magik_render_manager_t m, bool* is_dispatched) {
    if (!m) {
        if (is_dispatched) *is_dispatched = false;
        return MAGIK_ERROR_INVALID_POINTER;
    }
    bool done = false;
    if (m->back_released.load(std::memory_order_acquire)) {
        m->front.store(1 - m->front.load(std::memory_order_relaxed), std::memory_order_relaxed);
        m->back_released.store(false, std::memory_order_release);
        done = true;
    }
    if (is_dispatched) *is_dispatched = done;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_fetch_renderer_statistics(magik_render_manager_t m, bool* is_new_fetch,
                                                             magik_renderer_statistics_t* out) {
    if (!m || !out) {
        if (is_new_fetch) *is_new_fetch = false;
        return MAGIK_ERROR_INVALID_POINTER;
    }
    std::lock_guard<std::mutex> lk(m->stats_mutex);
    const bool fresh = m->stats_version != m->stats_fetched;
    *out = m->stats;
    m->fetched = m->history;
    out->h_latest_advance_A_queue_count_history = m->fetched.a.empty() ? nullptr : m->fetched.a.data();
    out->h_latest_advance_B_queue_count_history = m->fetched.b.empty() ? nullptr : m->fetched.b.data();
    out->h_latest_intersect_queue_count_history = m->fetched.isect.empty() ? nullptr : m->fetched.isect.data();
    out->h_latest_bxdf_queue_count_history = m->fetched.bxdf.empty() ? nullptr : m->fetched.bxdf.data();
    out->h_latest_redistribute_queue_count_history = m->fetched.redis.empty() ? nullptr : m->fetched.redis.data();
    out->h_latest_splat_queue_count_history = m->fetched.splat.empty() ? nullptr : m->fetched.splat.data();
    m->stats_fetched = m->stats_version;
    if (is_new_fetch) *is_new_fetch = fresh;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_destroy_renderer_statistics(magik_renderer_statistics_t* s) {
    if (!s) return MAGIK_ERROR_INVALID_POINTER;
    std::memset(s, 0, sizeof(*s));  // the arrays belong to the manager
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_configure_framebuffer_collection(magik_framebuffer_collection_external_t* fb,
                                                                    e_magik_framebuffer_collection_config_types t) {
    if (!fb) return MAGIK_ERROR_INVALID_POINTER;
    if (t < MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_HOST || t > MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_VULKAN_INTEROP)
        return MAGIK_UNKNOWN_ENUM_TYPE;
    auto* c = new (std::nothrow) magik_framebuffer_collection_external();
    if (!c) return MAGIK_ERROR_UNKNOWN;
    c->config_type = t;
    *fb = c;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_framebuffer_collection_fetch(magik_render_manager_t m, bool* is_new_fetch,
                                                                magik_framebuffer_collection_external_t fb) {
    if (is_new_fetch) *is_new_fetch = false;
    if (!m || !fb || !is_new_fetch) return MAGIK_ERROR_INVALID_POINTER;
    if (!m->running.load(std::memory_order_acquire)) return MAGIK_SUCCESS;
    if (m->display_type == MAGIK_DISPLAY_HEADLESS) return MAGIK_ERROR_AOV_SWAPCHAIN_NOT_INITALIZED;
    std::lock_guard<std::mutex> lk(m->frame_mutex);
    if (m->frame_version == fb->version) return MAGIK_SUCCESS;
    fb->collection.clear();
    for (const AovFrame& a : m->frame.aovs) fb->collection[a.name] = a;
    fb->x = m->frame.x;
    fb->y = m->frame.y;
    fb->version = m->frame_version;
    *is_new_fetch = true;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_extract_config_host(magik_render_manager_t m,
                                                       magik_framebuffer_container_config_host_t* container,
                                                       magik_framebuffer_collection_external_t fb, const char* name) {
    if (!m || !container || !fb || !name) return MAGIK_ERROR_INVALID_POINTER;
    if (fb->config_type != MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_HOST) return MAGIK_ERROR_AOV_INCORRECT_EXTRACT_CALL;
    auto it = fb->collection.find(name);
    if (it == fb->collection.end()) return MAGIK_SUCCESS;  // the reference leaves the container as it is
    container->x_resolution = fb->x;
    container->y_resolution = fb->y;
    container->channels = it->second.channels;
    container->size_of_data = it->second.data.size() * sizeof(float);
    container->h_data = it->second.data.data();
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_extract_config_cuda(magik_framebuffer_container_config_cuda_t* container,
                                                       magik_framebuffer_collection_external_t fb) {
    if (!container || !fb) return MAGIK_ERROR_INVALID_POINTER;
    return MAGIK_ERROR_AOV_INCORRECT_EXTRACT_CALL;  // "to be implemented" in the reference as well
}

MGK_API e_magik_result_types magik_extract_config_opengl_interop(
    magik_render_manager_t, magik_framebuffer_container_config_opengl_interop_t* container,
    magik_framebuffer_collection_external_t fb, const char*) {
    if (!container || !fb) return MAGIK_ERROR_INVALID_POINTER;
    return MAGIK_ERROR_GL_FUNCTIONS_NOT_LOADED;
}

MGK_API e_magik_result_types magik_extract_vulkan_interop(magik_framebuffer_container_config_vulkan_interop_t* container,
                                                          magik_framebuffer_collection_external_t fb) {
    if (!container || !fb) return MAGIK_ERROR_INVALID_POINTER;
    return MAGIK_ERROR_AOV_INCORRECT_EXTRACT_CALL;
}

MGK_API e_magik_result_types magik_destroy_framebuffer_collection(magik_framebuffer_collection_external_t fb) {
    delete fb;
    return MAGIK_SUCCESS;
}

MGK_API e_magik_result_types magik_gl_init(magik_gl_loader_proc) { return MAGIK_ERROR_GL_LOADER_FAILED; }

MGK_API e_magik_result_types magik_get_version(uint32_t* major, uint32_t* minor, uint32_t* revision,
                                               const char** as_char) {
    // the reference release this library serves (v0.7.0)
    if (major) *major = 0;
    if (minor) *minor = 7;
    if (revision) *revision = 0;
    if (as_char) *as_char = "Magik 0.7.0 - libmgk (sm_100a)";
    return MAGIK_SUCCESS;
}

}  // extern "C"
