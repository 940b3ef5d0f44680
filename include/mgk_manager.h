/*
 * mgk_manager.h - the reference's render-manager API served by libmgk.
 *
 * A render manager owns a worker thread on one GPU.  The host (the "DCC")
 * drives it through the command queue system: it pushes command structs into
 * a front buffer (magik_cqs_push_command) and hands that buffer to the worker
 * (magik_cqs_dispatch_command_buffer).  The worker applies the commands to its
 * stage, renders one sample per pixel per iteration with mgk_render (the room
 * scene of the reference's stage around the configured metric, the sampled
 * spectral sensor), accumulates the samples, resolves them to display colour
 * with mgk_display and publishes the result to every AOV (named output
 * buffer) the commands created.  The host fetches the newest published frame
 * into a framebuffer collection (magik_framebuffer_collection_fetch) and
 * reads an AOV's pixels from it (magik_extract_config_host).
 *
 * Types, names, enum values and struct layouts are the reference's
 * (include/magik/magik.h: 38-110 results, 222-313 manager, 380-428
 * statistics, 431-575 framebuffers, 660-1283 command queue system), so that a
 * program written against magik.h links against libmgk unchanged.  When the
 * reference's magik.h is included first its declarations are used instead.
 *
 * The stage helpers (mgk_stage_*) are this library's own: the command
 * semantics as plain functions, usable without a manager or a GPU.
 */
#ifndef MGK_MANAGER_H
#define MGK_MANAGER_H

#include "mgk.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef MAGIK_H
/* ------------------------------------------------------------ results */
typedef int32_t e_magik_result_types;
#define MAGIK_SUCCESS 0
#define MAGIK_ERROR_NOT_RUNNING 1
#define MAGIK_ERROR_INVALID_POINTER 2
#define MAGIK_UNKNOWN_ENUM_TYPE 3
#define MAGIK_INVALID_CUDA_DEVICE 4
#define MAGIK_ERROR_DEVICE_OUT_OF_MEMORY 200
#define MAGIK_ERROR_PROVIDED_ID_NOT_FOUND 401
#define MAGIK_ERROR_COMMAND_BUFFER_OVERFLOW 402
#define MAGIK_ERROR_INVALID_COMMAND 403
#define MAGIK_ERROR_PACKED_COMMAND_NOT_ALLIGNED 404
#define MAGIK_ERROR_COMMAND_BUFFER_ALLOCATION_FAILED 406
#define MAGIK_ERROR_COMMAND_SIZE_NOT_A_MULTIPLE_OF_4 407
#define MAGIK_ERROR_OUT_OF_BOUNDS_COMMAND_BUFFER_READ 408
#define MAGIK_ERROR_UNKNOWN_METRIC 707
#define MAGIK_ERROR_AOV_INCORRECT_EXTRACT_CALL 900
#define MAGIK_ERROR_AOV_SWAPCHAIN_NOT_INITALIZED 902
#define MAGIK_ERROR_GL_LOADER_FAILED 1000
#define MAGIK_ERROR_GL_FUNCTIONS_NOT_LOADED 1001
#define MAGIK_ERROR_UNKNOWN 10000

/* ------------------------------------------------------------ manager */
typedef int32_t e_magik_manager_display_types;
#define MAGIK_DISPLAY_SWAPCHAIN 0
#define MAGIK_DISPLAY_HEADLESS 1

typedef struct magik_manager_descriptor_t {
    e_magik_manager_display_types display_type; /* MAGIK_DISPLAY_SWAPCHAIN */
    uint32_t user_device_id;                    /* 0 */
    void* user_stream;                          /* NULL: the manager creates and owns a stream */
    uint32_t cqs_n_reserved_chunk;              /* 4-byte chunks per command buffer, 4096 */
    bool cqs_drop_overflow;                     /* false */
} magik_manager_descriptor_t;

typedef struct magik_render_manager* magik_render_manager_t;

MGK_API e_magik_result_types magik_render_manager_create(magik_render_manager_t* manager,
                                                         magik_manager_descriptor_t descriptor);
MGK_API e_magik_result_types magik_render_manager_destroy(magik_render_manager_t manager);
/* The first error the worker thread met (0 while none). */
MGK_API e_magik_result_types magik_render_manager_fetch_error(magik_render_manager_t manager);

/* ------------------------------------------------------------ statistics */
/* The manager owns the history arrays; they stay valid until the next fetch
 * on the same struct or magik_destroy_renderer_statistics. */
typedef struct magik_renderer_statistics_t {
    size_t x_sample;                                  /* samples per pixel accumulated */
    double total_render_time_seconds;                 /* worker loop, since the manager started */
    double latest_render_loop_iteration_time_seconds;
    double total_wavefront_sample_time_seconds;       /* device time of the sample renders */
    double latest_wavefront_sample_time_seconds;
    size_t latest_wavefront_history_length;           /* integrator passes of the latest sample */
    uint32_t* h_latest_advance_A_queue_count_history;   /* rays entering each pass */
    uint32_t* h_latest_advance_B_queue_count_history;   /* rays going on to the next pass */
    uint32_t* h_latest_intersect_queue_count_history;   /* steps handed to the crossing kernel */
    uint32_t* h_latest_bxdf_queue_count_history;        /* rays that met matter: hits + reflections */
    uint32_t* h_latest_redistribute_queue_count_history;/* rays ending on an emitter */
    uint32_t* h_latest_splat_queue_count_history;       /* rays finished in the pass (all classes) */
    size_t total_framebuffer_swapchain_size;          /* bytes of the published and pending AOVs */
    size_t total_wavefront_buffer_size;               /* bytes of the device scratch */
} magik_renderer_statistics_t;

MGK_API e_magik_result_types magik_fetch_renderer_statistics(magik_render_manager_t manager, bool* is_new_fetch,
                                                             magik_renderer_statistics_t* dcc_statistics);
MGK_API e_magik_result_types magik_destroy_renderer_statistics(magik_renderer_statistics_t* statistics);

/* ------------------------------------------------------------ framebuffers */
typedef int32_t e_magik_framebuffer_collection_config_types;
#define MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_HOST 0
#define MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_CUDA 1
#define MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_OPENGL_INTEROP 2
#define MAGIK_FRAMEBUFFER_COLLECTION_CONFIG_VULKAN_INTEROP 3

typedef struct magik_framebuffer_collection_external* magik_framebuffer_collection_external_t;

MGK_API e_magik_result_types magik_configure_framebuffer_collection(
    magik_framebuffer_collection_external_t* framebuffer, e_magik_framebuffer_collection_config_types config_type);
/* Copies the newest published frame into the collection; *is_new_fetch is
 * false when nothing was published since the last fetch. */
MGK_API e_magik_result_types magik_framebuffer_collection_fetch(magik_render_manager_t manager, bool* is_new_fetch,
                                                                magik_framebuffer_collection_external_t framebuffer);

typedef struct magik_framebuffer_container_config_host_t {
    uint32_t x_resolution;
    uint32_t y_resolution;
    uint32_t channels;
    size_t size_of_data; /* bytes */
    float* h_data;       /* owned by the collection */
} magik_framebuffer_container_config_host_t;

MGK_API e_magik_result_types magik_extract_config_host(magik_render_manager_t manager,
                                                       magik_framebuffer_container_config_host_t* container,
                                                       magik_framebuffer_collection_external_t framebuffer,
                                                       const char* name);

typedef struct magik_framebuffer_container_config_cuda_t {
    char reserved; /* empty in the reference */
} magik_framebuffer_container_config_cuda_t;
MGK_API e_magik_result_types magik_extract_config_cuda(magik_framebuffer_container_config_cuda_t* container,
                                                       magik_framebuffer_collection_external_t framebuffer);

typedef struct magik_framebuffer_container_config_opengl_interop_t {
    uint32_t x_resolution;
    uint32_t y_resolution;
    uint32_t channels;
    uint32_t gl_buffer_id;
    void* cuda_resources;
} magik_framebuffer_container_config_opengl_interop_t;
/* No graphics stack: always MAGIK_ERROR_GL_FUNCTIONS_NOT_LOADED. */
MGK_API e_magik_result_types magik_extract_config_opengl_interop(
    magik_render_manager_t manager, magik_framebuffer_container_config_opengl_interop_t* container,
    magik_framebuffer_collection_external_t framebuffer, const char* name);

typedef struct magik_framebuffer_container_config_vulkan_interop_t {
    char reserved;
} magik_framebuffer_container_config_vulkan_interop_t;
MGK_API e_magik_result_types magik_extract_vulkan_interop(magik_framebuffer_container_config_vulkan_interop_t* container,
                                                          magik_framebuffer_collection_external_t framebuffer);
MGK_API e_magik_result_types magik_destroy_framebuffer_collection(magik_framebuffer_collection_external_t framebuffer);

/* ------------------------------------------------------------ command queue system */
typedef int32_t e_magik_cqs_command_types;
#define MAGIK_COMMAND_SET_STATE_RENDER 1000
#define MAGIK_COMMAND_SET_STATE_PAUSE 1001
#define MAGIK_COMMAND_CLEAR_RENDER_BUFFER 1002
#define MAGIK_COMMAND_ADD_AOV 1003
#define MAGIK_COMMAND_REMOVE_AOV 1004
#define MAGIK_COMMAND_PRINTF 2000
#define MAGIK_COMMAND_SET_METRIC_MINKOWSKI 4000
#define MAGIK_COMMAND_SET_METRIC_SCHWARZSCHILD 4001
#define MAGIK_COMMAND_SET_METRIC_KERR 4002
#define MAGIK_COMMAND_SET_ABSOLUTE_ERROR_TOLERANCE 4100
#define MAGIK_COMMAND_SET_RELATIVE_ERROR_TOLERANCE 4101
#define MAGIK_COMMAND_SET_MAX_SUBSTEPS 4102
#define MAGIK_COMMAND_SET_OBSERVER_LOCAL_PROPER_VELOCITY 4200
#define MAGIK_COMMAND_SET_CELESTIAL_SPHERE_RADIUS 4300
#define MAGIK_COMMAND_SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR 4400
#define MAGIK_COMMAND_SET_SCHWARZSCHILD_MASS_PARAMETER 4401
#define MAGIK_COMMAND_SET_KERR_EVENT_HORIZON_SCALAR 4402
#define MAGIK_COMMAND_SET_KERR_MASS_PARAMETER 4403
#define MAGIK_COMMAND_SET_KERR_DIMENSIONLESS_SPIN_PARAMETER 4404
#define MAGIK_COMMAND_SET_ACTIVE_CAMERA 5000
#define MAGIK_COMMAND_SET_CAMERA_POSITION 5001
#define MAGIK_COMMAND_SET_CAMERA_ORIENTATION 5002
#define MAGIK_COMMAND_SET_CAMERA_RESOLUTION 5003
#define MAGIK_COMMAND_SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN 6000
#define MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MAXIMUM_WAVELENGTH_NM 6001
#define MAGIK_COMMAND_SET_SAMPLE_DOMAIN_MINIMUM_WAVELENGTH_NM 6002
#define MAGIK_COMMAND_SET_REDISTRIBUTION_STANDARD_DEVIATION_NM 6003
#define MAGIK_COMMAND_SET_COLOR_MATCHING_FUNCTION 6100
#define MAGIK_COMMAND_SET_SCENE_COLORSPACE 6101
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM 6102
#define MAGIK_COMMAND_SET_DISPLAY_COLORSPACE 6103
#define MAGIK_COMMAND_SET_OUTPUT_FORMAT 6104
#define MAGIK_COMMAND_SET_WHITE_BALANCE_WHITE_POINT 6200
#define MAGIK_COMMAND_SET_WHITE_BALANCE_TINT 6201
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_REINHARD_EXTENDED_WHITE_LUMINANCE 6300
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_START_COMPRESSION 6301
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_DESATURATION 6302
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_MODE 6304
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_SDR_PAPER_WHITE_BALANCE 6305
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_REFERENCE_LUMINANCE 6306
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR 6407 /* the reference's value */
#define MAGIK_COMMAND_SET_VIEW_TRANSFORM_AGX_LOOK 6308
#define MAGIK_COMMAND_SET_N_GEODESIC_STEP_LIMIT 7000
#define MAGIK_COMMAND_SET_N_REFLECTED_LIMIT 7001

/* Every command struct starts with its type; all are 4-byte aligned. */
typedef struct magik_command_set_state_render_t { e_magik_cqs_command_types embedded_type; } magik_command_set_state_render_t;
typedef struct magik_command_set_state_pause_t { e_magik_cqs_command_types embedded_type; } magik_command_set_state_pause_t;
typedef struct magik_command_clear_render_buffer_t { e_magik_cqs_command_types embedded_type; } magik_command_clear_render_buffer_t;
typedef struct magik_command_add_aov_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t length_of_name;
    char name[512];
    uint32_t channels;
} magik_command_add_aov_t;
typedef struct magik_command_remove_aov_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t length_of_name;
    char name[512];
} magik_command_remove_aov_t;
typedef struct magik_command_printf_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t length_of_text;
    char text[512];
} magik_command_printf_t;
typedef struct magik_command_set_metric_minkowski_t { e_magik_cqs_command_types embedded_type; } magik_command_set_metric_minkowski_t;
typedef struct magik_command_set_metric_schwarzschild_t { e_magik_cqs_command_types embedded_type; } magik_command_set_metric_schwarzschild_t;
typedef struct magik_command_set_metric_kerr_t { e_magik_cqs_command_types embedded_type; } magik_command_set_metric_kerr_t;
typedef struct magik_command_set_absolute_error_tolerance_t { e_magik_cqs_command_types embedded_type; float absolute_error_tolerance; } magik_command_set_absolute_error_tolerance_t;
typedef struct magik_command_set_relative_error_tolerance_t { e_magik_cqs_command_types embedded_type; float relative_error_tolerance; } magik_command_set_relative_error_tolerance_t;
typedef struct magik_command_set_max_substeps_t { e_magik_cqs_command_types embedded_type; uint32_t max_substeps; } magik_command_set_max_substeps_t;
typedef struct magik_command_set_observer_local_proper_velocity_t {
    e_magik_cqs_command_types embedded_type;
    float velocity_x, velocity_y, velocity_z; /* m/s */
} magik_command_set_observer_local_proper_velocity_t;
typedef struct magik_command_set_celestial_sphere_radius_t { e_magik_cqs_command_types embedded_type; float celestial_sphere_radius; } magik_command_set_celestial_sphere_radius_t;
typedef struct magik_command_set_schwarzschild_event_horizon_scalar_t { e_magik_cqs_command_types embedded_type; float scalar; } magik_command_set_schwarzschild_event_horizon_scalar_t;
typedef struct magik_command_set_schwarzschild_mass_parameter_t { e_magik_cqs_command_types embedded_type; float mass_parameter; } magik_command_set_schwarzschild_mass_parameter_t;
typedef struct magik_command_set_kerr_event_horizon_scalar_t { e_magik_cqs_command_types embedded_type; float scalar; } magik_command_set_kerr_event_horizon_scalar_t;
typedef struct magik_command_set_kerr_mass_parameter_t { e_magik_cqs_command_types embedded_type; float mass_parameter; } magik_command_set_kerr_mass_parameter_t;
typedef struct magik_command_set_kerr_dimensionless_spin_parameter_t { e_magik_cqs_command_types embedded_type; float dimensionless_spin_parameter; } magik_command_set_kerr_dimensionless_spin_parameter_t;
typedef struct magik_command_set_active_camera_t { e_magik_cqs_command_types embedded_type; uint32_t id; } magik_command_set_active_camera_t;
typedef struct magik_command_set_camera_position_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t id;
    float position_x, position_y, position_z; /* m */
} magik_command_set_camera_position_t;
typedef struct magik_command_set_camera_orientation_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t id;
    float rotation_x, rotation_y, rotation_z; /* rad: orientation = Rx Ry Rz */
} magik_command_set_camera_orientation_t;
typedef struct magik_command_set_camera_resolution_t {
    e_magik_cqs_command_types embedded_type;
    uint32_t x_resolution, y_resolution;
} magik_command_set_camera_resolution_t;
typedef struct magik_command_set_n_intrinsic_spectral_irradiance_bin_t { e_magik_cqs_command_types embedded_type; uint32_t n_isi_bin; } magik_command_set_n_intrinsic_spectral_irradiance_bin_t;
typedef struct magik_command_set_sample_domain_maximum_wavelength_nm_t { e_magik_cqs_command_types embedded_type; float maximum_wavelength_nm; } magik_command_set_sample_domain_maximum_wavelength_nm_t;
typedef struct magik_command_set_sample_domain_minimum_wavelength_nm_t { e_magik_cqs_command_types embedded_type; float minimum_wavelength_nm; } magik_command_set_sample_domain_minimum_wavelength_nm_t;
typedef struct magik_command_set_redistribution_standard_deviation_nm_t { e_magik_cqs_command_types embedded_type; float standard_deviation_nm; } magik_command_set_redistribution_standard_deviation_nm_t;
typedef struct magik_command_set_color_matching_function_t { e_magik_cqs_command_types embedded_type; int32_t cmf_type; } magik_command_set_color_matching_function_t;
typedef struct magik_command_set_scene_colorspace_t { e_magik_cqs_command_types embedded_type; int32_t scene_colorspace; } magik_command_set_scene_colorspace_t;
typedef struct magik_command_set_view_transform_t { e_magik_cqs_command_types embedded_type; int32_t view_transform; } magik_command_set_view_transform_t;
typedef struct magik_command_set_display_colorspace_t { e_magik_cqs_command_types embedded_type; int32_t display_colorspace; } magik_command_set_display_colorspace_t;
typedef struct magik_command_set_output_format_t { e_magik_cqs_command_types embedded_type; int32_t output_format; } magik_command_set_output_format_t;
typedef struct magik_command_set_white_balance_white_point_t { e_magik_cqs_command_types embedded_type; float white_point_kelvin; } magik_command_set_white_balance_white_point_t;
typedef struct magik_command_set_white_balance_tint_t { e_magik_cqs_command_types embedded_type; float tint; } magik_command_set_white_balance_tint_t;
typedef struct magik_command_set_view_transform_reinhard_extended_white_luminance_t { e_magik_cqs_command_types embedded_type; float white_luminance; } magik_command_set_view_transform_reinhard_extended_white_luminance_t;
typedef struct magik_command_set_view_transform_khronos_pbr_neutral_start_compression_t { e_magik_cqs_command_types embedded_type; float start_compression; } magik_command_set_view_transform_khronos_pbr_neutral_start_compression_t;
typedef struct magik_command_set_view_transform_khronos_pbr_neutral_desaturation_t { e_magik_cqs_command_types embedded_type; float desaturation; } magik_command_set_view_transform_khronos_pbr_neutral_desaturation_t;
typedef struct magik_command_set_view_transform_gt7_mode_t { e_magik_cqs_command_types embedded_type; int32_t mode; } magik_command_set_view_transform_gt7_mode_t;
typedef struct magik_command_set_view_transform_gt7_sdr_paper_white_balance_t { e_magik_cqs_command_types embedded_type; float sdr_paper_white_balance; } magik_command_set_view_transform_gt7_sdr_paper_white_balance_t;
typedef struct magik_command_set_view_transform_gt7_reference_luminance_t { e_magik_cqs_command_types embedded_type; float reference_luminance; } magik_command_set_view_transform_gt7_reference_luminance_t;
typedef struct magik_command_set_view_transform_gt7_jzazbz_exponent_scale_factor_t { e_magik_cqs_command_types embedded_type; float jzazbz_exponent_scale_factor; } magik_command_set_view_transform_gt7_jzazbz_exponent_scale_factor_t;
typedef struct magik_command_set_view_transform_agx_look_t { e_magik_cqs_command_types embedded_type; int32_t look; } magik_command_set_view_transform_agx_look_t;
typedef struct magik_command_set_n_geodesic_step_limit_t { e_magik_cqs_command_types embedded_type; uint32_t n_geodesic_step_limit; } magik_command_set_n_geodesic_step_limit_t;
typedef struct magik_command_set_n_reflected_limit_t { e_magik_cqs_command_types embedded_type; uint32_t n_reflected_limit; } magik_command_set_n_reflected_limit_t;

/* Appends a command to the front buffer (copied; the struct may be reused). */
MGK_API e_magik_result_types magik_cqs_push_command(magik_render_manager_t manager, const void* command);
/* Hands the front buffer to the worker if it has consumed the previous one;
 * otherwise *is_dispatched = false and the commands stay queued. */
MGK_API e_magik_result_types magik_cqs_dispatch_command_buffer(magik_render_manager_t manager, bool* is_dispatched);

/* No graphics stack: always MAGIK_ERROR_GL_LOADER_FAILED. */
typedef void* (*magik_gl_loader_proc)(const char* name);
MGK_API e_magik_result_types magik_gl_init(magik_gl_loader_proc loader);
MGK_API e_magik_result_types magik_get_version(uint32_t* major, uint32_t* minor, uint32_t* revision,
                                               const char** as_char);
#endif /* MAGIK_H */

/* ------------------------------------------------------------ stage */
/* The settings the commands change, in the reference's units and with its
 * defaults (relativity_settings.h, optical_system_settings.h,
 * color_settings.h, render_settings.h, stage.h), plus the manager's render
 * state and AOV list. */
#define MGK_MAX_AOV 16
#define MGK_AOV_NAME_BYTES 512

typedef struct mgk_aov {
    uint32_t channels;
    uint32_t name_length;
    char name[MGK_AOV_NAME_BYTES];
} mgk_aov;

typedef struct mgk_stage {
    int32_t metric_type;              /* MGK_METRIC_KERR */
    float abs_tol;                    /* 1e-3 */
    float rel_tol;                    /* 1e-10 */
    uint32_t n_max_substep;           /* 56 */
    float observer_velocity[3];       /* m/s, proper velocity (0) */
    float celestial_sphere_radius;    /* m, 1000 */
    float schwarzschild_horizon_scalar; /* 1.01 */
    float schwarzschild_mass;         /* kg, 6.7329546075e26 */
    float kerr_horizon_scalar;        /* 1.01 */
    float kerr_mass;                  /* kg, 6.7329546075e26 */
    float kerr_spin;                  /* 0.999 */
    uint32_t active_camera;           /* 0 */
    float focal_length_mm;            /* 12 */
    float iso, fps, shutter_angle;    /* 500, 24, 180 */
    float sensor_diagonal_mm;         /* 24 */
    uint32_t x_resolution, y_resolution; /* 2195, 1860 */
    float position[3];                /* m, (2, 0, 9) */
    float orientation[9];             /* row-major, identity */
    uint32_t n_isi_bin;               /* 24 */
    float isi_max_nm, isi_min_nm;     /* 830, 360 */
    float redistribution_sigma_nm;    /* 10 */
    int32_t cmf_type;                 /* 0: CIE 1931 */
    int32_t scene_colorspace, view_transform, display_colorspace;
    int32_t output_format;            /* 5: float32 */
    float white_point, tint;          /* 5600 K, 0 */
    float reinhard_white_luminance;   /* 4 */
    float khronos_start_compression, khronos_desaturation; /* 0.8, 0.15 */
    int32_t gt7_mode;
    float gt7_sdr_paper_white, gt7_reference_luminance, gt7_jzazbz_exponent_scale; /* 250, 100, 1.7 */
    int32_t agx_look;
    uint32_t n_geodesic_step_limit;   /* 512 */
    uint32_t n_reflected_limit;       /* 10 */
    float box_min[3], box_max[3];     /* m, (-20, -10, -20), (20, 10, 20) */
    float light_min[3], light_max[3]; /* m, (-10, 9.5, -10), (10, 10.5, 10) */
    uint32_t rendering;               /* 1 (SET_STATE_RENDER) or 0 (SET_STATE_PAUSE) */
    uint32_t clear_requested;         /* a command invalidated the accumulated samples */
    uint32_t n_aov;
    mgk_aov aov[MGK_MAX_AOV];
} mgk_stage;

MGK_API void mgk_stage_defaults(mgk_stage* stage);
/* Applies the commands of a buffer of n_chunks 4-byte chunks in order
 * (command.cpp: fetch_command_info / apply_command / consume_command_buffer).
 * Returns MAGIK_ERROR_INVALID_COMMAND for an unknown type and
 * MAGIK_ERROR_OUT_OF_BOUNDS_COMMAND_BUFFER_READ for a command that runs past
 * the end; the commands before it stay applied. */
MGK_API mgk_result mgk_stage_apply(mgk_stage* stage, const uint32_t* chunks, uint32_t n_chunks);
/* Size in bytes of a command type (0: not a command). */
MGK_API uint32_t mgk_command_size(int32_t command_type);
/* The scene and display settings one sample pass of the stage renders: the
 * metric's length scale G M / c^2 turns metres into M; the camera is the
 * explicit camera at the stage's position and orientation, moving with the
 * observer's proper velocity; the stage's box and light are the room; the
 * sampled spectral sensor over [isi_min, isi_max] with n_isi_bin bins; one
 * sample per pixel with the given seed.  Returns the scene's validation
 * result (mgk_render's). */
MGK_API mgk_result mgk_stage_scene(const mgk_stage* stage, uint64_t seed, mgk_scene* scene,
                                   mgk_display_settings* display);

#ifdef __cplusplus
}
#endif

#endif /* MGK_MANAGER_H */
