/*
 * mgk.h - C ABI of the B200-native geodesic path (libmgk.so).
 *
 * The library integrates null geodesics with the adaptive RKF45 scheme of
 * Magik (Minkowski / Schwarzschild / Kerr in Kerr-Schild Cartesian form, spin
 * axis +y), tests every accepted step against a thin accretion disk, an escape
 * radius and the horizon, and turns the terminated rays into blackbody spectra
 * and CIE XYZ film, all on one B200 through hand-written sm_100a kernels.
 *
 * Conventions follow the reference's public API (include/magik/magik.h):
 *  - every entry point returns e_magik_result_types (magik.h:38-110); new
 *    codes live at 10001 and above; nothing ever calls exit() or resets the
 *    device (the reference's check_cuda does, cuda_host_utilities.h:12-20);
 *  - caller-owned buffers are passed as plain pointers with explicit sizes;
 *  - device work is stream-ordered on the caller's stream (NULL = legacy
 *    default stream) and asynchronous unless stated otherwise.
 * Plain C types only: no torch or CUDA types appear in the signatures.
 */
#ifndef MGK_H
#define MGK_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(__GNUC__) || defined(__clang__)
#define MGK_API __attribute__((visibility("default")))
#else
#define MGK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ results */
/* Values 0..10000 are the reference's e_magik_result_types (magik.h:38-110). */
typedef int32_t mgk_result;
#define MGK_SUCCESS 0
#define MGK_ERROR_INVALID_POINTER 2
#define MGK_UNKNOWN_ENUM_TYPE 3
#define MGK_INVALID_CUDA_DEVICE 4
#define MGK_ERROR_HOST_ALLOCATION_FAILED 101
#define MGK_ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH 102
#define MGK_ERROR_DEVICE_OUT_OF_MEMORY 200
#define MGK_ERROR_UNKNOWN_METRIC 707
#define MGK_ERROR_UNKNOWN 10000
/* New codes. */
#define MGK_ERROR_INVALID_ARGUMENT 10001  /* a size, count or range is out of bounds */
#define MGK_ERROR_CUDA 10002              /* a CUDA runtime call failed */
#define MGK_ERROR_NO_DEVICE 10003         /* no sm_100 device / kernels not loadable */
#define MGK_ERROR_DEVICE_STATUS 10004     /* a kernel reported a bad status word */

/* --------------------------------------------------------------- enums */
/* Same values as e_magik_spacetime_metric_types (magik.h:583-588). */
#define MGK_METRIC_MINKOWSKI 0
#define MGK_METRIC_SCHWARZSCHILD 1
#define MGK_METRIC_KERR 2

/* Arithmetic of the integrator.
 *  REF32 - FP32 state and FP32 step control in the reference's exact operation
 *          order (no fused multiply-add): the kernels reproduce the reference
 *          CPU tracer's steps bit for bit.
 *  MIXED - FP32 state with fused multiply-add, the step's error estimate
 *          formed over the stage differences (exact cancellation of their
 *          common part), whole attempts in FP64 within MGK_WIDE_BAND of the
 *          outer horizon.  The production mode.
 *  F64   - FP64 everywhere (the accuracy reference run on the GPU). */
#define MGK_PRECISION_REF32 0
#define MGK_PRECISION_MIXED 1
#define MGK_PRECISION_F64 2

/* Distance (in M) from the outer horizon below which MIXED attempts run in FP64. */
#define MGK_WIDE_BAND 0.05

/* Secant iterations (after the first RK sub-step to the chord estimate)
 * spent locating a disk crossing on the geodesic; an escape crossing takes
 * the first sub-step only. */
#define MGK_REFINE_ITERS 4

/* Termination class of a ray. */
#define MGK_RAY_ALIVE 0
#define MGK_RAY_DISK 1
#define MGK_RAY_ESCAPED 2
#define MGK_RAY_HORIZON 3
#define MGK_RAY_STEP_LIMIT 4  /* also: more reflections than room_reflection_limit */
#define MGK_RAY_LIGHT 5       /* the room's light (MGK_SCENE room traceables) */
#define MGK_RAY_CLASSES 6

/* ------------------------------------------------------------ scene */
/* Everything one render or trace needs.  Geometric units, M = 1.
 * The integrator fields mirror the reference's metric params_t
 * (metric_kerr.cuh:112-123) and relativity settings
 * (relativity_settings.h:11-25). */
typedef struct mgk_scene {
    int32_t metric;          /* MGK_METRIC_* */
    int32_t precision;       /* MGK_PRECISION_* */
    int32_t time_reversed;   /* 1 for camera rays (the reference's kernels trace time-reversed) */
    uint32_t n_max_substep;  /* RKF45 attempts per accepted step (reference default 56) */
    double spin;             /* Kerr a, physical (flipped internally when time_reversed) */
    double mass_sign;        /* Schwarzschild: +1 or -1 */
    double horizon_scalar;   /* capture at horizon radius * this (reference 1.01) */
    double abs_tol;
    double rel_tol;
    double h_max;            /* largest affine step (reference 1000) */
    uint32_t max_steps;      /* accepted steps per ray before MGK_RAY_STEP_LIMIT */
    uint32_t n_bins;         /* spectral bins, 1..MGK_MAX_BINS */
    double escape_radius;    /* |x| at which a ray counts as escaped; MIXED needs
                                escape_radius + 2 h_max <= 1.5e4 */
    double disk_r_in;        /* thin disk in the plane y = 0; disk_r_out <= 0 disables it */
    double disk_r_out;
    double disk_T_in;        /* T(r) = disk_T_in * (r / disk_r_in)^(-3/4) */
    double cam_r;            /* camera at cam_r * (0, cos i, sin i) */
    double cam_incl_rad;     /* inclination i from the spin axis +y */
    double focal_length_mm;  /* horizontal FOV = 2 atan(sensor_diag / (2 focal_length)) */
    double sensor_diag_mm;
    uint32_t width;
    uint32_t height;
    uint32_t spp;            /* samples per pixel; ray id = pixel * spp + sample */
    uint32_t spectral_mode;  /* MGK_SPECTRAL_BINS or MGK_SPECTRAL_SAMPLED */
    uint64_t seed;           /* counter-based RNG seed (pixel jitter, star catalogue) */
    double lambda_min_nm;    /* bins are uniform over [lambda_min, lambda_max] */
    double lambda_max_nm;
    double star_radius_rad;  /* angular radius of a star's disc on the sky, (0, 0.02] */
    /* MGK_SPECTRAL_SAMPLED only: the reference's sensor (optical_system_settings.h,
     * color_settings.h) */
    double iso;                     /* reference default 500 */
    double fps;                     /* 24 */
    double shutter_angle_deg;       /* 180 */
    double redistribution_sigma_nm; /* Gaussian spread of a sample over the bins, 10 */
    /* The reference's box-and-light test scene (stage.h:19-22, matter_examples.cuh:33-77),
     * in units of M (the reference's metres divided by its length scale 0.5 m):
     * a diffuse box the camera sits in (walls normal to x reflect like mirrors,
     * the others are Lambertian, matter_examples.cuh:38-51) and a white-LED light
     * box (matter_examples.cuh:64-76).  room_on = 0 disables both. */
    uint32_t room_on;
    uint32_t room_reflection_limit;  /* reflections before MGK_RAY_STEP_LIMIT (render_settings.h:17, 10) */
    double room_min[3], room_max[3];    /* (-40, -20, -40), (40, 20, 40) */
    double light_min[3], light_max[3];  /* (-20, 19, -20), (20, 21, 20) */
    double light_scale;                 /* white-LED spectral radiance scale, 7e5 */
    /* Explicit camera (cam_explicit = 1) in place of the orbit camera
     * (cam_r, cam_incl_rad): position and orientation as the reference's
     * optical_system_settings hold them (optical_system_settings.h:33-34),
     * in units of M; the observer moves with proper velocity cam_velocity
     * (units of c) relative to the reference observer, in its tetrad with
     * seeds x, y, z (rest_frame_four_velocity, relativity_utilities.cuh:163-173). */
    uint32_t cam_explicit;
    /* Sample slices of one frame: the scene's spp samples per pixel are the
     * frame's samples sample_offset .. sample_offset + spp - 1 (their jitter
     * and random numbers), so that renders of disjoint slices combine, in
     * proportion to their spp, into the render of the whole frame.  0 by
     * default; sample_offset + spp <= 2^32. */
    uint32_t sample_offset;
    double cam_pos[3];
    double cam_axes[9];      /* columns right, up, back (the camera looks along -back) */
    double cam_velocity[3];
} mgk_scene;

#define MGK_MAX_BINS 64

/* Spectral modes.
 *  MGK_SPECTRAL_BINS (default): the emission is evaluated at the n_bins bin
 *    centres and the film holds radiance per bin.
 *  MGK_SPECTRAL_SAMPLED: the reference renderer's stochastic mode.  Each ray
 *    draws one wavelength from the CIE inverse CDF table
 *    (device_sensor_utilities.cuh:25-33; 256 entries, built like
 *    host_color_utilities.cuh:188-233 from the tabulated CIE 1931
 *    functions), its radiance there carries the throughput 1/pdf, is turned
 *    into sensor irradiance (device_color_utilities.cuh:22-29) and spread over
 *    the bins with a Gaussian of redistribution_sigma_nm
 *    (kernel_redistribute_radiance.cu:55-92).  The film holds irradiance. */
#define MGK_SPECTRAL_BINS 0
#define MGK_SPECTRAL_SAMPLED 1
#define MGK_CMF_ICDF_ENTRIES 256

/* One background star (32 bytes). */
typedef struct mgk_star {
    float dir[3];       /* unit direction on the celestial sphere */
    float amplitude;    /* peak radiance scale (W m^-3 sr^-1 per unit Planck) */
    float temperature;  /* blackbody temperature, K */
    float reserved[3];
} mgk_star;

/* Per-ray record of mgk_trace_rays (128 bytes). */
typedef struct mgk_ray_result {
    double x[4];        /* final four-position (x, y, z, t) */
    double p[4];        /* final covariant four-momentum (x, y, z, t) */
    double z;           /* redshift factor nu_obs / nu_em (disk and sky), else 0 */
    double r_hit;       /* disk crossing radius */
    double dir[3];      /* escape direction */
    uint32_t cls;       /* MGK_RAY_* */
    uint32_t steps;     /* accepted steps */
    uint32_t attempts;  /* RKF45 attempts */
    uint32_t wide_attempts; /* attempts run in FP64 */
    uint32_t refine_evals;  /* RK sub-steps spent locating the crossing */
    uint32_t bounces;       /* reflections off the room's walls */
} mgk_ray_result;

#define MGK_PASS_HISTORY 16

/* Counters of one render. */
typedef struct mgk_render_stats {
    uint64_t rays;
    uint64_t attempts;
    uint64_t steps;
    uint64_t wide_attempts;
    uint64_t refine_evals;
    uint64_t class_count[MGK_RAY_CLASSES];  /* indexed by MGK_RAY_* */
    double integrate_ms;      /* device time of the integrator launches */
    double total_ms;          /* device time of the whole render */
    uint64_t crossings;       /* steps handed to the crossing kernel */
    uint64_t resumed;         /* rays continued by the tail kernel */
    uint64_t fallback_rays;   /* surrogate renders: rays routed to RKF45 */
    double surrogate_ms;      /* surrogate renders: device time of network + routing */
    uint64_t reflections;     /* room scene: reflections off the walls */
    /* Per integrator pass (room scenes run one pass per reflection; other
     * scenes one pass), summed over the render's chunks; passes past
     * MGK_PASS_HISTORY - 1 are added into the last entry. */
    uint32_t n_passes;
    uint32_t reserved_passes;
    uint64_t pass_rays[MGK_PASS_HISTORY];       /* rays entering the pass */
    uint64_t pass_crossings[MGK_PASS_HISTORY];  /* steps handed to the crossing kernel */
    uint64_t pass_hits[MGK_PASS_HISTORY];       /* rays ending on an emitter (disk, sky, light) */
    uint64_t pass_continued[MGK_PASS_HISTORY];  /* rays going on to the next pass */
    uint64_t pass_to_tail[MGK_PASS_HISTORY];    /* rays handed to the tail kernel */
} mgk_render_stats;

typedef struct mgk_context mgk_context;

/* ----------------------------------------------------------- context */
/* Binds a device, loads the kernels and owns the scratch arena of the
 * wavefront queues (the reference's device arena, device_arena.h:18-58). */
MGK_API mgk_result mgk_context_create(int32_t device, mgk_context** out);
MGK_API mgk_result mgk_context_destroy(mgk_context* ctx);
/* Last CUDA error text seen by the context (static storage, never NULL). */
MGK_API const char* mgk_last_error(mgk_context* ctx);

/* Defaults of the Kerr render workload: a = 0.9, camera at r = 50 M and 75 degrees
 * inclination, 60 degree horizontal field of view, 1920x1080 at 16 samples per
 * pixel, thin disk from the ISCO to 20 M at 1e4 K, 32 bins over 380-780 nm,
 * atol = rtol = 1e-7, 56 attempts per step (the reference default,
 * relativity_settings.h:13), escape radius 1000 M, MIXED precision. */
MGK_API void mgk_scene_defaults(mgk_scene* s);

/* Radius of the innermost stable circular prograde orbit for spin a (M = 1),
 * Bardeen, Press and Teukolsky (1972). */
MGK_API double mgk_isco_radius(double spin);

/* ---------------------------------------------------- host utilities */
/* Per-bin CIE 1931 XYZ weights w[3*k + c] for n_bins uniform bins over
 * [lambda_min, lambda_max] (taken as float), computed in float from the
 * tabulated CIE 1931 2-degree observer (1 nm, 360-830 nm) exactly as the
 * reference's compute_normalized_isi_cmf_weights does
 * (host_color_utilities.cuh:145-178, color_matching_functions.cuh:22-44). */
MGK_API mgk_result mgk_xyz_weights(uint32_t n_bins, double lambda_min_nm, double lambda_max_nm, float* w_out);
/* Opt-in: the same normalisation in double over the multi-lobe Gaussian fit
 * of the CIE 1931 functions (Wyman, Sloan and Shirley, JCGT 2(2), 2013);
 * within 1 % of the peak weight of mgk_xyz_weights.  No reference counterpart. */
MGK_API mgk_result mgk_xyz_weights_analytic(uint32_t n_bins, double lambda_min_nm, double lambda_max_nm, float* w_out);
/* The CIE inverse CDF table of the sampled spectral mode (MGK_SPECTRAL_SAMPLED)
 * for [lambda_min_nm, lambda_max_nm]: MGK_CMF_ICDF_ENTRIES wavelengths (nm) at
 * equidistant probabilities, built in float from the tabulated CIE 1931
 * functions as the reference's compute_tabulated_cmf_inverse_cdf
 * (host_color_utilities.cuh:188-233, floor 5 %).  Host only. */
MGK_API mgk_result mgk_cmf_inverse_cdf(double lambda_min_nm, double lambda_max_nm, float* table_out);
/* Opt-in: the same table from the analytic fit (no reference counterpart). */
MGK_API mgk_result mgk_cmf_inverse_cdf_analytic(double lambda_min_nm, double lambda_max_nm, float* table_out);

/* Seeded star catalogue: directions uniform on the sphere, magnitudes uniform
 * in [0, 10] (fluxes log-uniform over four decades), temperatures uniform in
 * [3000, 30000] K. */
MGK_API mgk_result mgk_star_catalog(uint64_t seed, uint32_t n_stars, mgk_star* out);
/* Derived per-scene constants (camera tetrad etc.), 32 doubles; for tests. */
MGK_API mgk_result mgk_scene_constants(const mgk_scene* s, double* out32);

/* Measured peak FP32 (non-tensor) throughput of the context's device in
 * FLOP/s (FMA = 2 FLOP), from a dependent-chain FMA probe kernel; the
 * denominator of the integrator's roofline.  Synchronous. */
MGK_API mgk_result mgk_fp32_peak(mgk_context* ctx, double* flops_per_s);

/* Measured peak FP64 (non-tensor) throughput in FLOP/s, from the same probe
 * with double FMA chains; the denominator of the roofline line of the FP64
 * attempts next to the horizon.  Synchronous. */
MGK_API mgk_result mgk_fp64_peak(mgk_context* ctx, double* flops_per_s);

/* Self-check of the MIXED mode's square root and reciprocal (no counterpart
 * in the reference).  The fused RHS takes them from the hardware
 * approximations with one FMA correction each; they are defined as
 *   msqrt(a) = IEEE sqrt(max(a, 2^-100)), NaN for a = +inf,
 *   mrcp(b)  = IEEE 1/b for normal b with a normal reciprocal, +-0 for
 *              |b| > 2^126, NaN for b = +-0, subnormal or infinite,
 * which the CPU oracle restates.  Evaluates both on the device for all 2^32
 * float inputs and writes the number of inputs where each differs from its
 * definition (0 on a conforming device).  Synchronous; about a millisecond. */
MGK_API mgk_result mgk_check_rounding(mgk_context* ctx, uint64_t mismatches[2]);

/* ------------------------------------------------------------- render */
/* Renders the scene's full frame: width*height*spp camera rays through the
 * persistent integrator, shading of the hit queues, per-pixel resolve.
 * d_stars (n_stars entries) and d_xyz_w (3*n_bins floats) are device
 * pointers; d_xyz_w may be NULL (then mgk_xyz_weights is used).
 * d_film_xyz receives 3 floats per pixel (X, Y, Z; mean over samples);
 * d_film_spectral, if not NULL, receives n_bins floats per pixel.
 * stats (host, may be NULL) is filled after the render completes; asking for
 * it synchronises the stream. */
MGK_API mgk_result mgk_render(mgk_context* ctx, const mgk_scene* s, const mgk_star* d_stars, uint32_t n_stars,
                              const float* d_xyz_w, float* d_film_xyz, float* d_film_spectral,
                              mgk_render_stats* stats, void* stream);

/* The same render from host memory: copies the star catalogue and weights in,
 * renders, copies the XYZ film out, and returns when the film is in h_film_xyz. */
MGK_API mgk_result mgk_render_host(mgk_context* ctx, const mgk_scene* s, const mgk_star* h_stars, uint32_t n_stars,
                                   const float* h_xyz_w, float* h_film_xyz, mgk_render_stats* stats, void* stream);

/* ------------------------------------------------------------ display */
/* The colour resolve after the XYZ film: white balance and the scene
 * colourspace, a view transform, the display colourspace and its transfer
 * function (color_pipeline.cuh:21-48, device_color_utilities.cuh:56-70,
 * view_transform.cuh, colorspaces.cuh).  The enumerations keep the
 * reference's values (magik.h:328-367). */
#define MGK_SCENE_COLORSPACE_CIE_XYZ 0
#define MGK_SCENE_COLORSPACE_CIE_RGB 1
#define MGK_SCENE_COLORSPACE_LINEAR_REC709 2
#define MGK_SCENE_COLORSPACE_LINEAR_REC2020 3
#define MGK_SCENE_COLORSPACE_ACES_CG 4
#define MGK_SCENE_COLORSPACE_ADOBE_RGB_1998 5
#define MGK_DISPLAY_COLORSPACE_SRGB 0
#define MGK_DISPLAY_COLORSPACE_REC709 1
#define MGK_DISPLAY_COLORSPACE_REC2100_PQ 2
#define MGK_DISPLAY_COLORSPACE_REC2100_HLG 3
#define MGK_DISPLAY_COLORSPACE_DCI_P3_THEATRICAL_WHITE_POINT 4
#define MGK_DISPLAY_COLORSPACE_DISPLAY_P3 5
#define MGK_DISPLAY_COLORSPACE_ADOBE_RGB 6
#define MGK_VIEW_TRANSFORM_NONE 0
#define MGK_VIEW_TRANSFORM_REINHARD_SIMPLE 1
#define MGK_VIEW_TRANSFORM_REINHARD_EXTENDED 2
#define MGK_VIEW_TRANSFORM_GRAN_TURISMO_7 3
#define MGK_VIEW_TRANSFORM_AGX 4
#define MGK_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL 5
#define MGK_GT7_MODE_ICTCP 0
#define MGK_GT7_MODE_JZAZBZ 1
#define MGK_AGX_LOOK_NONE 0
#define MGK_AGX_LOOK_GOLDEN 1
#define MGK_AGX_LOOK_PUNCHY 2

/* The colour settings of the resolve (color_settings.h:9-35; defaults from
 * mgk_display_defaults are the reference's). */
typedef struct mgk_display_settings {
    int32_t scene_colorspace;    /* MGK_SCENE_COLORSPACE_* (LINEAR_REC709) */
    int32_t view_transform;      /* MGK_VIEW_TRANSFORM_* (GRAN_TURISMO_7) */
    int32_t display_colorspace;  /* MGK_DISPLAY_COLORSPACE_* (REC709) */
    int32_t gt7_mode;            /* MGK_GT7_MODE_* (JZAZBZ) */
    int32_t agx_look;            /* MGK_AGX_LOOK_* (GOLDEN) */
    int32_t reserved;
    double white_point_K;        /* white balance: blackbody temperature (5600) */
    double tint;                 /* offset normal to the Planckian locus in CIE 1960 uv (0) */
    double reinhard_white_luminance;   /* 4 */
    double khronos_start_compression;  /* 0.8 */
    double khronos_desaturation;       /* 0.15 */
    double gt7_sdr_paper_white;        /* 250 cd/m^2 */
    double gt7_reference_luminance;    /* 100 cd/m^2 */
    double gt7_jzazbz_exponent_scale;  /* 1.7 */
} mgk_display_settings;

/* Everything the display kernel needs, prepared on the host from the
 * settings (mgk_display_prepare) or filled by the caller.  Matrices are
 * row-major 3 x 3; the colour of a pixel goes
 *   XYZ -> xyz_to_scene -> view transform -> scene_to_display -> transfer function.
 * The view transforms work in Rec.709 (Khronos PBR neutral) or Rec.2020
 * (GT7, AgX) linear light: vt_to_working / vt_from_working. */
typedef struct mgk_display_pipeline {
    int32_t view_transform, display_colorspace, gt7_mode, agx_look;
    float xyz_to_scene[9];      /* white-balanced XYZ -> scene colourspace */
    float scene_to_display[9];  /* scene colourspace -> display colourspace, with its chromatic adaptation */
    float vt_to_working[9];
    float vt_from_working[9];
    float agx_inset[9];
    float agx_outset[9];
    float luminance_weights[3]; /* scene colourspace -> Y (Reinhard extended) */
    float reinhard_white_luminance;
    float khronos_start_compression, khronos_desaturation;
    /* GT7 tone curve (view_transform.cuh:115-462) */
    float gt7_reference_luminance, gt7_jzazbz_exponent_scale;
    float gt7_peak_intensity, gt7_alpha, gt7_mid_point, gt7_linear_section, gt7_toe_strength;
    float gt7_kA, gt7_kB, gt7_kC;
    float gt7_sdr_correction, gt7_fb_luminance_target, gt7_fb_luminance_target_ucs;
    float gt7_blend_ratio, gt7_fade_start, gt7_fade_end;
    float reserved[3];
} mgk_display_pipeline;

MGK_API void mgk_display_defaults(mgk_display_settings* ds);

/* Host: the pipeline of the settings, as color_pipeline_descriptor_t::create
 * and the view transforms' make_params build it (the white point integrates
 * the blackbody against the tabulated CIE 1931 functions at their 471
 * wavelengths, as compute_white_point_xyz does). */
MGK_API mgk_result mgk_display_prepare(const mgk_display_settings* ds, mgk_display_pipeline* out);

/* Device: n_pixels XYZ triples (d_xyz, e.g. an mgk_render film) -> display
 * RGB triples (d_rgb, float32).  d_xyz and d_rgb may be the same buffer.
 * Stream-ordered.  Replaces kernel_splat_to_renderbuffer's colour part
 * (kernel_splat_to_renderbuffer.cu:37-57). */
MGK_API mgk_result mgk_display(mgk_context* ctx, const mgk_display_pipeline* p, const float* d_xyz, uint64_t n_pixels,
                               float* d_rgb, void* stream);

/* Traces camera rays [first_ray, first_ray + n_rays) of the scene and writes
 * one mgk_ray_result per ray to d_out (device pointer). */
MGK_API mgk_result mgk_trace_rays(mgk_context* ctx, const mgk_scene* s, uint64_t first_ray, uint32_t n_rays,
                                  mgk_ray_result* d_out, void* stream);

/* mgk_trace_rays without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc once running: a host
 * application that gives the renderer a fixed share of the GPU and forbids
 * later allocations, or an interactive loop that cannot take the device-wide
 * synchronisation cudaMalloc / cudaFree may cause.  No context is needed: the
 * scratch is a file-scope __device__ array of 8 MiB inside the library, held
 * by every device that loads the library until the process exits.  At most
 * MGK_STATIC_MAX_RAYS rays per call (more returns MGK_ERROR_INVALID_ARGUMENT).
 * Runs on the current device; its first call there looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture; calls must not span a cudaDeviceReset.  All calls share the
 * array: calls whose work overlaps on the GPU race, so issue them on one
 * stream.  d_out as for mgk_trace_rays.  There are no continuation queues in
 * the array: rays that go on after a room reflection or a disk miss finish
 * in the tail kernel instead of further integrator passes, with the same
 * records. */
#define MGK_STATIC_MAX_RAYS 16384
MGK_API mgk_result mgk_trace_rays_static(const mgk_scene* s, uint64_t first_ray, uint32_t n_rays,
                                         mgk_ray_result* d_out, void* stream);

/* Per-ray spectra -> XYZ of camera rays [first_ray, first_ray + n_rays):
 * 3 floats per ray into d_xyz (device).  For parity tests of the shading. */
MGK_API mgk_result mgk_shade_rays(mgk_context* ctx, const mgk_scene* s, const mgk_star* d_stars, uint32_t n_stars,
                                  const float* d_xyz_w, uint64_t first_ray, uint32_t n_rays, float* d_xyz,
                                  void* stream);

/* --------------------------------------------------- deflection surrogate */
/* A learned stand-in for the integrator: an MLP 7 -> 256 -> 256 -> 256 -> 256 -> 8
 * with SiLU activations, BF16 weights and activations, FP32 accumulation, run on
 * tensor cores by the library's own forward / backward / Adam kernels.
 * Inputs: [(r_obs - 55) / 45, cos i, sin i, 2 a / 0.998 - 1, 2 n_x, 2 n_y,
 * 4 n_z + 3], with n the photon direction in the observer's frame (camera
 * looking along -z).
 * Outputs: [disk logit, escape logit (horizon logit 0), (r_hit - 10) / 10,
 * disk redshift, escape direction minus the undeflected direction (3),
 * confidence logit].  The undeflected direction is n in the flat camera basis
 * right = +x, up = (0, sin i, -cos i), back = (0, cos i, sin i).
 * Rays with low confidence or near the critical curve go to RKF45. */
typedef struct mgk_sample_label {
    int32_t cls;    /* 0 disk, 1 escape, 2 dark */
    float r;        /* (r_hit - 10) / 10 */
    float g;        /* disk redshift factor */
    float dir[3];   /* escape direction minus the undeflected direction */
    float reserved[2];
} mgk_sample_label;

typedef struct mgk_train_config {
    uint32_t batch;          /* samples per step, multiple of 1024 (65536) */
    uint32_t epochs;         /* passes over the sample set (20) */
    float lr, beta1, beta2, eps;  /* Adam (1e-3, 0.9, 0.999, 1e-8) */
    uint64_t seed;           /* shuffling */
    float w_cls, w_r, w_g, w_dir, w_conf;  /* loss weights */
    float tol_r, tol_g, tol_dir;           /* confidence target: prediction within these */
    float lr_final;          /* cosine decay of the step size from lr to lr_final over
                                all steps (default lr_final = lr: constant) */
    uint32_t reserved;
} mgk_train_config;

typedef struct mgk_surrogate mgk_surrogate;

MGK_API void mgk_train_defaults(mgk_train_config* c);
/* Number of FP32 parameters (with the padding of the first and last layer). */
MGK_API uint64_t mgk_surrogate_param_count(void);
/* Creates a network with seeded uniform initial weights on the context's device. */
MGK_API mgk_result mgk_surrogate_create(mgk_context* ctx, uint64_t seed, mgk_surrogate** out);
MGK_API mgk_result mgk_surrogate_destroy(mgk_surrogate* net);
MGK_API mgk_result mgk_surrogate_get_params(mgk_surrogate* net, float* h_params);
MGK_API mgk_result mgk_surrogate_set_params(mgk_surrogate* net, const float* h_params);
/* n training samples (features n x 7, labels n) traced by the F64 integrator.
 * n_spin_buckets == 0: camera rays of `base` (its observer, spin and field of
 *   view), from frames seeded seed, seed + 1, ... that each cover the whole
 *   field of view: n / (width height) samples per pixel, or a coarser pixel
 *   grid over the same sensor when n is below the pixel count - a surrogate
 *   for one view.
 * n_spin_buckets >= 1: observers uniform in r [10, 100] M and inclination
 *   [0, 90] deg, directions uniform on the camera's forward hemisphere, spins
 *   uniform in [0, 0.998] over the buckets (base.spin for one bucket), disk
 *   r_in at the ISCO of each spin; needs base->escape_radius >= 100.
 * The metric, disk, escape radius and tolerances come from `base`. */
MGK_API mgk_result mgk_make_samples(mgk_context* ctx, const mgk_scene* base, uint64_t seed, uint32_t n,
                                    uint32_t n_spin_buckets, float* d_features, mgk_sample_label* d_labels,
                                    void* stream);
/* Forward pass (fused tcgen05 kernel, asynchronous): d_out receives 16 floats
 * per sample (8 outputs + padding). */
MGK_API mgk_result mgk_surrogate_forward(mgk_surrogate* net, const float* d_features, uint32_t n, float* d_out,
                                         void* stream);
/* The same forward pass on the tiled mma.sync GEMM kernels of the training
 * path (for comparisons; the fused tcgen05 kernel above is the fast path). */
MGK_API mgk_result mgk_surrogate_forward_tiled(mgk_surrogate* net, const float* d_features, uint32_t n,
                                               float* d_out, void* stream);
/* Status word of the fused inference kernel: 0, or bit 1 when one of its
 * bounded waits gave up (its outputs are then invalid).  Synchronous. */
MGK_API mgk_result mgk_surrogate_status(mgk_surrogate* net, uint32_t* status);
/* Loss and gradient of one batch (n a multiple of 1024) into host memory
 * (mgk_surrogate_param_count floats); synchronous. */
MGK_API mgk_result mgk_surrogate_gradient(mgk_surrogate* net, const mgk_train_config* cfg, const float* d_features,
                                          const mgk_sample_label* d_labels, uint32_t n, float* h_grad,
                                          float* h_loss);
/* Adam training over the sample set; h_epoch_loss (may be NULL) receives the
 * mean batch loss of each epoch.  Synchronous.  On the tensor-core path the
 * run is driven from the device (step and batch counters, tables of the
 * Adam constants and order keys) and the epochs after the first replay a
 * CUDA graph of one epoch, kept for later calls with the same data, shapes
 * and loss weights; the host waits once, at the end.  Environment (read per
 * call): MGK_SURROGATE_GRAPH=0 launches every epoch, MGK_SURROGATE_PDL=0
 * launches without programmatic dependences, MGK_SURROGATE_FUSED=0 runs the
 * forward and backward chains as two kernels, MGK_DW_CTAS=n runs the weight
 * gradients on n CTAs (default 7/8 of the SMs; read when the training buffers
 * are first sized), MGK_DW_JOBS=h,l0,l4 sets their jobs per 256-column layer,
 * for W1 and for W5 instead, MGK_CHAIN_GRID=n the layer chains on n CTAs,
 * MGK_SURROGATE_PAIRS=1 and
 * MGK_SURROGATE_CHAIN=tmem select the CTA-pair and tensor-memory layer
 * chains (the same results; slower on B200). */
MGK_API mgk_result mgk_surrogate_train(mgk_surrogate* net, const mgk_train_config* cfg, const float* d_features,
                                       const mgk_sample_label* d_labels, uint32_t n, float* h_epoch_loss,
                                       void* stream);
/* Data-parallel training, one step at a time, for one rank of several that
 * each hold a shard of the sample set: between mgk_surrogate_gradient_step and
 * mgk_surrogate_adam_step the caller sums d_grad over the ranks (an all-reduce
 * on the same stream), and every rank then takes the same Adam step.  With one
 * rank, shuffle seed cfg->seed, rows [b B, (b + 1) B) of epoch e and progress
 * (e nb + b) / (epochs nb) this is the loop of mgk_surrogate_train.
 * mgk_surrogate_shuffle: the order of the n samples for one epoch (the
 *   keyed permutation mgk_surrogate_train uses, computed on the device);
 *   stream-ordered.
 * mgk_surrogate_gradient_step: forward and backward of rows [first, first + n)
 *   of that order (n a multiple of 1024, the same n on every call for one
 *   network); the gradient of the batch mean loss into d_grad
 *   (mgk_surrogate_param_count floats), the batch mean loss added to
 *   *d_loss_sum (device).  Asynchronous.
 * mgk_surrogate_adam_step: one Adam step with gradient d_grad x grad_scale,
 *   step size from cfg's cosine schedule at `progress` in [0, 1].
 *   Asynchronous. */
MGK_API mgk_result mgk_surrogate_shuffle(mgk_surrogate* net, uint64_t seed, uint32_t epoch, uint32_t n,
                                         void* stream);
/* The first n entries of the sample order of the latest shuffle (or of the
 * latest epoch of mgk_surrogate_train), copied to the host; synchronous.
 * The order is a keyed pseudo-random permutation: a 4-round Feistel network
 * on the smallest even number of bits covering n, round keys from the
 * counter-based hash of (seed, epoch), walked back into [0, n). */
MGK_API mgk_result mgk_surrogate_order(mgk_surrogate* net, uint32_t* h_order, uint32_t n);
MGK_API mgk_result mgk_surrogate_gradient_step(mgk_surrogate* net, const mgk_train_config* cfg,
                                               const float* d_features, const mgk_sample_label* d_labels,
                                               uint32_t first, uint32_t n, float* d_grad, float* d_loss_sum,
                                               void* stream);
MGK_API mgk_result mgk_surrogate_adam_step(mgk_surrogate* net, const mgk_train_config* cfg, const float* d_grad,
                                           float grad_scale, double progress, void* stream);
/* mgk_render with the surrogate in front of the integrator: every camera ray
 * goes through the network; rays whose confidence is below conf_min, or whose
 * impact parameter lies within crit_frac of the critical curve, are
 * integrated with RKF45 (the scene's precision); the rest are shaded from the
 * network's outputs. */
MGK_API mgk_result mgk_render_surrogate(mgk_context* ctx, mgk_surrogate* net, const mgk_scene* s,
                                        const mgk_star* d_stars, uint32_t n_stars, const float* d_xyz_w,
                                        float conf_min, float crit_frac, float* d_film_xyz,
                                        mgk_render_stats* stats, void* stream);

/* ------------------------------------ reference-compatible trace API */
/* Same types and layout as magik.h:583-648; when the reference's magik.h is
 * included first its declarations are used instead. */
#ifndef MAGIK_H
typedef enum e_mgk_test_particle_types { MGK_MASSIVE = 0, MGK_MASSLESS = 1 } e_mgk_test_particle_types;

typedef struct magik_trace_geodesic_metric_parameters_t {
    int32_t metric_type; /* e_magik_spacetime_metric_types */
    bool time_reversed;
    float event_horizon_scalar;
    float schwarzschild_mass; /* kg */
    float kerr_mass;          /* kg */
    float kerr_spin;
} magik_trace_geodesic_metric_parameters_t;

typedef struct magik_trace_geodesic_integrator_parameters_t {
    unsigned int n_integrator_max_substep;
    float integrator_absolute_error_tolerance;
    float integrator_relative_error_tolerance;
} magik_trace_geodesic_integrator_parameters_t;

typedef struct magik_trace_geodesic_inital_conditions_t {
    int32_t test_particle_type; /* e_magik_test_particle_types */
    float spatial_position_x, spatial_position_y, spatial_position_z;
    float x_rotation, y_rotation, z_rotation;
    float local_proper_velocity_x, local_proper_velocity_y, local_proper_velocity_z;
    float massive_particle_speed;
} magik_trace_geodesic_inital_conditions_t;

typedef struct magik_trace_geodesic_step_t {
    float four_position[4];
    float four_momentum[4];
    float moment_derivative[4];
    float four_vector_contraction;
    float affine_parameter;
    float delta_affine_parameter;
} magik_trace_geodesic_step_t;

typedef struct magik_trace_geodesic_container_t {
    uint64_t capacity;
    uint32_t n_allocated_step;
    uint32_t n_written;
    magik_trace_geodesic_step_t* steps;
} magik_trace_geodesic_container_t;

/* Drop-in for the reference's magik_trace_geodesic (magik.h:656,
 * magik.cpp:196-207): one geodesic into a caller-owned host step array, on
 * the caller thread, synchronous.  Computed on the GPU (device 0 of the
 * calling thread's current device) with the REF32 kernels, so the steps equal
 * the reference CPU tracer's. */
MGK_API int32_t magik_trace_geodesic(magik_trace_geodesic_container_t* container,
                                     magik_trace_geodesic_inital_conditions_t initial_conditions,
                                     magik_trace_geodesic_metric_parameters_t metric_parameters,
                                     magik_trace_geodesic_integrator_parameters_t integrator_parameters);
#endif /* MAGIK_H */

/* Batch form: n geodesics, one container each, traced concurrently on the GPU
 * (one thread per geodesic). */
MGK_API mgk_result mgk_trace_geodesic_batch(mgk_context* ctx, magik_trace_geodesic_container_t* containers,
                                            const magik_trace_geodesic_inital_conditions_t* initial_conditions,
                                            const magik_trace_geodesic_metric_parameters_t* metric_parameters,
                                            const magik_trace_geodesic_integrator_parameters_t* integrator_parameters,
                                            uint32_t n);

#ifdef __cplusplus
}
#endif

#endif /* MGK_H */
