// Internal interfaces between the C-ABI layer (api.cu) and the kernels
// (kernels.cu).  Not installed.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mgk.h"

namespace mgk {

// Device-side counters of one integrator pass (one chunk of rays).
struct Counters {
    unsigned long long attempts;
    unsigned long long steps;
    unsigned long long wide_attempts;
    unsigned long long refine_evals;
    unsigned long long class_count[MGK_RAY_CLASSES];
    unsigned long long reflections;  // room-wall reflections
    unsigned long long crossings_prev;  // crossing-queue entries of earlier passes (room scenes)
    uint32_t cont_count[2];  // room scenes: entries in the two continuation queues
    uint32_t cont_head;      // next continuation-queue index handed to a warp
    uint32_t n_hist;         // passes recorded in hist
    // per finished pass (k_next_pass): crossings, continued rays, and the hit
    // and resume counts so far
    uint32_t hist[MGK_PASS_HISTORY][4];
    uint32_t queue_head;    // next queue index handed to a warp
    uint32_t hit_count;     // entries in the hit queue
    uint32_t refine_count;  // disk-crossing entries (from the front of the crossing queue)
    uint32_t escape_count;  // escape-crossing entries (from the back of the crossing queue)
    uint32_t resume_count;  // entries in the resume queue
    uint32_t status;        // 0 = ok; bit 0: a queue overflowed
    uint32_t fallback_count;  // surrogate renders: rays routed to RKF45
    uint32_t resume_head;     // next resume-queue index handed to a warp of the tail kernel
};

// Hit-queue entry (disk and sky rays; dark rays are not queued).
template <class T> struct alignas(16) HitEntry {
    uint32_t ray;  // index within the chunk
    uint32_t cls;
    T z, r_hit;
    T d0, d1, d2;
    T pad;
};

// Crossing-queue entry: a step whose end crossed the disk plane near the
// disk, the escape sphere or (room scene) a wall or the light; the crossing
// kernel locates it.
template <class T> struct alignas(16) RefineEntry {
    T y0[7], y1[7];
    T pt, h, h_next, c0;
    uint32_t ray, steps, attempts, wide, evals, bounces, pad[2];
};

// Resume-queue entry: a ray that continues in the tail kernel (MIXED rays
// inside the FP64 band, rays whose disk candidate missed the disk, rays
// reflected off a wall of the room).
template <class T> struct alignas(16) ResumeEntry {
    T y[7];
    T pt, h, c0;
    uint32_t ray, steps, attempts, wide, evals, bounces, pad[2];
};

// Views of the arena for one chunk.
struct ChunkBuffers {
    void* qx;              // float4 / double[4] positions
    void* qp;              // float4 / double[4] momenta (px, py, pz, pt)
    void* qc;              // float / double c0
    void* hits;            // HitEntry<T>[n]
    void* refine;          // RefineEntry<T>[n]
    void* resume;          // ResumeEntry<T>[n]
    void* cont[2] = {nullptr, nullptr};  // room scenes: ResumeEntry<T>[n] each, alternating passes
    float* xyz_ray;        // 3 floats per ray
    Counters* counters;
    const uint32_t* ray_ids = nullptr;  // queue position -> ray index (null: identity)
    uint32_t hit_cap = 0;               // hit-queue capacity (0: the launch's ray count)
};

struct StarGridDev {
    const uint32_t* cell_start;
    const uint32_t* cell_stars;
    uint32_t n;
};

// Launchers (kernels.cu).  All asynchronous on `stream`.
cudaError_t launch_generate(const mgk_scene& s, const void* dev_scene, uint64_t first_ray, uint32_t n,
                            const ChunkBuffers& b, cudaStream_t stream);
cudaError_t launch_integrate(const mgk_scene& s, const void* dev_scene, uint64_t first_ray, uint32_t n,
                             const ChunkBuffers& b, mgk_ray_result* results, int sm_count, cudaStream_t stream);
cudaError_t launch_shade(const mgk_scene& s, const void* dev_scene, uint64_t first_ray, uint32_t n,
                         const ChunkBuffers& b, const mgk_star* stars, StarGridDev grid, const float* d_w,
                         float* film_spectral, int sm_count, cudaStream_t stream);
cudaError_t launch_resolve(const mgk_scene& s, uint64_t first_pixel, uint32_t n_pixels, const float* xyz_ray,
                           float* film_xyz, cudaStream_t stream);
// Surrogate support (kernels.cu).
cudaError_t launch_generate_samples(const mgk_scene& s, const void* dev_scene, uint64_t seed, uint32_t first,
                                    uint32_t n, const ChunkBuffers& b, float* feat, cudaStream_t stream);
cudaError_t launch_labels(const mgk_ray_result* res, const float* feat, uint32_t n, void* labels, cudaStream_t stream);
cudaError_t launch_camera_features(const mgk_scene& s, const void* dev_scene, uint64_t first_ray, uint32_t n,
                                   const ChunkBuffers& b, float* feat, cudaStream_t stream);
cudaError_t launch_route(const mgk_scene& s, const void* dev_scene, uint32_t base, uint32_t n, uint32_t cap,
                         const float* out, const float* feat, float conf_min, float crit_frac, const ChunkBuffers& b,
                         uint32_t* fallback_ids, void* fallback_q, cudaStream_t stream);
// Inference of the surrogate network (surrogate.cu): 16 floats per row of out.
cudaError_t surrogate_infer(mgk_surrogate* net, const float* feat, uint32_t n, float* out, cudaStream_t stream);
uint32_t surrogate_status(mgk_surrogate* net);
int context_device(mgk_context* ctx);
size_t context_device_bytes(mgk_context* ctx);  // scratch arena and staging
mgk_result validate_scene(const mgk_scene* s);   // mgk_render's scene checks
cudaError_t launch_fma_probe(uint32_t blocks, uint32_t iters, float* sink, cudaStream_t stream);
cudaError_t launch_dfma_probe(uint32_t blocks, uint32_t iters, double* sink, cudaStream_t stream);
cudaError_t launch_check_rounding(int sm_count, unsigned long long* out, cudaStream_t stream);
cudaError_t launch_trace_geodesic(const void* jobs, uint32_t n, void* steps, uint32_t* written, cudaStream_t stream);

// Size of DevScene<T> for the scene's precision.
size_t dev_scene_size(const mgk_scene& s);
// Fills the device-scene table (host memory, dev_scene_size bytes).
void fill_dev_scene(const mgk_scene& s, const float* xyz_w, void* out);
// The tabulated CIE 1931 colour-matching functions (x, y, z) at nm, linearly
// interpolated in float (api.cu).
void cie1931_sample(float nm, float out[3]);
// The colour resolve (display.cu).
void display_defaults(mgk_display_settings* ds);
mgk_result display_prepare(const mgk_display_settings& s, mgk_display_pipeline* out);
cudaError_t launch_display(const mgk_display_pipeline& p, const float* xyz, uint64_t n, float* rgb,
                           cudaStream_t stream);
// The CIE inverse CDF table of the sampled spectral mode (api.cu):
// MGK_CMF_ICDF_ENTRIES wavelengths in nm, from the tabulated CIE 1931
// functions (or the analytic fit with `fit`).
void cmf_inverse_cdf_table(double lmin_nm, double lmax_nm, float* out, bool fit = false);

// One geodesic of the reference-compatible trace API (host-prepared inputs).
struct TraceJob {
    int32_t metric;
    int32_t n_max;
    float spin, mass_sign, horizon, spin_abs_gt1, atol, rtol;
    float length_scale;   // positions are multiplied by it at the end
    float squared_norm;   // 0 for photons, -1 for massive particles
    float x0[4];          // dimensionless start position
    float seed[3][4];     // tetrad seeds of the observer velocity (rotated camera basis)
    float w[3];           // local proper velocity / c, already sign-flipped if time reversed
    float dir[3];         // spatial direction / length scale
    uint32_t n_steps;     // capacity
    uint32_t step_offset; // first step slot in the shared step buffer
    uint32_t n_written;   // out
    uint32_t pad;
};

}  // namespace mgk
