// Thin C entry points over the reference's own code, compiled together with
// the reference sources into oracle/_ref (never shipped).  Mirrors the
// argument checks of magik_trace_geodesic (src/magik.cpp:196-207) and exposes
// the reference's colour-weight routine (host_color_utilities.cuh:145-178).
#include "host_trace_geodesic.h"
#include "host_color_utilities.cuh"
#include "magik.h"

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
