// Allocation-free trace entry point: mgk_trace_rays_static.
//
// Some callers cannot allocate device memory once they are running.  A host
// application that hands the renderer a fixed share of the GPU at start-up
// and reserves the rest for its own memory pool forbids later cudaMalloc
// calls.  An interactive loop cannot afford them either: cudaMalloc and
// cudaFree may synchronise the whole device and stall the frame.  Such a
// caller cannot use mgk_trace_rays, whose context grows a scratch arena with
// cudaMalloc on first use.  This entry point runs the same kernels on a
// scratch array that lives in the library image: g_static_scratch, a
// file-scope __device__ array of kStaticBytes (8 MiB), which every device
// that loads the library holds until the process exits.  It traces at most
// kStaticMaxRays (16384) rays per call.
//
// The array's host-side name is only a stand-in: host code must not pass it
// to a kernel.  The device address comes from cudaGetSymbolAddress, taken
// once per device (with that device current) by the first call there and
// cached; that first call on a device should therefore come before any
// stream capture.  The cached address belongs to the device's current CUDA
// context: calls must not span a cudaDeviceReset (which ends that context and
// frees the module holding the array).  Every call shares the one array and
// finds the previous call's contents in it, so the counters are cleared at
// the start of each call.  Calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on the array;
// callers serialise them, for example by issuing them on one stream.
//
// The array holds no continuation queues.  mgk_trace_rays runs rays that go
// on after a room reflection or a disk miss through further passes of the
// persistent integrator; here those rays finish in the tail kernel instead.
// Both integrate the same steps in the same arithmetic, so the records are
// the same bytes (the no-allocation tests compare them, room scenes
// included); only the kernel that takes the later steps differs.
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "dev_scene.cuh"
#include "internal.h"

namespace mgk {

namespace {

constexpr uint32_t kStaticMaxRays = 16384;
constexpr size_t kStaticBytes = size_t(8) << 20;

struct StaticLayout {
    size_t qx, qp, qc, hits, refine, resume, xyz, counters, total;
};

constexpr size_t up256(size_t v) { return (v + 255) / 256 * 256; }

constexpr StaticLayout static_layout(bool f64, uint32_t n) {
    const size_t T = f64 ? 8 : 4;
    StaticLayout L{};
    size_t o = 0;
    L.qx = o; o = up256(o + size_t(n) * 4 * T);
    L.qp = o; o = up256(o + size_t(n) * 4 * T);
    L.qc = o; o = up256(o + size_t(n) * T);
    L.hits = o; o = up256(o + size_t(n) * (f64 ? sizeof(HitEntry<double>) : sizeof(HitEntry<float>)));
    L.refine = o; o = up256(o + size_t(n) * (f64 ? sizeof(RefineEntry<double>) : sizeof(RefineEntry<float>)));
    L.resume = o; o = up256(o + size_t(n) * (f64 ? sizeof(ResumeEntry<double>) : sizeof(ResumeEntry<float>)));
    L.xyz = o; o = up256(o + size_t(n) * 12);
    L.counters = o; o = up256(o + sizeof(Counters));
    L.total = o;
    return L;
}

// The documented limit must fit the array in both state widths.
static_assert(static_layout(true, kStaticMaxRays).total <= kStaticBytes, "F64 layout exceeds the static scratch");
static_assert(static_layout(false, kStaticMaxRays).total <= kStaticBytes, "FP32 layout exceeds the static scratch");

std::mutex g_mu;
void* g_addr[64] = {};

// Device address of g_static_scratch on the current device (set up once).
cudaError_t static_scratch_address(int device, void** out);

}  // namespace

// The scratch of mgk_trace_rays_static (see the top of this file).
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

namespace {
cudaError_t static_scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return cudaSuccess;
}
}  // namespace

}  // namespace mgk

using namespace mgk;

extern "C" MGK_API mgk_result mgk_trace_rays_static(const mgk_scene* s, uint64_t first_ray, uint32_t n_rays,
                                                    mgk_ray_result* d_out, void* stream) {
    if (!s || !d_out) return MGK_ERROR_INVALID_POINTER;
    mgk_result rc = validate_scene(s);
    if (rc != MGK_SUCCESS) return rc;
    if (n_rays > kStaticMaxRays) return MGK_ERROR_INVALID_ARGUMENT;
    const uint64_t total = uint64_t(s->width) * s->height * s->spp;
    if (first_ray > total || n_rays > total - first_ray) return MGK_ERROR_INVALID_ARGUMENT;
    if (n_rays == 0) return MGK_SUCCESS;
    const StaticLayout L = static_layout(s->precision == MGK_PRECISION_F64, n_rays);
    if (L.total > kStaticBytes) return MGK_ERROR_INVALID_ARGUMENT;

    int device = 0, sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
        cudaGetLastError();
        return MGK_ERROR_NO_DEVICE;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return MGK_ERROR_NO_DEVICE;
    }
    void* base = nullptr;
    if (static_scratch_address(device, &base) != cudaSuccess) {
        cudaGetLastError();
        return MGK_ERROR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* A = static_cast<char*>(base);
    ChunkBuffers B;
    B.qx = A + L.qx;
    B.qp = A + L.qp;
    B.qc = A + L.qc;
    B.hits = A + L.hits;
    B.refine = A + L.refine;
    B.resume = A + L.resume;
    B.xyz_ray = reinterpret_cast<float*>(A + L.xyz);
    B.counters = reinterpret_cast<Counters*>(A + L.counters);

    // the previous call's counters are still in the array
    if (cudaMemsetAsync(B.counters, 0, sizeof(Counters), st) != cudaSuccess) {
        cudaGetLastError();
        return MGK_ERROR_CUDA;
    }
    float w[3 * MGK_MAX_BINS];
    std::memset(w, 0, sizeof(w));
    alignas(16) unsigned char table[sizeof(DevScene<double>)];
    fill_dev_scene(*s, w, table);
    if (launch_generate(*s, table, first_ray, n_rays, B, st) != cudaSuccess ||
        launch_integrate(*s, table, first_ray, n_rays, B, d_out, sms, st) != cudaSuccess) {
        cudaGetLastError();
        return MGK_ERROR_CUDA;
    }
    return MGK_SUCCESS;
}
