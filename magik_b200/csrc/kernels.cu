// sm_100a kernels of the geodesic path.
//
//  k_generate   camera rays -> SoA ray queue (float4 x, float4 p, c0)
//               [kernel_generate_thin_lens_ray.cu + kernel_generate_initial_conditions.cu]
//  k_integrate  persistent RKF45 integrator: each warp refills its dead lanes
//               from the HBM queue in chunks, every lane runs one attempt per
//               trip, accepted steps go through the termination tests, and
//               steps that end past a disk, escape or room crossing are
//               compacted by warp ballot into the crossing queue; in MIXED
//               mode rays entering the FP64 band are compacted into the
//               resume queue
//               [kernel_advance_geodesic.cu + kernel_intersect.cu + kernel_enforce_ray_limits.cu]
//  k_refine     locates the disk / escape / wall / light crossings handed over
//               by k_integrate on the geodesic (secant iterations over RK
//               sub-steps); reflects rays off the room's walls
//               [kernel_bxdf.cu, bxdf_utilities.cuh:139-154]
//  k_tail       resumed rays (MIXED rays inside the FP64 band near the horizon,
//               rays whose disk candidate missed, reflected rays), persistent
//               with per-lane refill
//  k_shade      one thread per hit: blackbody or white-LED emission at the bin
//               wavelengths (or the sampled wavelength), star lookup, spectral
//               film, XYZ [kernel_bxdf.cu + kernel_redistribute_radiance.cu]
//  k_resolve    per-pixel mean over samples [kernel_splat_to_renderbuffer.cu]
//  k_trace_geodesic  the reference-compatible single-geodesic trace
//               [host_trace_geodesic.cu:74-117]
//
// Compiled with -fmad=false: no multiply-add is fused unless written as mad().
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

#include "dev_pair.cuh"
#include "dev_physics.cuh"
#include "dev_scene.cuh"
#include "internal.h"

namespace mgk {

constexpr unsigned kFull = 0xffffffffu;
// 1: scenes without the room continue disk-miss rays in one more pass of the
// persistent integrator instead of the tail kernel.
#ifndef MGK_MISS_PASS
#define MGK_MISS_PASS 1
#endif
#ifndef MGK_INTEGRATE_THREADS
#define MGK_INTEGRATE_THREADS 128
#endif
#ifndef MGK_INTEGRATE_MIN_BLOCKS
#define MGK_INTEGRATE_MIN_BLOCKS 7
#endif
constexpr int kIntegrateThreads = MGK_INTEGRATE_THREADS;
// FP64 state needs about twice the registers: fewer resident blocks
constexpr int kIntegrateMinBlocksF64 = 4;
// two rays per thread (k_integrate_x2): about twice the registers as well
#ifndef MGK_X2_MIN_BLOCKS
#define MGK_X2_MIN_BLOCKS 3
#endif
// resident blocks of the crossing kernel (one thread per crossing)
#ifndef MGK_REFINE_MIN_BLOCKS
#define MGK_REFINE_MIN_BLOCKS 4
#endif
// MIXED Kerr / Schwarzschild frames run k_integrate_x2 (1) or k_integrate (0)
#ifndef MGK_MIXED_X2
#define MGK_MIXED_X2 0
#endif
constexpr uint32_t kChunk = 64;  // queue entries a warp takes per refill

template <int MODE> struct ModeT { using T = float; static constexpr Fuse F = Fuse::Fma; };
template <> struct ModeT<MGK_PRECISION_REF32> { using T = float; static constexpr Fuse F = Fuse::None; };
template <> struct ModeT<MGK_PRECISION_F64> { using T = double; static constexpr Fuse F = Fuse::Fma; };

// Queue element loads/stores.
__device__ __forceinline__ void q_store(void* base, uint32_t i, float a, float b, float c, float d) {
    reinterpret_cast<float4*>(base)[i] = make_float4(a, b, c, d);
}
__device__ __forceinline__ void q_store(void* base, uint32_t i, double a, double b, double c, double d) {
    double2* p = reinterpret_cast<double2*>(base) + 2 * size_t(i);
    p[0] = make_double2(a, b);
    p[1] = make_double2(c, d);
}
__device__ __forceinline__ void q_load(const void* base, uint32_t i, float v[4]) {
    float4 q = reinterpret_cast<const float4*>(base)[i];
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void q_load(const void* base, uint32_t i, double v[4]) {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * size_t(i);
    double2 a = p[0], b = p[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// ---------------------------------------------------------------- generate
template <int MODE>
__global__ void __launch_bounds__(256) k_generate(const DevScene<typename ModeT<MODE>::T> P, uint64_t first_ray,
                                                  uint32_t n, void* qx, void* qp, void* qc) {
    using T = typename ModeT<MODE>::T;
    constexpr Fuse F = ModeT<MODE>::F;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    S7<T> y;
    T pt, c0;
    camera_ray<F, T>(P, first_ray + i, y, pt, c0);
    q_store(qx, i, y.x, y.y, y.z, y.t);
    q_store(qp, i, y.px, y.py, y.pz, pt);
    reinterpret_cast<T*>(qc)[i] = c0;
}

// ------------------------------------------------------------ one attempt
template <int METRIC, int MODE, class T>
__device__ __forceinline__ void attempt(const DevScene<T>& P, const S7<T>& y, T pt, T h, S7<T>& y1, T& h_next,
                                        bool& ok) {
    constexpr Fuse F = ModeT<MODE>::F;
    if constexpr (metric<METRIC>::explicit_euler) {
        // explicit Euler with a fixed step, metric_minkowski.cuh:49-53
        S7<T> f;
        rhs<METRIC, F, T>(y, pt, P.m, f);
        y1 = axpy<F>(h, f, y);
        h_next = h;
        ok = true;
    } else {
        S7<T> k[6];
        rkf45_stages<METRIC, F, T>(y, pt, h, P.m, y1, k);
        if constexpr (MODE == MGK_PRECISION_REF32) {
            S7<float> e = rkf45_error<Fuse::None, float>(h, k);
            float err = rms_error<Fuse::None, float>(e, y, y1, P.m.abs_tol, P.m.rel_tol);
            float safe = err > 1e-30f ? err : 1e-30f;
            h_next = propose_h_ref(h, safe, P.m.h_max);
            ok = safe < 1.0f;
        } else if constexpr (MODE == MGK_PRECISION_MIXED) {
            control_mixed(y, y1, k, h, P.m, h_next, ok);
        } else {
            control_f64(y, y1, k, h, P.m, h_next, ok);
        }
    }
}

// FP64 attempt of the MIXED mode (state rounded back to float).
template <int METRIC>
__device__ __forceinline__ void attempt_wide(const DevScene<float>& P, const S7<float>& y, float pt, float h,
                                             S7<float>& y1, float& h_next, bool& ok) {
    S7<double> yd = cvt<double>(y), y1d;
    S7<double> k[6];
    rkf45_stages<METRIC, Fuse::Fma, double>(yd, double(pt), double(h), P.md, y1d, k);
    double hn;
    control_f64(yd, y1d, k, double(h), P.md, hn, ok);
    h_next = float(hn);
    y1 = cvt<float>(y1d);
}

// True if the KS radius of (x, y, z) lies within MGK_WIDE_BAND of r_plus.
// r_KS >= sqrt(|x|^2 - a^2): positions clearly outside skip the FP64 radius.
__device__ __forceinline__ bool in_band(const DevScene<float>& P, float x, float y, float z) {
    float q = (x * x + y * y + z * z) - P.kerr_a * P.kerr_a;
    if (q > float(P.band_pre2)) return false;
    double r = kerr_schild_r<double>(double(x), double(y), double(z), P.spin_d);
    return r - P.r_plus < MGK_WIDE_BAND;
}

template <class T>
__device__ __forceinline__ void write_result(mgk_ray_result* res, uint32_t ray, const S7<T>& y, T pt,
                                             const Term<T>& t, uint32_t steps, uint32_t att, uint32_t wide,
                                             uint32_t evals, uint32_t bounces) {
    mgk_ray_result r;
    r.x[0] = double(y.x); r.x[1] = double(y.y); r.x[2] = double(y.z); r.x[3] = double(y.t);
    r.p[0] = double(y.px); r.p[1] = double(y.py); r.p[2] = double(y.pz); r.p[3] = double(pt);
    r.z = double(t.z); r.r_hit = double(t.r_hit);
    r.dir[0] = double(t.d0); r.dir[1] = double(t.d1); r.dir[2] = double(t.d2);
    r.cls = t.cls; r.steps = steps; r.attempts = att; r.wide_attempts = wide; r.refine_evals = evals;
    r.bounces = bounces;
    res[ray] = r;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Pushes the lanes with `flag` set into a queue with one atomic per warp;
// returns this lane's slot (or ~0u when not flagged or the queue is full).
__device__ __forceinline__ uint32_t warp_push(bool flag, uint32_t* count, uint32_t cap, uint32_t* status) {
    unsigned m = __ballot_sync(kFull, flag);
    if (m == 0) return ~0u;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, uint32_t(__popc(m)));
    base = __shfl_sync(kFull, base, leader);
    if (!flag) return ~0u;
    uint32_t slot = base + __popc(m & ((1u << lane) - 1u));
    if (slot >= cap) {
        atomicOr(status, 1u);
        return ~0u;
    }
    return slot;
}

// Single-thread queue push (kernels whose threads are not warp-synchronous).
__device__ __forceinline__ uint32_t thread_push(uint32_t* count, uint32_t cap, uint32_t* status) {
    uint32_t slot = atomicAdd(count, 1u);
    if (slot >= cap) {
        atomicOr(status, 1u);
        return ~0u;
    }
    return slot;
}

template <class T>
__device__ __forceinline__ void push_hit(HitEntry<T>* hits, uint32_t slot, uint32_t ray, const Term<T>& t) {
    HitEntry<T> e;
    e.ray = ray; e.cls = t.cls; e.z = t.z; e.r_hit = t.r_hit;
    e.d0 = t.d0; e.d1 = t.d1; e.d2 = t.d2; e.pad = T(0);
    hits[slot] = e;
}

template <class T>
__device__ __forceinline__ void store_resume(ResumeEntry<T>* q, uint32_t slot, const S7<T>& y, T pt, T h, T c0,
                                             uint32_t ray, uint32_t steps, uint32_t att, uint32_t wide,
                                             uint32_t evals, uint32_t bounces) {
    ResumeEntry<T> e;
    e.y[0] = y.x; e.y[1] = y.y; e.y[2] = y.z; e.y[3] = y.t; e.y[4] = y.px; e.y[5] = y.py; e.y[6] = y.pz;
    e.pt = pt; e.h = h; e.c0 = c0;
    e.ray = ray; e.steps = steps; e.attempts = att; e.wide = wide; e.evals = evals;
    e.bounces = bounces; e.pad[0] = e.pad[1] = 0;
    q[slot] = e;
}

template <class T> __device__ __forceinline__ S7<T> s7(const T* v) {
    return S7<T>{v[0], v[1], v[2], v[3], v[4], v[5], v[6]};
}

// -------------------------------------------------------------- integrate
// Persistent: every warp loops until the queue is drained.  A lane whose
// step ends near the disk plane crossing, beyond the escape radius or (room
// scene) outside the room or near the light hands the step to the crossing
// queue; in MIXED mode a lane entering the FP64 band hands its ray to the
// resume queue.  Both pushes are warp-ballot compactions with one atomic per
// warp.
//  KIND 0: the camera-ray queue (qx, qp, qc; nq rays), no room.
//  KIND 1: the camera-ray queue of a room scene (room pre-test on).
//  KIND 2: a room scene's continuation queue of whole ray states (rays
//          reflected by the previous pass's crossing kernel), cont_in with
//          cnt->cont_count[sel] entries; nq is then only the chunk's queue
//          capacity.
//  KIND 3: the continuation queue of a scene without the room (rays whose
//          disk candidate missed the disk).
template <int METRIC, int MODE, int KIND>
__global__ void __launch_bounds__(kIntegrateThreads, MODE == MGK_PRECISION_F64 ? kIntegrateMinBlocksF64 : MGK_INTEGRATE_MIN_BLOCKS)
    k_integrate(const DevScene<typename ModeT<MODE>::T> P, uint32_t nq, const void* __restrict__ qx,
                const void* __restrict__ qp, const void* __restrict__ qc,
                RefineEntry<typename ModeT<MODE>::T>* refq, ResumeEntry<typename ModeT<MODE>::T>* resq,
                mgk_ray_result* res, Counters* cnt, const uint32_t* __restrict__ ray_ids,
                const ResumeEntry<typename ModeT<MODE>::T>* __restrict__ cont_in, uint32_t sel) {
    using T = typename ModeT<MODE>::T;
    constexpr Fuse F = ModeT<MODE>::F;
    constexpr bool CONT = KIND >= 2, ROOM = KIND == 1 || KIND == 2;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    // rays in the input queue; its head counter
    const uint32_t n_in = CONT ? min(cnt->cont_count[sel], nq) : nq;
    uint32_t* const head = CONT ? &cnt->cont_head : &cnt->queue_head;

    bool alive = false;
    S7<T> y{};
    T pt = 0, c0 = 0, h = 0;
    uint32_t ray = 0, steps = 0, tries = 0, att = 0;
    uint32_t evals = 0, bounces = 0;  // carried by continued rays (zero for camera rays)
    uint32_t cbeg = 0, cend = 0;
    bool drained = false;
    uint32_t n_att = 0, n_steps = 0;  // per lane: below 2^32 (a lane runs at most max_steps x n_max per ray)
    uint32_t n_cls[MGK_RAY_CLASSES] = {0, 0, 0, 0, 0, 0};

    for (;;) {
        // ---- refill dead lanes from the queue (warp-uniform control flow)
        unsigned dead = __ballot_sync(kFull, !alive);
        bool to_band = false;
        if (dead != 0u && !(drained && cbeg == cend)) {
            uint32_t need = __popc(dead);
            uint32_t rem = cend - cbeg;
            uint32_t nb = 0, ne = 0;
            if (need > rem && !drained) {
                uint32_t got = 0;
                if (lane == 0) got = atomicAdd(head, kChunk);
                got = __shfl_sync(kFull, got, 0);
                if (got >= n_in) {
                    drained = true;
                } else {
                    nb = got;
                    ne = min(got + kChunk, n_in);
                    if (ne == n_in) drained = true;
                }
            }
            if (!alive) {
                uint32_t rank = __popc(dead & lt);
                uint32_t idx = ~0u;
                if (rank < rem) idx = cbeg + rank;
                else if (rank - rem < ne - nb) idx = nb + (rank - rem);
                if (idx != ~0u) {
                    if constexpr (CONT) {
                        const ResumeEntry<T> e = cont_in[idx];
                        y = s7(e.y);
                        pt = e.pt; c0 = e.c0; h = e.h;
                        ray = e.ray; steps = e.steps; att = e.attempts; evals = e.evals; bounces = e.bounces;
                    } else {
                        T a[4], b[4];
                        q_load(qx, idx, a);
                        q_load(qp, idx, b);
                        y = S7<T>{a[0], a[1], a[2], a[3], b[0], b[1], b[2]};
                        pt = b[3];
                        c0 = reinterpret_cast<const T*>(qc)[idx];
                        h = P.h0;
                        ray = ray_ids ? ray_ids[idx] : idx;
                        steps = 0; att = 0;
                    }
                    tries = 0;
                    alive = true;
                    if constexpr (MODE == MGK_PRECISION_MIXED && metric<METRIC>::has_horizon)
                        to_band = in_band(P, y.x, y.y, y.z);
                }
            }
            uint32_t used_old = min(need, rem);
            if (ne > nb) {
                uint32_t used_new = min(need - used_old, ne - nb);
                cbeg = nb + used_new;
                cend = ne;
            } else {
                cbeg += used_old;
            }
        }
        if (__ballot_sync(kFull, alive) == 0u) break;

        // ---- one RKF45 attempt per live lane
        uint32_t cls = MGK_RAY_ALIVE;
        bool cross = false, disk = false;
        S7<T> y0 = y;
        T h_used = h;
        if (alive && !to_band) {
            S7<T> y1;
            T hn;
            bool ok;
            attempt<METRIC, MODE, T>(P, y, pt, h, y1, hn, ok);
            ++att; ++tries; ++n_att;
            h = hn;
            if (ok || tries >= P.m.n_max) {
                tries = 0;
                ++steps; ++n_steps;
                y = y1;
                T r2 = radius2<F>(y1);
                disk = disk_candidate<F, T>(P, y0, y1);
                if constexpr (ROOM) disk = disk || room_candidate<T>(P, y0, y1);
                cross = disk || r2 >= P.escape_r2;
                if (!cross) {
                    cls = plain_terminal<METRIC, F, T>(P, y1, r2, steps);
                    if constexpr (MODE == MGK_PRECISION_MIXED && metric<METRIC>::has_horizon) {
                        if (cls == MGK_RAY_ALIVE) to_band = in_band(P, y.x, y.y, y.z);
                    }
                }
            }
        }

        // ---- compaction of the hand-offs: disk candidates fill the crossing
        // queue from the front, escapes from the back, so that the crossing
        // kernel's warps see one kind (escapes take one sub-step, disks iterate)
        if (cls != MGK_RAY_ALIVE) {
            if (res) {
                Term<T> t{cls, T(0), T(0), T(0), T(0), T(0)};
                write_result<T>(res, ray, y, pt, t, steps, att, MODE == MGK_PRECISION_F64 ? att : 0u, evals, bounces);
            }
            ++n_cls[cls];
        }
        // one ballot skips the three pushes on the (common) trips with no hand-off
        if (__ballot_sync(kFull, cross || to_band) != 0u) {
            uint32_t slot = warp_push(cross && disk, &cnt->refine_count, nq, &cnt->status);
            uint32_t eslot = warp_push(cross && !disk, &cnt->escape_count, nq, &cnt->status);
            if (eslot != ~0u) slot = nq - 1u - eslot;
            if (slot != ~0u) {
                RefineEntry<T> e;
                e.y0[0] = y0.x; e.y0[1] = y0.y; e.y0[2] = y0.z; e.y0[3] = y0.t;
                e.y0[4] = y0.px; e.y0[5] = y0.py; e.y0[6] = y0.pz;
                e.y1[0] = y.x; e.y1[1] = y.y; e.y1[2] = y.z; e.y1[3] = y.t;
                e.y1[4] = y.px; e.y1[5] = y.py; e.y1[6] = y.pz;
                e.pt = pt; e.h = h_used; e.h_next = h; e.c0 = c0;
                e.ray = ray; e.steps = steps; e.attempts = att;
                e.wide = MODE == MGK_PRECISION_F64 ? att : 0u;
                e.evals = evals; e.bounces = bounces; e.pad[0] = e.pad[1] = 0;
                refq[slot] = e;
            }
            if constexpr (MODE == MGK_PRECISION_MIXED) {
                uint32_t bslot = warp_push(to_band, &cnt->resume_count, nq, &cnt->status);
                if (bslot != ~0u) store_resume<T>(resq, bslot, y, pt, h, c0, ray, steps, att, 0u, evals, bounces);
            }
        }
        if (cls != MGK_RAY_ALIVE || cross || to_band) alive = false;
    }

    // ---- counters: one atomic per warp and counter
    const unsigned long long w_att = warp_sum((unsigned long long)n_att);
    const unsigned long long w_steps = warp_sum((unsigned long long)n_steps);
    unsigned long long c[MGK_RAY_CLASSES];
#pragma unroll
    for (int i = 0; i < MGK_RAY_CLASSES; ++i) c[i] = warp_sum((unsigned long long)n_cls[i]);
    if (lane == 0) {
        atomicAdd(&cnt->attempts, w_att);
        atomicAdd(&cnt->steps, w_steps);
        if (MODE == MGK_PRECISION_F64) atomicAdd(&cnt->wide_attempts, w_att);
#pragma unroll
        for (int i = 1; i < MGK_RAY_CLASSES; ++i)
            if (c[i]) atomicAdd(&cnt->class_count[i], c[i]);
    }
}

// ------------------------------------------------- integrate, two rays per thread
// MIXED Kerr and Schwarzschild: k_integrate with two rays per thread (slots
// 0 and 1, the halves of every float2 in dev_pair.cuh), so that each FP32
// operation of an attempt is one packed f32x2 instruction for both rays.
// The refill, the termination tests and the hand-offs are k_integrate's,
// per slot: a warp refills its dead slots (slot 0 of every lane before slot 1)
// from chunks of the queue, and each hand-off queue gets one ballot per slot.
// Both slots run an attempt on every trip; a dead slot's result is ignored.
template <int S>
__device__ __forceinline__ void x2_refill(const DevScene<float>& P, const void* __restrict__ qx,
                                          const void* __restrict__ qp, const void* __restrict__ qc,
                                          const uint32_t* __restrict__ ray_ids, uint32_t idx, S7<F2>& y, F2& pt,
                                          F2& c0, F2& h, uint32_t& ray, bool& to_band) {
    const float4 a = reinterpret_cast<const float4*>(qx)[idx];
    const float4 b = reinterpret_cast<const float4*>(qp)[idx];
    set_slot<S>(y, S7<float>{a.x, a.y, a.z, a.w, b.x, b.y, b.z});
    set_lane<S>(pt, b.w);
    set_lane<S>(c0, reinterpret_cast<const float*>(qc)[idx]);
    set_lane<S>(h, P.h0);
    ray = ray_ids ? ray_ids[idx] : idx;
    to_band = in_band(P, a.x, a.y, a.z);
}

template <int METRIC>
__global__ void __launch_bounds__(kIntegrateThreads, MGK_X2_MIN_BLOCKS)
    k_integrate_x2(const DevScene<float> P, uint32_t nq, const void* __restrict__ qx, const void* __restrict__ qp,
                   const void* __restrict__ qc, RefineEntry<float>* refq, ResumeEntry<float>* resq,
                   mgk_ray_result* res, Counters* cnt, const uint32_t* __restrict__ ray_ids) {
    constexpr Fuse F = Fuse::Fma;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;

    bool alive[2] = {false, false};
    S7<F2> y{};
    F2 pt = b2(0.f), c0 = b2(0.f), h = b2(0.f);
    uint32_t ray[2] = {0, 0}, steps[2] = {0, 0}, tries[2] = {0, 0}, att[2] = {0, 0};
    uint32_t cbeg = 0, cend = 0;
    bool drained = false;
    uint32_t n_att = 0, n_steps = 0;
    uint32_t n_cls[MGK_RAY_CLASSES] = {0, 0, 0, 0, 0, 0};

    for (;;) {
        // ---- refill dead slots (warp-uniform control flow)
        const unsigned d0 = __ballot_sync(kFull, !alive[0]);
        const unsigned d1 = __ballot_sync(kFull, !alive[1]);
        bool to_band[2] = {false, false};
        if ((d0 | d1) != 0u && !(drained && cbeg == cend)) {
            const uint32_t n0 = __popc(d0);
            const uint32_t need = n0 + __popc(d1);
            const uint32_t rem = cend - cbeg;
            uint32_t nb = 0, ne = 0;
            if (need > rem && !drained) {
                uint32_t got = 0;
                if (lane == 0) got = atomicAdd(&cnt->queue_head, kChunk);
                got = __shfl_sync(kFull, got, 0);
                if (got >= nq) {
                    drained = true;
                } else {
                    nb = got;
                    ne = min(got + kChunk, nq);
                    if (ne == nq) drained = true;
                }
            }
            auto pick = [&](uint32_t rank) {
                if (rank < rem) return cbeg + rank;
                if (rank - rem < ne - nb) return nb + (rank - rem);
                return ~0u;
            };
            if (!alive[0]) {
                const uint32_t idx = pick(__popc(d0 & lt));
                if (idx != ~0u) {
                    x2_refill<0>(P, qx, qp, qc, ray_ids, idx, y, pt, c0, h, ray[0], to_band[0]);
                    steps[0] = 0; tries[0] = 0; att[0] = 0;
                    alive[0] = true;
                }
            }
            if (!alive[1]) {
                const uint32_t idx = pick(n0 + __popc(d1 & lt));
                if (idx != ~0u) {
                    x2_refill<1>(P, qx, qp, qc, ray_ids, idx, y, pt, c0, h, ray[1], to_band[1]);
                    steps[1] = 0; tries[1] = 0; att[1] = 0;
                    alive[1] = true;
                }
            }
            const uint32_t used_old = min(need, rem);
            if (ne > nb) {
                cbeg = nb + min(need - used_old, ne - nb);
                cend = ne;
            } else {
                cbeg += used_old;
            }
        }
        if (__ballot_sync(kFull, alive[0] || alive[1]) == 0u) break;

        // ---- one RKF45 attempt for both slots
        const S7<F2> y0 = y;
        const F2 h_used = h;
        S7<F2> y1;
        F2 hn;
        bool ok[2];
        attempt_x2<METRIC>(P.m, y, pt, h, y1, hn, ok);

        uint32_t cls[2] = {MGK_RAY_ALIVE, MGK_RAY_ALIVE};
        bool cross[2] = {false, false}, disk[2] = {false, false};
        auto accept = [&](auto sc) {
            constexpr int s = decltype(sc)::value;
            if (!(alive[s] && !to_band[s])) return;
            ++att[s]; ++tries[s]; ++n_att;
            set_lane<s>(h, lane_of<s>(hn));
            if (!(ok[s] || tries[s] >= P.m.n_max)) return;
            tries[s] = 0;
            ++steps[s]; ++n_steps;
            const S7<float> a0 = slot_of<s>(y0), a1 = slot_of<s>(y1);
            set_slot<s>(y, a1);
            const float r2 = radius2<F>(a1);
            disk[s] = disk_candidate<F, float>(P, a0, a1) || room_candidate<float>(P, a0, a1);
            cross[s] = disk[s] || r2 >= P.escape_r2;
            if (!cross[s]) {
                cls[s] = plain_terminal<METRIC, F, float>(P, a1, r2, steps[s]);
                if (cls[s] == MGK_RAY_ALIVE) to_band[s] = in_band(P, a1.x, a1.y, a1.z);
            }
        };
        accept(std::integral_constant<int, 0>{});
        accept(std::integral_constant<int, 1>{});

        auto finish = [&](auto sc) {
            constexpr int s = decltype(sc)::value;
            if (cls[s] == MGK_RAY_ALIVE) return;
            if (res) {
                Term<float> t{cls[s], 0.f, 0.f, 0.f, 0.f, 0.f};
                write_result<float>(res, ray[s], slot_of<s>(y), lane_of<s>(pt), t, steps[s], att[s], 0u, 0u, 0u);
            }
            ++n_cls[cls[s]];
        };
        finish(std::integral_constant<int, 0>{});
        finish(std::integral_constant<int, 1>{});

        // ---- hand-offs: disk candidates from the front of the crossing queue,
        // escapes from the back, FP64-band rays to the resume queue
        if (__ballot_sync(kFull, cross[0] || cross[1] || to_band[0] || to_band[1]) != 0u) {
            auto hand_off = [&](auto sc) {
                constexpr int s = decltype(sc)::value;
                uint32_t slot = warp_push(cross[s] && disk[s], &cnt->refine_count, nq, &cnt->status);
                const uint32_t eslot = warp_push(cross[s] && !disk[s], &cnt->escape_count, nq, &cnt->status);
                if (eslot != ~0u) slot = nq - 1u - eslot;
                if (slot != ~0u) {
                    const S7<float> a0 = slot_of<s>(y0), a1 = slot_of<s>(y);
                    RefineEntry<float> e;
                    e.y0[0] = a0.x; e.y0[1] = a0.y; e.y0[2] = a0.z; e.y0[3] = a0.t;
                    e.y0[4] = a0.px; e.y0[5] = a0.py; e.y0[6] = a0.pz;
                    e.y1[0] = a1.x; e.y1[1] = a1.y; e.y1[2] = a1.z; e.y1[3] = a1.t;
                    e.y1[4] = a1.px; e.y1[5] = a1.py; e.y1[6] = a1.pz;
                    e.pt = lane_of<s>(pt); e.h = lane_of<s>(h_used); e.h_next = lane_of<s>(h); e.c0 = lane_of<s>(c0);
                    e.ray = ray[s]; e.steps = steps[s]; e.attempts = att[s];
                    e.wide = 0u; e.evals = 0; e.bounces = 0; e.pad[0] = e.pad[1] = 0;
                    refq[slot] = e;
                }
                const uint32_t bslot = warp_push(to_band[s], &cnt->resume_count, nq, &cnt->status);
                if (bslot != ~0u)
                    store_resume<float>(resq, bslot, slot_of<s>(y), lane_of<s>(pt), lane_of<s>(h), lane_of<s>(c0),
                                        ray[s], steps[s], att[s], 0u, 0u, 0u);
            };
            hand_off(std::integral_constant<int, 0>{});
            hand_off(std::integral_constant<int, 1>{});
        }
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (cls[s] != MGK_RAY_ALIVE || cross[s] || to_band[s]) alive[s] = false;
    }

    const unsigned long long w_att = warp_sum((unsigned long long)n_att);
    const unsigned long long w_steps = warp_sum((unsigned long long)n_steps);
    unsigned long long c[MGK_RAY_CLASSES];
#pragma unroll
    for (int i = 0; i < MGK_RAY_CLASSES; ++i) c[i] = warp_sum((unsigned long long)n_cls[i]);
    if (lane == 0) {
        atomicAdd(&cnt->attempts, w_att);
        atomicAdd(&cnt->steps, w_steps);
#pragma unroll
        for (int i = 1; i < MGK_RAY_CLASSES; ++i)
            if (c[i]) atomicAdd(&cnt->class_count[i], c[i]);
    }
}

// -------------------------------------------------------------- crossings
// One thread per handed-off step: locate the disk / escape / room crossing,
// then emit the hit, or send the ray on when nothing ended it (a disk or
// light candidate that missed, a reflected ray): to the continuation queue
// contq (room scenes, counted by *cont_count) for the next integrator pass,
// else to the tail kernel's resume queue.
template <int METRIC, int MODE, bool ROOM>
__global__ void __launch_bounds__(128, MGK_REFINE_MIN_BLOCKS) k_refine(const DevScene<typename ModeT<MODE>::T> P,
                                                const RefineEntry<typename ModeT<MODE>::T>* __restrict__ refq,
                                                uint32_t cap, HitEntry<typename ModeT<MODE>::T>* hits,
                                                ResumeEntry<typename ModeT<MODE>::T>* resq, mgk_ray_result* res,
                                                Counters* cnt, uint32_t hit_cap,
                                                ResumeEntry<typename ModeT<MODE>::T>* contq, uint32_t* cont_count) {
    using T = typename ModeT<MODE>::T;
    constexpr Fuse F = ModeT<MODE>::F;
    const uint32_t nd = min(cnt->refine_count, cap);
    const uint32_t n = min(nd + min(cnt->escape_count, cap), cap);
    unsigned long long n_evals = 0;
    uint32_t n_cls[MGK_RAY_CLASSES] = {0, 0, 0, 0, 0, 0};
    uint32_t n_refl = 0;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    // warp-uniform trip count so the queue pushes can use warp ballots;
    // indices [0, nd) are the disk entries, the rest the escapes at the back
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint32_t v = base + lane;
        const bool valid = v < n;
        const uint32_t i = v < nd ? v : cap - 1u - (v - nd);
        Term<T> t{MGK_RAY_ALIVE, T(0), T(0), T(0), T(0), T(0)};
        RefineEntry<T> e;
        S7<T> ye{};
        uint32_t evals = 0;
        Bounce bn{0u, 0ull, false};
        if (valid) {
            e = refq[i];
            S7<T> y0 = s7(e.y0);
            S7<T> y1 = s7(e.y1);
            evals = e.evals;
            bn.count = e.bounces;
            bn.ray_id = P.ray_base + e.ray;
            t = resolve<METRIC, F, T, ROOM>(P, y0, y1, e.pt, e.h, e.c0, e.steps, bn, ye, evals);
            n_evals += evals - e.evals;
            n_refl += bn.reflected ? 1u : 0u;
        }
        // a ray that goes on (candidate missed, or reflected: restart with the first step size)
        ResumeEntry<T>* const oq = contq ? contq : resq;
        uint32_t rslot = warp_push(valid && t.cls == MGK_RAY_ALIVE, contq ? cont_count : &cnt->resume_count, cap,
                                   &cnt->status);
        if (rslot != ~0u)
            store_resume<T>(oq, rslot, ye, e.pt, bn.reflected ? P.h0 : e.h_next, e.c0, e.ray, e.steps, e.attempts,
                            e.wide, evals, bn.count);
        bool lit = valid && (t.cls == MGK_RAY_DISK || t.cls == MGK_RAY_ESCAPED || t.cls == MGK_RAY_LIGHT);
        uint32_t hslot = warp_push(lit, &cnt->hit_count, hit_cap, &cnt->status);
        if (hslot != ~0u) push_hit<T>(hits, hslot, e.ray, t);
        if (valid && t.cls != MGK_RAY_ALIVE) {
            if (res) write_result<T>(res, e.ray, ye, e.pt, t, e.steps, e.attempts, e.wide, evals, bn.count);
            ++n_cls[t.cls];
        }
    }
    if (n_evals) atomicAdd(&cnt->refine_evals, n_evals);
    if (n_refl) atomicAdd(&cnt->reflections, (unsigned long long)n_refl);
    for (int i = 1; i < MGK_RAY_CLASSES; ++i)
        if (n_cls[i]) atomicAdd(&cnt->class_count[i], (unsigned long long)n_cls[i]);
}

// Between two integrator passes of a room scene: the crossing queue's counts
// go into the running total and restart at zero, as do the continuation
// queue's head and the count of the queue the next pass's crossings write.
__global__ void k_next_pass(Counters* cnt, uint32_t next_sel) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    // the finished pass's record (the continuation queue it wrote is the other one)
    const uint32_t k = min(cnt->n_hist, uint32_t(MGK_PASS_HISTORY - 1));
    cnt->hist[k][0] += cnt->refine_count + cnt->escape_count;
    cnt->hist[k][1] += cnt->cont_count[next_sel ^ 1u];
    cnt->hist[k][2] = cnt->hit_count;
    cnt->hist[k][3] = cnt->resume_count;
    cnt->n_hist += 1u;
    cnt->crossings_prev += (unsigned long long)cnt->refine_count + cnt->escape_count;
    cnt->refine_count = 0;
    cnt->escape_count = 0;
    cnt->cont_head = 0;
    cnt->cont_count[next_sel] = 0;
}

// ------------------------------------------------------------------- tail
// Resumed rays (MIXED rays inside the FP64 band, rays whose disk candidate
// missed), run to termination.  Persistent like k_integrate: every lane
// holds one ray and takes one attempt per trip, and a warp refills its
// finished lanes from the resume queue in chunks, so that no lane waits for
// the longest ray of its warp.  MIXED mode: FP64 attempts while within
// MGK_WIDE_BAND of r_plus, FP32 otherwise.
template <int METRIC, int MODE, bool ROOM>
__global__ void __launch_bounds__(128, 4) k_tail(const DevScene<typename ModeT<MODE>::T> P,
                                              const ResumeEntry<typename ModeT<MODE>::T>* __restrict__ resq,
                                              uint32_t cap, HitEntry<typename ModeT<MODE>::T>* hits,
                                              mgk_ray_result* res, Counters* cnt, uint32_t hit_cap) {
    using T = typename ModeT<MODE>::T;
    constexpr Fuse F = ModeT<MODE>::F;
    const uint32_t n = min(cnt->resume_count, cap);
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    unsigned long long n_att = 0, n_steps = 0, n_wide = 0, n_evals = 0, n_refl = 0;
    uint32_t n_cls[MGK_RAY_CLASSES] = {0, 0, 0, 0, 0, 0};

    bool alive = false;
    S7<T> y{};
    T pt = 0, c0 = 0, h = 0;
    uint32_t ray = 0, steps = 0, att = 0, wide = 0, evals = 0, tries = 0;
    Bounce bn{0u, 0ull, false};
    double r_cur = 0.0;
    uint32_t cbeg = 0, cend = 0;
    bool drained = false;

    for (;;) {
        // ---- refill finished lanes (warp-uniform control flow)
        const unsigned dead = __ballot_sync(kFull, !alive);
        if (dead != 0u && !(drained && cbeg == cend)) {
            const uint32_t need = __popc(dead);
            const uint32_t rem = cend - cbeg;
            uint32_t nb = 0, ne = 0;
            if (need > rem && !drained) {
                uint32_t got = 0;
                if (lane == 0) got = atomicAdd(&cnt->resume_head, kChunk);
                got = __shfl_sync(kFull, got, 0);
                if (got >= n) {
                    drained = true;
                } else {
                    nb = got;
                    ne = min(got + kChunk, n);
                    if (ne == n) drained = true;
                }
            }
            if (!alive) {
                const uint32_t rank = __popc(dead & lt);
                uint32_t idx = ~0u;
                if (rank < rem) idx = cbeg + rank;
                else if (rank - rem < ne - nb) idx = nb + (rank - rem);
                if (idx != ~0u) {
                    const ResumeEntry<T> e = resq[idx];
                    y = s7(e.y);
                    pt = e.pt; c0 = e.c0; h = e.h;
                    ray = e.ray; steps = e.steps; att = e.attempts; wide = e.wide; evals = e.evals;
                    bn.count = e.bounces;
                    bn.ray_id = P.ray_base + e.ray;
                    tries = 0;
                    if constexpr (MODE == MGK_PRECISION_MIXED)
                        r_cur = kerr_schild_r<double>(double(y.x), double(y.y), double(y.z), P.spin_d);
                    alive = true;
                }
            }
            const uint32_t used_old = min(need, rem);
            if (ne > nb) {
                cbeg = nb + min(need - used_old, ne - nb);
                cend = ne;
            } else {
                cbeg += used_old;
            }
        }
        if (__ballot_sync(kFull, alive) == 0u) break;

        // ---- one attempt per live lane
        Term<T> t{MGK_RAY_ALIVE, T(0), T(0), T(0), T(0), T(0)};
        bool done = false;
        if (alive) {
            S7<T> y1;
            T hn;
            bool ok;
            const T h_used = h;
            bool w = false;
            if constexpr (MODE == MGK_PRECISION_MIXED && metric<METRIC>::has_horizon) {
                w = r_cur - P.r_plus < MGK_WIDE_BAND;
                if (w) attempt_wide<METRIC>(P, y, pt, h, y1, hn, ok);
                else attempt<METRIC, MODE, T>(P, y, pt, h, y1, hn, ok);
            } else {
                attempt<METRIC, MODE, T>(P, y, pt, h, y1, hn, ok);
            }
            ++att; ++tries; ++n_att;
            if (w || MODE == MGK_PRECISION_F64) { ++wide; ++n_wide; }
            h = hn;
            if (ok || tries >= P.m.n_max) {
                tries = 0;
                ++steps; ++n_steps;
                S7<T> ye;
                const uint32_t ev0 = evals;
                t = resolve<METRIC, F, T, ROOM>(P, y, y1, pt, h_used, c0, steps, bn, ye, evals);
                n_evals += evals - ev0;
                y = ye;
                if (bn.reflected) {
                    h = P.h0;
                    ++n_refl;
                }
                if (t.cls != MGK_RAY_ALIVE) done = true;
                else if constexpr (MODE == MGK_PRECISION_MIXED)
                    r_cur = kerr_schild_r<double>(double(y.x), double(y.y), double(y.z), P.spin_d);
            }
        }

        // ---- finished rays: hit queue (one ballot per warp) and per-ray records
        const bool lit = done && (t.cls == MGK_RAY_DISK || t.cls == MGK_RAY_ESCAPED || t.cls == MGK_RAY_LIGHT);
        const uint32_t hslot = warp_push(lit, &cnt->hit_count, hit_cap, &cnt->status);
        if (hslot != ~0u) push_hit<T>(hits, hslot, ray, t);
        if (done) {
            if (res) write_result<T>(res, ray, y, pt, t, steps, att, wide, evals, bn.count);
            ++n_cls[t.cls];
            alive = false;
        }
    }
    if (n_att) {
        atomicAdd(&cnt->attempts, n_att);
        atomicAdd(&cnt->steps, n_steps);
        atomicAdd(&cnt->wide_attempts, n_wide);
    }
    if (n_evals) atomicAdd(&cnt->refine_evals, n_evals);
    if (n_refl) atomicAdd(&cnt->reflections, n_refl);
    for (int i = 1; i < MGK_RAY_CLASSES; ++i)
        if (n_cls[i]) atomicAdd(&cnt->class_count[i], (unsigned long long)n_cls[i]);
}

// ------------------------------------------------------------------ shade
// One thread per hit (a warp shades 32 hits at once, so the dependent loads of
// the entry, the star cell and the stars overlap across lanes).  The boosted
// blackbody I(lambda_obs) = B(z lambda_obs, T) z^5 is evaluated as
//   a / (exp(b / (z T)) - 1),  a = 2 h c^2 / lambda^5,  b = h c / (k_B lambda),
// since the z^5 of the boost cancels the z^-5 of B at the shifted wavelength:
// one exponential and one quotient per wavelength.
//  MGK_SPECTRAL_BINS: the emission at every bin centre (a_k, b_k and the XYZ
//    weights staged in shared memory); the film holds radiance per bin.
//  MGK_SPECTRAL_SAMPLED: the reference's stochastic sensor.  The ray's
//    wavelength comes from the CIE inverse CDF (device_sensor_utilities.cuh:
//    25-33, u = rng(seed, sample, pixel, 2)) with throughput 1/pdf; its
//    radiance times throughput times the sensor gain is the sampled
//    irradiance (device_color_utilities.cuh:22-29), spread over the bins by
//    the Gaussian CDF differences at the bin edges
//    (kernel_redistribute_radiance.cu:55-92).
//  ROOM: the scene has the room's light (a separate instantiation, so that
//    scenes without it run the disk and star code alone).
template <class T, bool ROOM>
__global__ void __launch_bounds__(256) k_shade(const DevScene<T> P, const HitEntry<T>* __restrict__ hits,
                                               uint32_t cap, const Counters* cnt, const mgk_star* __restrict__ stars,
                                               StarGridDev grid, const float* __restrict__ d_w,
                                               float* __restrict__ xyz_ray, float* __restrict__ film_spec,
                                               uint64_t first_ray) {
    // per bin: the XYZ weights as one 16-byte and the Planck factors as one
    // 8- or 16-byte shared-memory load
    struct alignas(2 * sizeof(T)) PlanckAB { T a, b; };
    __shared__ float4 sw[MGK_MAX_BINS];
    __shared__ PlanckAB sab[MGK_MAX_BINS];
    __shared__ float sicdf[MGK_CMF_ICDF_ENTRIES];
    const uint32_t nb = P.n_bins;
    const bool sampled = P.spectral_mode == MGK_SPECTRAL_SAMPLED;
    for (uint32_t i = threadIdx.x; i < MGK_MAX_BINS; i += blockDim.x) {
        float4 w4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < nb) {
            const float* src = d_w ? d_w : P.xyz_w;
            w4 = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.f);
        }
        sw[i] = w4;
        // float: b_k log2(e), for exp(b_k u) = 2^(b_k log2(e) u) in one ex2
        sab[i] = PlanckAB{P.planck_a[i],
                          std::is_same_v<T, float> ? T(P.planck_b[i] * T(1.4426950408889634)) : P.planck_b[i]};
    }
    for (uint32_t i = threadIdx.x; i < MGK_CMF_ICDF_ENTRIES; i += blockDim.x) sicdf[i] = sampled ? P.cmf_icdf[i] : 0.f;
    __syncthreads();
    const uint32_t n = min(cnt->hit_count, cap);
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const HitEntry<T> h = hits[e];
        const uint64_t ray_id = first_ray + h.ray;
        float X = 0.f, Y = 0.f, Z = 0.f;
        float* spec = film_spec ? film_spec + (ray_id / P.spp) * nb : nullptr;
        // sampled mode: the ray's wavelength, throughput and Planck factors there
        T lam = T(0), tput = T(0), a_s = T(0), b_s = T(0), rad = T(0);
        if (sampled) {
            const uint32_t pixel = uint32_t(ray_id / P.spp), sample = uint32_t(ray_id % P.spp) + P.sample_offset;
            const float x = rng_unit(P.seed, sample, pixel, 2) * float(MGK_CMF_ICDF_ENTRIES - 1);
            const uint32_t k = uint32_t(fminf(x, float(MGK_CMF_ICDF_ENTRIES) - 2.0f));
            const float f = x - float(k);
            const float t0 = sicdf[k], t1 = sicdf[k + 1];
            lam = T((t0 * (1.0f - f)) + (t1 * f));  // lerp, internal_math.h:2040-2043
            tput = T(float(MGK_CMF_ICDF_ENTRIES - 1) * (t1 - t0));
            const T lm = lam * T(1e-9), l2 = lm * lm, l4 = l2 * l2, l5 = l4 * lm;
            a_s = P.planck_c1 / l5;
            b_s = P.planck_c2 / lm;
        }
        auto add = [&](T amp, T temp) {
            const T u = T(1) / (h.z * temp);
            if (sampled) {
                rad += clamp_radiance<T>(amp * (a_s / (exp(b_s * u) - T(1))));
                return;
            }
            for (uint32_t k = 0; k < nb; ++k) {
                const PlanckAB ab = sab[k];
                float sv;
                if constexpr (std::is_same_v<T, float>) {
                    // ex2.approx and the corrected reciprocal: a few ulp, far
                    // inside the film's 1e-4 (b_k u >= 0.2 for every emitter here,
                    // so e - 1 loses at most 2^-23 / 0.2 to cancellation).  e = 1
                    // or inf gives NaN, cleared by the clamp like the quotient's inf / 0.
                    const float e = ex2_approx(ab.b * u);
                    sv = clamp_radiance<float>(amp * (ab.a * mrcp(e - 1.0f)));
                } else {
                    sv = float(clamp_radiance<T>(amp * (ab.a / (exp(ab.b * u) - T(1)))));
                }
                const float4 w = sw[k];
                X = __fmaf_rn(sv, w.x, X);
                Y = __fmaf_rn(sv, w.y, Y);
                Z = __fmaf_rn(sv, w.z, Z);
                if (spec) atomicAdd(spec + k, sv * P.inv_spp);
            }
        };
        // the emission of the matter the ray ended on (src/renderer/bxdf/matter.cuh)
        if (h.cls == MGK_RAY_DISK) {
            matter<MGK_RAY_DISK>::blackbodies(P, h, stars, grid, add);
        } else if (ROOM && h.cls == MGK_RAY_LIGHT) {
            // spectral radiance at the shifted wavelength, boosted by z^5
            // (matter_examples.cuh:67-76, bxdf_utilities.cuh:156-163)
            using L = matter<MGK_RAY_LIGHT>;
            const T z2 = h.z * h.z, z5 = z2 * z2 * h.z;
            if (sampled) {
                rad = clamp_radiance<T>(L::radiance<T>(P, h.z * lam) * z5);
            } else {
                for (uint32_t k = 0; k < nb; ++k) {
                    float sv = float(clamp_radiance<T>(L::radiance<T>(P, h.z * P.lambda[k]) * z5));
                    const float4 w = sw[k];
                    X = __fmaf_rn(sv, w.x, X);
                    Y = __fmaf_rn(sv, w.y, Y);
                    Z = __fmaf_rn(sv, w.z, Z);
                    if (spec) atomicAdd(spec + k, sv * P.inv_spp);
                }
            }
        } else {
            matter<MGK_RAY_ESCAPED>::blackbodies(P, h, stars, grid, add);  // the hit queue holds no other class
        }
        if (sampled) {
            const T irr = (rad * tput) * P.sensor_gain;
            if (irr > T(0)) {
                T phi0 = T(0.5) * (T(1) + erf((P.lambda_lo - lam) * P.inv_sigma_sqrt2));
                for (uint32_t k = 0; k < nb; ++k) {
                    const T e1 = P.lambda_lo + T(k + 1) * P.dlambda;
                    const T phi1 = T(0.5) * (T(1) + erf((e1 - lam) * P.inv_sigma_sqrt2));
                    const float sv = float(irr * (phi1 - phi0));
                    phi0 = phi1;
                    const float4 w = sw[k];
                    X = __fmaf_rn(sv, w.x, X);
                    Y = __fmaf_rn(sv, w.y, Y);
                    Z = __fmaf_rn(sv, w.z, Z);
                    if (spec) atomicAdd(spec + k, sv * P.inv_spp);
                }
            }
        }
        xyz_ray[3 * size_t(h.ray) + 0] = X;
        xyz_ray[3 * size_t(h.ray) + 1] = Y;
        xyz_ray[3 * size_t(h.ray) + 2] = Z;
    }
}

// ---------------------------------------------------------------- resolve
__global__ void __launch_bounds__(256) k_resolve(uint64_t first_pixel, uint32_t n_pixels, uint32_t spp,
                                                 const float* __restrict__ xyz_ray, float* __restrict__ film) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pixels) return;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    const float* src = xyz_ray + 3 * size_t(i) * spp;
    for (uint32_t s = 0; s < spp; ++s) {
        a0 += src[3 * s + 0];
        a1 += src[3 * s + 1];
        a2 += src[3 * s + 2];
    }
    float fs = float(spp);
    float* dst = film + 3 * (first_pixel + i);
    dst[0] = a0 / fs;
    dst[1] = a1 / fs;
    dst[2] = a2 / fs;
}

// --------------------------------------------------------- trace_geodesic
// One geodesic of the reference trace in the metric with tag METRIC.
template <int METRIC>
__device__ __forceinline__ uint32_t trace_geodesic_one(const TraceJob& J, magik_trace_geodesic_step_t* st) {
    using MT = metric<METRIC>;
    MP<float> m{};
    m.spin = J.spin; m.mass_sign = J.mass_sign; m.horizon = J.horizon; m.spin_abs_gt1 = J.spin_abs_gt1;
    m.h_max = 1000.0f; m.abs_tol = J.atol; m.rel_tol = J.rtol; m.n_max = uint32_t(J.n_max);
    set_spin_consts(m);
    V4<float> x0{J.x0[0], J.x0[1], J.x0[2], J.x0[3]};
    Sym4<float> g = MT::template compute_g<float>(x0.x, x0.y, x0.z, m);
    V4<float> u_ref = MT::template reference_observer<float>(x0.x, x0.y, x0.z, m);
    V4<float> X{J.seed[0][0], J.seed[0][1], J.seed[0][2], J.seed[0][3]};
    V4<float> Yv{J.seed[1][0], J.seed[1][1], J.seed[1][2], J.seed[1][3]};
    V4<float> Z{J.seed[2][0], J.seed[2][1], J.seed[2][2], J.seed[2][3]};
    Tetrad<float> e = build_tetrad<float>(g, X, Yv, Z, u_ref);
    float w2 = J.w[0] * J.w[0] + J.w[1] * J.w[1] + J.w[2] * J.w[2];
    V4<float> u = local_to_global<float>(e, V4<float>{J.w[0], J.w[1], J.w[2], sqrtf(w2 - -1.0f)});
    Tetrad<float> e2 = build_tetrad<float>(g, V4<float>{1, 0, 0, 0}, V4<float>{0, 1, 0, 0}, V4<float>{0, 0, 1, 0}, u);
    float d2 = J.dir[0] * J.dir[0] + J.dir[1] * J.dir[1] + J.dir[2] * J.dir[2];
    V4<float> p_up = local_to_global<float>(e2, V4<float>{J.dir[0], J.dir[1], J.dir[2], sqrtf(d2 - J.squared_norm)});
    V4<float> p0 = contract<float>(g, p_up);

    S7<float> y{x0.x, x0.y, x0.z, x0.t, p0.x, p0.y, p0.z};
    float pt = p0.t;
    const float contraction = dot4<float>(u, p0);
    float h = float(MT::initial_h_step());
    float aff = 0.0f;
    auto put = [&](uint32_t k, const S7<float>& s, const S7<float>& ds) {
        magik_trace_geodesic_step_t o;
        o.four_position[0] = s.x; o.four_position[1] = s.y; o.four_position[2] = s.z; o.four_position[3] = s.t;
        o.four_momentum[0] = s.px; o.four_momentum[1] = s.py; o.four_momentum[2] = s.pz; o.four_momentum[3] = pt;
        o.moment_derivative[0] = ds.px; o.moment_derivative[1] = ds.py; o.moment_derivative[2] = ds.pz;
        o.moment_derivative[3] = 0.0f;
        o.four_vector_contraction = contraction;
        o.affine_parameter = aff;
        o.delta_affine_parameter = h;
        st[k] = o;
    };
    S7<float> ys;
    rhs<METRIC, Fuse::None, float>(y, pt, m, ys);
    put(0, y, ys);
    uint32_t nw = 1;
    while (nw < J.n_steps) {
        S7<float> y1;
        float h_taken = h;
        if constexpr (MT::explicit_euler) {
            S7<float> f;
            rhs<METRIC, Fuse::None, float>(y, pt, m, f);
            y1 = axpy<Fuse::None>(h, f, y);
        } else {
            float temp_h = h;
            for (uint32_t a = 0; a < m.n_max; ++a) {
                S7<float> k[6];
                rkf45_stages<METRIC, Fuse::None, float>(y, pt, temp_h, m, y1, k);
                S7<float> er = rkf45_error<Fuse::None, float>(temp_h, k);
                float err = rms_error<Fuse::None, float>(er, y, y1, m.abs_tol, m.rel_tol);
                float safe = err > 1e-30f ? err : 1e-30f;
                float hn = propose_h_ref(temp_h, safe, m.h_max);
                h_taken = temp_h;
                temp_h = hn;
                if (safe < 1.0f) break;
            }
            h = temp_h;
        }
        y = y1;
        rhs<METRIC, Fuse::None, float>(y, pt, m, ys);
        aff = aff + h_taken;
        put(nw, y, ys);
        ++nw;
        if (MT::has_horizon && in_domain<METRIC, float>(y.x, y.y, y.z, m)) break;
    }
    for (uint32_t k = 0; k < nw; ++k)
        for (int c = 0; c < 4; ++c) st[k].four_position[c] *= J.length_scale;
    return nw;
}

// host_trace_geodesic.cu:13-130 on the GPU, REF32 arithmetic, one thread per
// geodesic; the observer set-up that needs sin/cos is done on the host.
__global__ void __launch_bounds__(64) k_trace_geodesic(const TraceJob* __restrict__ jobs, uint32_t n,
                                                       magik_trace_geodesic_step_t* steps_all, uint32_t* written) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TraceJob J = jobs[i];
    magik_trace_geodesic_step_t* st = steps_all + J.step_offset;
    uint32_t nw = 0;
    with_metric(J.metric, [&](auto mt) { nw = trace_geodesic_one<decltype(mt)::tag>(J, st); });
    written[i] = nw;
}

// Device-scene table passed by value to the kernels.
template <class T> static const DevScene<T>& ds(const void* p) { return *reinterpret_cast<const DevScene<T>*>(p); }

// ------------------------------------------------------------- surrogate
// Features of the surrogate network, shared by training and rendering:
// [(r_obs - 55) / 45, cos i, sin i, 2 a / 0.998 - 1, 2 n_x, 2 n_y, 4 n_z + 3]
// with n the photon's direction in the observer's frame (camera looks along
// -z); the direction is scaled so that a camera's field of view spans O(1).
__device__ __forceinline__ void write_features(float* f, double r_obs, double ci, double si, double spin, double nx,
                                               double ny, double nz) {
    f[0] = float((r_obs - 55.0) / 45.0);
    f[1] = float(ci);
    f[2] = float(si);
    f[3] = float(2.0 * spin / 0.998 - 1.0);
    f[4] = float(2.0 * nx);
    f[5] = float(2.0 * ny);
    f[6] = float(4.0 * nz + 3.0);
}

// Training samples: each ray has its own observer (r in [10, 100] M,
// inclination in [0, 90] degrees) and a direction uniform on the camera's
// forward hemisphere; the spin is the launch's.  The observer tetrad is built
// per ray in double, like scene_consts does once per frame.
template <int MODE>
__global__ void __launch_bounds__(128) k_generate_samples(const DevScene<typename ModeT<MODE>::T> P, uint64_t seed,
                                                          uint32_t first, uint32_t n, void* qx, void* qp, void* qc,
                                                          float* feat) {
    using T = typename ModeT<MODE>::T;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = first + i;
    const double u0 = rng_unit(seed, 0x5A3Bu, id, 0), u1 = rng_unit(seed, 0x5A3Bu, id, 1);
    const double u2 = rng_unit(seed, 0x5A3Bu, id, 2), u3 = rng_unit(seed, 0x5A3Bu, id, 3);
    const double r_obs = 10.0 + 90.0 * u0, incl = 0.5 * 3.14159265358979323846 * u1;
    const double ci = cos(incl), si = sin(incl);
    const double ct = u2, st = sqrt(fmax(0.0, 1.0 - ct * ct)), ph = 2.0 * 3.14159265358979323846 * u3;
    const double nx = st * cos(ph), ny = st * sin(ph), nz = -ct;
    V4<double> q{0.0, r_obs * ci, r_obs * si, 0.0};
    V4<double> X{1, 0, 0, 0}, Y{0, si, -ci, 0}, Z{0, ci, si, 0};
    V4<double> u{};
    Sym4<double> g{};
    with_metric(P.metric, [&](auto mt) {
        using MT = decltype(mt);
        u = MT::template reference_observer<double>(q.x, q.y, q.z, P.md);
        g = MT::template compute_g<double>(q.x, q.y, q.z, P.md);
    });
    Tetrad<double> e = build_tetrad<double>(g, X, Y, Z, u);
    V4<double> pu = local_to_global<double>(e, V4<double>{nx, ny, nz, 1.0});
    V4<double> p = contract<double>(g, pu);
    q_store(qx, i, T(q.x), T(q.y), T(q.z), T(0));
    q_store(qp, i, T(p.x), T(p.y), T(p.z), T(p.t));
    reinterpret_cast<T*>(qc)[i] = T(dot4<double>(u, p));
    write_features(feat + size_t(i) * 7, r_obs, ci, si, double(P.spin_phys), nx, ny, nz);
}

cudaError_t launch_generate_samples(const mgk_scene& s, const void* dsc, uint64_t seed, uint32_t first, uint32_t n,
                                    const ChunkBuffers& b, float* feat, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    if (s.precision == MGK_PRECISION_F64)
        k_generate_samples<MGK_PRECISION_F64><<<(n + 127) / 128, 128, 0, st>>>(ds<double>(dsc), seed, first, n, b.qx,
                                                                               b.qp, b.qc, feat);
    else if (s.precision == MGK_PRECISION_MIXED)
        k_generate_samples<MGK_PRECISION_MIXED><<<(n + 127) / 128, 128, 0, st>>>(ds<float>(dsc), seed, first, n, b.qx,
                                                                                 b.qp, b.qc, feat);
    else
        k_generate_samples<MGK_PRECISION_REF32><<<(n + 127) / 128, 128, 0, st>>>(ds<float>(dsc), seed, first, n, b.qx,
                                                                                 b.qp, b.qc, feat);
    return cudaGetLastError();
}

// Undeflected direction of a photon from its features: the camera-frame
// direction n in the flat camera basis right = +x, up = (0, sin i, -cos i),
// back = (0, cos i, sin i).  The network predicts the escape direction as a
// residual from it, which is small away from the black hole.
__device__ __forceinline__ void flat_direction(const float* f, float d[3]) {
    const float ci = f[1], si = f[2], nx = 0.5f * f[4], ny = 0.5f * f[5], nz = 0.25f * (f[6] - 3.0f);
    d[0] = nx;
    d[1] = ny * si + nz * ci;
    d[2] = -ny * ci + nz * si;
}

// Labels of the traced samples (layout of mgk_sample_label); feat holds the
// samples' features (7 floats each).
__global__ void k_labels(const mgk_ray_result* __restrict__ res, const float* __restrict__ feat, uint32_t n,
                         mgk_sample_label* __restrict__ lab) {
    static_assert(sizeof(mgk_sample_label) == 32, "label layout");
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const mgk_ray_result r = res[i];
    mgk_sample_label L;
    L.cls = r.cls == MGK_RAY_DISK ? 0 : (r.cls == MGK_RAY_ESCAPED ? 1 : 2);
    L.r = r.cls == MGK_RAY_DISK ? float((r.r_hit - 10.0) / 10.0) : 0.f;
    L.g = r.cls == MGK_RAY_DISK ? float(r.z) : 0.f;
    float d0[3];
    flat_direction(feat + size_t(i) * 7, d0);
    for (int k = 0; k < 3; ++k) L.dir[k] = r.cls == MGK_RAY_ESCAPED ? float(r.dir[k] - double(d0[k])) : 0.f;
    L.reserved[0] = L.reserved[1] = 0.f;
    lab[i] = L;
}

cudaError_t launch_labels(const mgk_ray_result* res, const float* feat, uint32_t n, void* labels, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_labels<<<(n + 255) / 256, 256, 0, st>>>(res, feat, n, reinterpret_cast<mgk_sample_label*>(labels));
    return cudaGetLastError();
}

// Features of the camera rays of a frame (same direction as camera_ray).
template <class T>
__global__ void k_camera_features(const DevScene<T> P, uint64_t first_ray, uint32_t n, float* feat) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t ray_id = first_ray + i;
    const uint32_t pixel = uint32_t(ray_id / P.spp), sample = uint32_t(ray_id % P.spp) + P.sample_offset;
    const uint32_t px = pixel % P.width, py = pixel / P.width;
    const double sx = (double(px) + rng_unit(P.seed, sample, pixel, 0)) * double(P.pix_a) + double(P.pix_b);
    const double sy = (double(py) + rng_unit(P.seed, sample, pixel, 1)) * double(P.pix_c) + double(P.pix_d);
    const double len = sqrt(sx * sx + sy * sy + 1.0);
    const double cy = double(P.cam[1]), cz = double(P.cam[2]);
    const double r = sqrt(cy * cy + cz * cz);
    write_features(feat + size_t(i) * 7, r, cy / r, cz / r, double(P.spin_phys), sx / len, sy / len, -1.0 / len);
}

cudaError_t launch_camera_features(const mgk_scene& s, const void* dsc, uint64_t first, uint32_t n,
                                   const ChunkBuffers&, float* feat, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    if (s.precision == MGK_PRECISION_F64) k_camera_features<double><<<(n + 255) / 256, 256, 0, st>>>(ds<double>(dsc), first, n, feat);
    else k_camera_features<float><<<(n + 255) / 256, 256, 0, st>>>(ds<float>(dsc), first, n, feat);
    return cudaGetLastError();
}

// Distance of a photon's conserved quantities from the Kerr critical curve.
// lambda = L/E, eta = Q/E^2 from the Kerr-Schild state (spin axis y; the
// oblate-spheroidal theta has dx^i/dtheta = (x cot, r-sin, z cot) terms);
// the critical curve is the spherical photon orbits' (Bardeen 1973):
//   lambda_c(r) = -(r^3 - 3 r^2 + a^2 r + a^2) / (a (r - 1)),
//   eta_c(r)    = r^3 (4 a^2 - r (r - 3)^2) / (a^2 (r - 1)^2),
// r between the prograde and retrograde circular photon orbits.  Returns
// |b - b_c| / b_c with b = sqrt(eta + lambda^2) (1e30 when lambda lies
// outside the curve's range).
__device__ __forceinline__ double critical_distance(double x, double y, double z, double px, double py, double pz,
                                                    double pt, double a) {
    const double E = -pt, L = z * px - x * pz;
    const double r = kerr_schild_r<double>(x, y, z, a);
    const double ct = y / r, st2 = fmax(1e-300, 1.0 - ct * ct), st = sqrt(st2);
    const double pth = (ct / st) * (x * px + z * pz) - r * st * py;
    const double Q = pth * pth + ct * ct * (L * L / st2 - a * a * E * E);
    const double lam = L / E, eta = Q / (E * E), b = sqrt(fmax(0.0, eta + lam * lam));
    if (fabs(a) < 1e-3) {
        const double bc = sqrt(27.0);
        return fabs(b - bc) / bc;
    }
    const double aa = fabs(a);
    double r1 = 2.0 * (1.0 + cos(2.0 / 3.0 * acos(-aa))), r2 = 2.0 * (1.0 + cos(2.0 / 3.0 * acos(aa)));
    auto lc = [&](double rr) { return -(rr * rr * rr - 3.0 * rr * rr + a * a * rr + a * a) / (a * (rr - 1.0)); };
    double l1 = lc(r1), l2 = lc(r2);
    if (!((lam - l1) * (lam - l2) <= 0.0)) return 1e30;
    for (int it = 0; it < 60; ++it) {
        double rm = 0.5 * (r1 + r2), lm = lc(rm);
        if ((lm - lam) * (l1 - lam) > 0.0) { r1 = rm; l1 = lm; } else { r2 = rm; }
    }
    const double rs = 0.5 * (r1 + r2);
    const double etac = rs * rs * rs * (4.0 * a * a - rs * (rs - 3.0) * (rs - 3.0)) / (a * a * (rs - 1.0) * (rs - 1.0));
    const double bc = sqrt(fmax(1e-300, etac + lam * lam));
    return fabs(b - bc) / bc;
}

// Routing of a frame chunk after the surrogate's forward pass: rays with low
// confidence or near the critical curve go to the RKF45 fallback queue
// (compacted by warp ballot, with their ray index); the others become hits
// straight from the network's outputs.
template <int MODE>
__global__ void __launch_bounds__(256) k_route(const DevScene<typename ModeT<MODE>::T> P, uint32_t base_ray, uint32_t n,
                                               uint32_t cap, const float* __restrict__ out,
                                               const float* __restrict__ feat, float conf_min,
                                               float crit_frac, const void* __restrict__ qx,
                                               const void* __restrict__ qp, const void* __restrict__ qc, void* fqx,
                                               void* fqp, void* fqc, uint32_t* fallback_ids,
                                               HitEntry<typename ModeT<MODE>::T>* hits, Counters* cnt) {
    using T = typename ModeT<MODE>::T;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane;
        const uint32_t ray = base_ray + i;
        const bool valid = i < n;
        bool fall = false, lit = false;
        Term<T> t{MGK_RAY_ALIVE, T(0), T(0), T(0), T(0), T(0)};
        T a4[4] = {T(0), T(0), T(0), T(0)}, b4[4] = {T(0), T(0), T(0), T(0)}, c0 = T(0);
        if (valid) {
            const float* o = out + size_t(i) * 16;
            q_load(qx, ray, a4);
            q_load(qp, ray, b4);
            c0 = reinterpret_cast<const T*>(qc)[ray];
            const float conf = 1.0f / (1.0f + expf(-o[7]));
            const double dc = critical_distance(double(a4[0]), double(a4[1]), double(a4[2]), double(b4[0]),
                                                double(b4[1]), double(b4[2]), double(b4[3]), P.spin_d);
            fall = conf < conf_min || dc < double(crit_frac);
            if (!fall) {
                const int cls = (o[0] >= o[1] && o[0] >= 0.f) ? 0 : (o[1] >= 0.f ? 1 : 2);
                if (cls == 0) {
                    t.cls = MGK_RAY_DISK;
                    t.r_hit = T(10.0f + 10.0f * o[2]);
                    t.z = T(o[3]);
                    lit = t.r_hit >= P.disk_r_in && t.r_hit <= P.disk_r_out;
                } else if (cls == 1) {
                    float d[3];
                    flat_direction(feat + size_t(i) * 7, d);
                    d[0] += o[4]; d[1] += o[5]; d[2] += o[6];
                    const float dn = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    t.cls = MGK_RAY_ESCAPED;
                    t.d0 = T(d[0] / dn); t.d1 = T(d[1] / dn); t.d2 = T(d[2] / dn);
                    t.z = redshift_clamp<T>(c0 / b4[3]);
                    lit = true;
                }
            }
        }
        uint32_t fslot = warp_push(valid && fall, &cnt->fallback_count, cap, &cnt->status);
        if (fslot != ~0u) {
            q_store(fqx, fslot, a4[0], a4[1], a4[2], a4[3]);
            q_store(fqp, fslot, b4[0], b4[1], b4[2], b4[3]);
            reinterpret_cast<T*>(fqc)[fslot] = c0;
            fallback_ids[fslot] = ray;
        }
        uint32_t hslot = warp_push(lit, &cnt->hit_count, cap, &cnt->status);
        if (hslot != ~0u) push_hit<T>(hits, hslot, ray, t);
    }
}

cudaError_t launch_route(const mgk_scene& s, const void* dsc, uint32_t base, uint32_t n, uint32_t cap,
                         const float* out, const float* feat, float conf_min, float crit_frac, const ChunkBuffers& b,
                         uint32_t* fallback_ids, void* fallback_q, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const bool f64 = s.precision == MGK_PRECISION_F64;
    const size_t T = f64 ? 8 : 4;
    char* fq = static_cast<char*>(fallback_q);
    void* fqx = fq;
    void* fqp = fq + size_t(cap) * 4 * T;
    void* fqc = fq + size_t(cap) * 8 * T;
    const uint32_t blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    if (f64)
        k_route<MGK_PRECISION_F64><<<blocks, 256, 0, st>>>(ds<double>(dsc), base, n, cap, out, feat, conf_min, crit_frac,
                                                           b.qx, b.qp, b.qc, fqx, fqp, fqc, fallback_ids,
                                                           reinterpret_cast<HitEntry<double>*>(b.hits), b.counters);
    else
        k_route<MGK_PRECISION_MIXED><<<blocks, 256, 0, st>>>(ds<float>(dsc), base, n, cap, out, feat, conf_min, crit_frac,
                                                             b.qx, b.qp, b.qc, fqx, fqp, fqc, fallback_ids,
                                                             reinterpret_cast<HitEntry<float>*>(b.hits), b.counters);
    return cudaGetLastError();
}

// --------------------------------------------------------------- FP32 probe
// Peak FP32 throughput: 8 independent FMA chains per thread, enough warps to
// hide the pipeline latency.  Each loop trip is 8 FMA = 16 FLOP per thread.
__global__ void __launch_bounds__(256) k_fma_probe(uint32_t iters, float seed, float* sink) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.999999f, c = 1e-7f;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 = __fmaf_rn(a0, m, c); a1 = __fmaf_rn(a1, m, c); a2 = __fmaf_rn(a2, m, c); a3 = __fmaf_rn(a3, m, c);
            a4 = __fmaf_rn(a4, m, c); a5 = __fmaf_rn(a5, m, c); a6 = __fmaf_rn(a6, m, c); a7 = __fmaf_rn(a7, m, c);
        }
    }
    float r = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (r == 12345.f) sink[threadIdx.x] = r;
}

// Peak FP64 throughput, the same shape with double FMA chains: each loop trip
// is 8 DFMA = 16 FLOP per thread.
__global__ void __launch_bounds__(256) k_dfma_probe(uint32_t iters, double seed, double* sink) {
    double a0 = seed + threadIdx.x, a1 = a0 + 1.0, a2 = a0 + 2.0, a3 = a0 + 3.0;
    double a4 = a0 + 4.0, a5 = a0 + 5.0, a6 = a0 + 6.0, a7 = a0 + 7.0;
    const double m = 0.999999999, c = 1e-12;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 = __fma_rn(a0, m, c); a1 = __fma_rn(a1, m, c); a2 = __fma_rn(a2, m, c); a3 = __fma_rn(a3, m, c);
            a4 = __fma_rn(a4, m, c); a5 = __fma_rn(a5, m, c); a6 = __fma_rn(a6, m, c); a7 = __fma_rn(a7, m, c);
        }
    }
    double r = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (r == 12345.0) sink[threadIdx.x] = r;
}

// ----------------------------------------------------- rounding self-check
// msqrt / mrcp (dev_physics.cuh) against their definitions, on every one of
// the 2^32 float inputs: the definitions use the IEEE-rounded __fsqrt_rn and
// __frcp_rn with the stated clamp and special values.  out[0] / out[1]
// receive the number of inputs where msqrt / mrcp differ (NaNs compare equal).
__device__ __forceinline__ float msqrt_definition(float a) {
    a = fmaxf(a, kSqrtFloor);
    if (isinf(a)) return __int_as_float(0x7fc00000);
    return __fsqrt_rn(a);
}
__device__ __forceinline__ float mrcp_definition(float b) {
    const float ab = fabsf(b);
    if (isnan(b) || ab < 1.17549435e-38f || isinf(b)) return __int_as_float(0x7fc00000);
    if (ab > 8.507059173023462e37f) return copysignf(0.0f, b);  // 1/b subnormal: |b| > 2^126
    return __frcp_rn(b);
}
__device__ __forceinline__ bool same_bits(float a, float b) {
    return __float_as_uint(a) == __float_as_uint(b) || (isnan(a) && isnan(b));
}
__global__ void __launch_bounds__(256) k_check_rounding(unsigned long long* out) {
    unsigned long long bad_s = 0, bad_r = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (1ull << 32); i += stride) {
        const float a = __uint_as_float(uint32_t(i));
        bad_s += !same_bits(msqrt(a), msqrt_definition(a));
        bad_r += !same_bits(mrcp(a), mrcp_definition(a));
    }
    bad_s = warp_sum(bad_s);
    bad_r = warp_sum(bad_r);
    if ((threadIdx.x & 31) == 0) {
        if (bad_s) atomicAdd(&out[0], bad_s);
        if (bad_r) atomicAdd(&out[1], bad_r);
    }
}

cudaError_t launch_check_rounding(int sms, unsigned long long* out, cudaStream_t st) {
    k_check_rounding<<<sms * 8, 256, 0, st>>>(out);
    return cudaGetLastError();
}

cudaError_t launch_fma_probe(uint32_t blocks, uint32_t iters, float* sink, cudaStream_t st) {
    k_fma_probe<<<blocks, 256, 0, st>>>(iters, 1.0f, sink);
    return cudaGetLastError();
}

cudaError_t launch_dfma_probe(uint32_t blocks, uint32_t iters, double* sink, cudaStream_t st) {
    k_dfma_probe<<<blocks, 256, 0, st>>>(iters, 1.0, sink);
    return cudaGetLastError();
}

// =============================================================== launchers

template <int MODE>
static cudaError_t gen_t(const void* dev_scene, uint64_t first, uint32_t n, const ChunkBuffers& b, cudaStream_t st) {
    using T = typename ModeT<MODE>::T;
    k_generate<MODE><<<(n + 255) / 256, 256, 0, st>>>(ds<T>(dev_scene), first, n, b.qx, b.qp, b.qc);
    return cudaGetLastError();
}

cudaError_t launch_generate(const mgk_scene& s, const void* dev_scene, uint64_t first, uint32_t n,
                            const ChunkBuffers& b, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    switch (s.precision) {
        case MGK_PRECISION_REF32: return gen_t<MGK_PRECISION_REF32>(dev_scene, first, n, b, st);
        case MGK_PRECISION_MIXED: return gen_t<MGK_PRECISION_MIXED>(dev_scene, first, n, b, st);
        default: return gen_t<MGK_PRECISION_F64>(dev_scene, first, n, b, st);
    }
}

template <int METRIC, int MODE, bool ROOM>
static cudaError_t integ_t(const void* dsc, uint64_t first, uint32_t n, const ChunkBuffers& b, mgk_ray_result* res,
                           int sms, cudaStream_t st) {
    using T = typename ModeT<MODE>::T;
    DevScene<T> P = ds<T>(dsc);
    P.ray_base = first;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_integrate<METRIC, MODE, 0>, kIntegrateThreads, 0);
    if (per_sm < 1) per_sm = 1;
    const uint32_t full = uint32_t(sms * per_sm);
    uint32_t blocks = full;
    uint32_t need = (n + kIntegrateThreads - 1) / kIntegrateThreads;
    if (blocks > need) blocks = need;
    auto* refq = reinterpret_cast<RefineEntry<T>*>(b.refine);
    auto* resq = reinterpret_cast<ResumeEntry<T>*>(b.resume);
    auto* hits = reinterpret_cast<HitEntry<T>*>(b.hits);
    ResumeEntry<T>* cont[2] = {reinterpret_cast<ResumeEntry<T>*>(b.cont[0]),
                               reinterpret_cast<ResumeEntry<T>*>(b.cont[1])};
    // with continuation queues, rays that go on after the crossing kernel
    // (room scenes: reflected rays and light misses; other scenes: disk
    // misses) go back through the integrator: one pass per reflection plus
    // one in room scenes, one pass otherwise; the last pass's crossing
    // kernel sends what still goes on to the tail kernel
    uint32_t passes = 0;
    if constexpr (ROOM) passes = (cont[0] && cont[1]) ? P.room_limit + 1u : 0u;
    else passes = (MGK_MISS_PASS && cont[1]) ? 1u : 0u;
    if constexpr (MGK_MIXED_X2 && MODE == MGK_PRECISION_MIXED && (METRIC == MGK_METRIC_KERR || METRIC == MGK_METRIC_SCHWARZSCHILD)) {
        // two rays per thread: half the threads for the same rays
        per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_integrate_x2<METRIC>, kIntegrateThreads, 0);
        if (per_sm < 1) per_sm = 1;
        blocks = uint32_t(sms * per_sm);
        need = (n + 2 * kIntegrateThreads - 1) / (2 * kIntegrateThreads);
        if (blocks > need) blocks = need;
        k_integrate_x2<METRIC><<<blocks, kIntegrateThreads, 0, st>>>(P, n, b.qx, b.qp, b.qc, refq, resq, res,
                                                                     b.counters, b.ray_ids);
    } else {
        k_integrate<METRIC, MODE, ROOM ? 1 : 0><<<blocks, kIntegrateThreads, 0, st>>>(
            P, n, b.qx, b.qp, b.qc, refq, resq, res, b.counters, b.ray_ids, nullptr, 0u);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint32_t hit_cap = b.hit_cap ? b.hit_cap : n;
    int refine_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&refine_per_sm, k_refine<METRIC, MODE, ROOM>, 128, 0);
    if (refine_per_sm < 1) refine_per_sm = 1;
    const uint32_t refine_blocks = uint32_t(sms * refine_per_sm * 2);
    // pass p reads continuation queue p & 1 and its crossings write queue (p + 1) & 1
    k_refine<METRIC, MODE, ROOM><<<refine_blocks, 128, 0, st>>>(P, refq, n, hits, resq, res, b.counters, hit_cap,
                                                          passes ? cont[1] : nullptr, &b.counters->cont_count[1]);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    for (uint32_t p = 1; p <= passes; ++p) {
        const uint32_t in = p & 1u, out = (p + 1u) & 1u;
        k_next_pass<<<1, 32, 0, st>>>(b.counters, out);
        k_integrate<METRIC, MODE, ROOM ? 2 : 3><<<full, kIntegrateThreads, 0, st>>>(
            P, n, nullptr, nullptr, nullptr, refq, resq, res, b.counters, nullptr, cont[in], in);
        k_refine<METRIC, MODE, ROOM><<<refine_blocks, 128, 0, st>>>(P, refq, n, hits, resq, res, b.counters, hit_cap,
                                                              p < passes ? cont[out] : nullptr,
                                                              &b.counters->cont_count[out]);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    int tail_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tail_per_sm, k_tail<METRIC, MODE, ROOM>, 128, 0);
    if (tail_per_sm < 1) tail_per_sm = 1;
    k_tail<METRIC, MODE, ROOM><<<sms * tail_per_sm, 128, 0, st>>>(P, resq, n, hits, res, b.counters, hit_cap);
    return cudaGetLastError();
}

template <int MODE>
static cudaError_t integ_m(int metric, bool room, const void* dsc, uint64_t first, uint32_t n, const ChunkBuffers& b,
                           mgk_ray_result* res, int sms, cudaStream_t st) {
    // the reference's dispatch_list over supported_metrics
    cudaError_t e = cudaErrorInvalidValue;
    with_metric(metric, [&](auto mt) {
        constexpr int TAG = decltype(mt)::tag;
        e = room ? integ_t<TAG, MODE, true>(dsc, first, n, b, res, sms, st)
                 : integ_t<TAG, MODE, false>(dsc, first, n, b, res, sms, st);
    });
    return e;
}

cudaError_t launch_integrate(const mgk_scene& s, const void* dsc, uint64_t first, uint32_t n, const ChunkBuffers& b,
                             mgk_ray_result* res, int sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    switch (s.precision) {
        case MGK_PRECISION_REF32:
            return integ_m<MGK_PRECISION_REF32>(s.metric, s.room_on != 0, dsc, first, n, b, res, sms, st);
        case MGK_PRECISION_MIXED:
            return integ_m<MGK_PRECISION_MIXED>(s.metric, s.room_on != 0, dsc, first, n, b, res, sms, st);
        default: return integ_m<MGK_PRECISION_F64>(s.metric, s.room_on != 0, dsc, first, n, b, res, sms, st);
    }
}

template <class T, bool ROOM>
static void shade_t(const void* dsc, uint64_t first, uint32_t n, const ChunkBuffers& b, const mgk_star* stars,
                    StarGridDev grid, const float* d_w, float* film_spec, uint32_t blocks, cudaStream_t st) {
    k_shade<T, ROOM><<<blocks, 256, 0, st>>>(ds<T>(dsc), reinterpret_cast<const HitEntry<T>*>(b.hits), n, b.counters,
                                             stars, grid, d_w, b.xyz_ray, film_spec, first);
}

cudaError_t launch_shade(const mgk_scene& s, const void* dsc, uint64_t first, uint32_t n, const ChunkBuffers& b,
                         const mgk_star* stars, StarGridDev grid, const float* d_w, float* film_spec, int sms,
                         cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t blocks = uint32_t(sms) * 8u;
    const bool room = s.room_on != 0;
    if (s.precision == MGK_PRECISION_F64) {
        if (room) shade_t<double, true>(dsc, first, n, b, stars, grid, d_w, film_spec, blocks, st);
        else shade_t<double, false>(dsc, first, n, b, stars, grid, d_w, film_spec, blocks, st);
    } else {
        if (room) shade_t<float, true>(dsc, first, n, b, stars, grid, d_w, film_spec, blocks, st);
        else shade_t<float, false>(dsc, first, n, b, stars, grid, d_w, film_spec, blocks, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_resolve(const mgk_scene& s, uint64_t first_pixel, uint32_t n_pixels, const float* xyz_ray,
                           float* film, cudaStream_t st) {
    if (n_pixels == 0) return cudaSuccess;
    k_resolve<<<(n_pixels + 255) / 256, 256, 0, st>>>(first_pixel, n_pixels, s.spp, xyz_ray, film);
    return cudaGetLastError();
}

cudaError_t launch_trace_geodesic(const void* jobs, uint32_t n, void* steps, uint32_t* written, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_trace_geodesic<<<(n + 63) / 64, 64, 0, st>>>(reinterpret_cast<const TraceJob*>(jobs), n,
                                                   reinterpret_cast<magik_trace_geodesic_step_t*>(steps), written);
    return cudaGetLastError();
}

// ------------------------------------------------------ device scene table
size_t dev_scene_size(const mgk_scene& s) {
    return s.precision == MGK_PRECISION_F64 ? sizeof(DevScene<double>) : sizeof(DevScene<float>);
}

template <class T> static void fill_t(const mgk_scene& s, const float* xyz_w, DevScene<T>* P) {
    SceneConsts c = scene_consts(s);
    *P = DevScene<T>{};
    double spin = 0.0, h0 = 1.0;
    with_metric(s.metric, [&](auto mt) {
        using MT = decltype(mt);
        // the metric's parameters (params_t / make_params) in T and in double;
        // the FP64 attempts of the MIXED mode capture at the radius and with
        // the flag the FP32 state uses
        P->m = scene_params<MT, T>(s);
        P->md = scene_params<MT, double>(s);
        P->md.horizon = double(P->m.horizon);
        P->md.spin_abs_gt1 = double(P->m.spin_abs_gt1);
        spin = MT::spin(s);
        h0 = MT::initial_h_step();
    });
    const double a_t = P->md.spin;  // the spin as integrated (0 for spherical metrics)
    for (int i = 0; i < 4; ++i) {
        P->cam[i] = T(c.cam_pos[i]);
        P->u_obs[i] = T(c.u_obs[i]);
        for (int j = 0; j < 4; ++j) P->M[i][j] = T(c.M[i][j]);
    }
    P->pix_a = T(c.pix_a); P->pix_b = T(c.pix_b); P->pix_c = T(c.pix_c); P->pix_d = T(c.pix_d);
    P->h0 = T(h0);
    P->disk_on = s.disk_r_out > 0.0 ? 1u : 0u;
    P->disk_r_in = T(s.disk_r_in);
    P->disk_r_out = T(s.disk_r_out);
    P->disk_T_in = T(s.disk_T_in);
    P->disk_lo = T(0.98 * s.disk_r_in - 0.02);
    P->disk_hi = T(1.02 * s.disk_r_out + 0.02);
    T er = T(s.escape_radius);
    P->escape_r2 = er * er;
    P->spin_phys = T(spin);
    P->omega_sign = T(c.omega_sign);
    P->kerr_a = T(a_t);
    P->r_plus = c.r_plus;
    double pre = c.r_plus + MGK_WIDE_BAND + 0.01;
    P->band_pre2 = pre * pre;
    P->atol_d = s.abs_tol;
    P->rtol_d = s.rel_tol;
    P->hmax_d = s.h_max;
    P->spin_d = a_t;
    T rr = T(s.star_radius_rad);
    P->star_inv_r2 = T(1) / (rr * rr);
    double dl = (s.lambda_max_nm - s.lambda_min_nm) / s.n_bins;
    for (uint32_t k = 0; k < s.n_bins && k < MGK_MAX_BINS; ++k) {
        const double lam = s.lambda_min_nm + (k + 0.5) * dl;
        P->lambda[k] = T(lam);
        // boosted blackbody a_k / (exp(b_k / (z T)) - 1), internal_math.h:2511-2526 with the
        // wavelength in metres
        const double h = 6.62607015E-34, c = 299792458.0, kb = 1.380649E-23, wl = lam * 1e-9;
        P->planck_a[k] = T(2.0 * h * c * c / (wl * wl * wl * wl * wl));
        P->planck_b[k] = T(h * c / (wl * kb));
    }
    for (uint32_t k = 0; k < 3 * s.n_bins && k < 3 * MGK_MAX_BINS; ++k) P->xyz_w[k] = xyz_w[k];
    P->seed = s.seed;
    P->width = s.width; P->height = s.height; P->spp = s.spp; P->n_bins = s.n_bins;
    P->max_steps = s.max_steps;
    P->metric = s.metric;
    P->inv_spp = 1.0f / float(s.spp);
    P->sample_offset = s.sample_offset;
    P->spectral_mode = s.spectral_mode;
    if (s.spectral_mode == MGK_SPECTRAL_SAMPLED) {
        cmf_inverse_cdf_table(s.lambda_min_nm, s.lambda_max_nm, P->cmf_icdf);
        const double h = 6.62607015E-34, c = 299792458.0, kb = 1.380649E-23;
        P->planck_c1 = T(2.0 * h * c * c);
        P->planck_c2 = T(h * c / kb);
        // radiance_to_irradiance (device_color_utilities.cuh:22-29): the sensor of
        // sensor_diag_mm with the frame's aspect (compute_inv_b,
        // device_sensor_utilities.cuh:59-62), area per pixel times
        // iso 2 pi / ((360 fps) / shutter angle)
        const double W = s.width, H = s.height;
        const double inv_b = s.sensor_diag_mm / std::sqrt(W * W + H * H);
        const double area_m2 = (W * inv_b) * (H * inv_b) / 1e6;
        P->sensor_gain = T((area_m2 / (W * H)) * s.iso * 2.0 * M_PI / ((360.0 * s.fps) / s.shutter_angle_deg));
        P->lambda_lo = T(s.lambda_min_nm);
        P->dlambda = T(dl);
        P->inv_sigma_sqrt2 = T(1.0 / (s.redistribution_sigma_nm * std::sqrt(2.0)));
    }
    P->room_on = s.room_on ? 1u : 0u;
    P->room_limit = s.room_reflection_limit;
    for (int a = 0; a < 3; ++a) {
        P->room_lo[a] = T(s.room_min[a]);
        P->room_hi[a] = T(s.room_max[a]);
        P->light_lo[a] = T(s.light_min[a]);
        P->light_hi[a] = T(s.light_max[a]);
    }
    P->light_scale = T(s.light_scale);
    P->ray_base = 0;
}

void fill_dev_scene(const mgk_scene& s, const float* xyz_w, void* out) {
    if (s.precision == MGK_PRECISION_F64) fill_t<double>(s, xyz_w, reinterpret_cast<DevScene<double>*>(out));
    else fill_t<float>(s, xyz_w, reinterpret_cast<DevScene<float>*>(out));
}

}  // namespace mgk
