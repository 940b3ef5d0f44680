// Host-side checks of the metric plugins (compiled by tests/test_plugin.py
// with nvcc, built into a variant with the test plugin of
// metric_schwarzschild_user.cuh, run on the CPU):
//  * g * g^-1 = 1 for every supported metric at seeded points (double);
//  * the reference observer is a unit timelike vector, g(u, u) = -1;
//  * the plugin's host-callable members equal the built-in Schwarzschild's
//    bit for bit, in float and in double.
// Prints "ok" and exits 0, or names the first failure and exits 1.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../magik_b200/csrc/dev_scene.cuh"

using namespace mgk;

namespace {

int fails = 0;
void check(bool ok, const char* what, int tag) {
    if (!ok && fails++ < 8) std::printf("FAIL metric %d: %s\n", tag, what);
}

template <class T> T g_uv(const Sym4<T>& g, const V4<T>& u, const V4<T>& v) { return inner_product(g, u, v); }

template <class T> bool same_bits(const T* a, const T* b, size_t n) { return std::memcmp(a, b, n * sizeof(T)) == 0; }

template <class MT> void check_metric(const mgk_scene& s0) {
    mgk_scene s = s0;
    s.metric = MT::tag;
    MP<double> m = scene_params<MT, double>(s);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < 2000; ++i) {
        double q[3];
        for (int c = 0; c < 3; ++c) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            q[c] = (double(x >> 11) / 9007199254740992.0 - 0.5) * 60.0;
        }
        const double r = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        if (r < 3.0) continue;
        const Sym4<double> g = MT::template compute_g<double>(q[0], q[1], q[2], m);
        const Sym4<double> h = MT::template compute_inv_g<double>(q[0], q[1], q[2], m);
        // rows of g and h as full 4x4 matrices in (x, y, z, t) order
        const double G[4][4] = {{g.xx, g.xy, g.xz, g.tx}, {g.xy, g.yy, g.yz, g.ty}, {g.xz, g.yz, g.zz, g.tz},
                                {g.tx, g.ty, g.tz, g.tt}};
        const double H[4][4] = {{h.xx, h.xy, h.xz, h.tx}, {h.xy, h.yy, h.yz, h.ty}, {h.xz, h.yz, h.zz, h.tz},
                                {h.tx, h.ty, h.tz, h.tt}};
        double worst = 0.0;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                double acc = 0.0;
                for (int k = 0; k < 4; ++k) acc += G[a][k] * H[k][b];
                worst = std::fmax(worst, std::fabs(acc - (a == b ? 1.0 : 0.0)));
            }
        check(worst < 1e-12, "g * g^-1 != 1", MT::tag);
        const V4<double> u = MT::template reference_observer<double>(q[0], q[1], q[2], m);
        check(std::fabs(g_uv(g, u, u) + 1.0) < 1e-12, "g(u, u) != -1", MT::tag);
    }
}

template <class T> void check_plugin_equals_schwarzschild(const mgk_scene& s0) {
    using A = metric<MGK_METRIC_SCHWARZSCHILD>;
    using B = metric<16>;
    for (int ms = 0; ms < 2; ++ms) {
        mgk_scene s = s0;
        s.mass_sign = ms ? -1.0 : 1.0;
        s.horizon_scalar = 1.01;
        const MP<T> ma = scene_params<A, T>(s), mb = scene_params<B, T>(s);
        check(same_bits(reinterpret_cast<const char*>(&ma), reinterpret_cast<const char*>(&mb), sizeof(ma)),
              "make_params differs", 16);
        check(A::initial_h_step() == B::initial_h_step() && A::outer_horizon(s) == B::outer_horizon(s) &&
                  A::spin(s) == B::spin(s) && A::length_scale(2e30) == B::length_scale(2e30),
              "scalar members differ", 16);
        uint64_t x = 0x0123456789ABCDEFull;
        for (int i = 0; i < 2000; ++i) {
            T q[3];
            for (int c = 0; c < 3; ++c) {
                x ^= x << 13; x ^= x >> 7; x ^= x << 17;
                q[c] = T((double(x >> 11) / 9007199254740992.0 - 0.5) * 80.0);
            }
            const Sym4<T> ga = A::template compute_g<T>(q[0], q[1], q[2], ma);
            const Sym4<T> gb = B::template compute_g<T>(q[0], q[1], q[2], mb);
            const Sym4<T> ha = A::template compute_inv_g<T>(q[0], q[1], q[2], ma);
            const Sym4<T> hb = B::template compute_inv_g<T>(q[0], q[1], q[2], mb);
            const V4<T> ua = A::template reference_observer<T>(q[0], q[1], q[2], ma);
            const V4<T> ub = B::template reference_observer<T>(q[0], q[1], q[2], mb);
            check(same_bits(&ga.tt, &gb.tt, 10) && same_bits(&ha.tt, &hb.tt, 10) && same_bits(&ua.x, &ub.x, 4),
                  "compute_g / compute_inv_g / reference_observer differ", 16);
        }
    }
}

}  // namespace

int main() {
    mgk_scene s{};
    s.spin = 0.9;
    s.time_reversed = 1;
    s.mass_sign = 1.0;
    s.horizon_scalar = 1.01;
    s.h_max = 1000.0;
    s.abs_tol = 1e-7;
    s.rel_tol = 1e-7;
    s.n_max_substep = 56;
    check_metric<metric<MGK_METRIC_MINKOWSKI>>(s);
    check_metric<metric<MGK_METRIC_SCHWARZSCHILD>>(s);
    check_metric<metric<MGK_METRIC_KERR>>(s);
    check_metric<metric<16>>(s);
    check_plugin_equals_schwarzschild<float>(s);
    check_plugin_equals_schwarzschild<double>(s);
    check(metric_supported(16) && metric_supported(MGK_METRIC_KERR) && !metric_supported(3) &&
              !metric_supported(17),
          "supported_metrics", 16);
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
