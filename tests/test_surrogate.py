"""The deflection surrogate: network kernels against the numpy oracle,
training, and the routed render (network in front of RKF45).

Tolerances.  The GPU accumulates in FP32 in a different order than the
oracle (float64 accumulation rounded to float32), so a value that lands next
to a BF16 rounding boundary can round the other way; everything else rounds
at the same points.  Outputs: max |gpu - oracle| <= 2e-2 + 2e-2 |oracle|,
median <= 1e-3.  Gradients: relative L2 error of every layer's weight and
bias gradient <= 2e-2 against the BF16-emulating oracle and <= 1e-1 against
the exact float64 gradient.
"""
import ctypes as C

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from oracle import mlp_oracle as O
from tests.conftest import small_scene


# ------------------------------------------------------------------ CPU
def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(0).normal(size=200_000).astype(np.float32) * 37.0
    x[:4] = [0.0, -0.0, 1e-40, 3.0e38]
    assert np.array_equal(O.bf16(x), torch.from_numpy(x).to(torch.bfloat16).float().numpy())


def test_oracle_backward_matches_finite_differences():
    p = O.init_params(3).astype(np.float64)
    f, lab = O.random_batch(48, 5)
    w = O.weights_of(M.train_defaults())
    _, g = O.loss_and_grad(p, f, lab, w, bf16_mode=False)
    L, _ = O.layout()
    rng = np.random.default_rng(1)
    checked = 0
    for li, (wo, bo, n_out, n_in) in enumerate(L):
        real_in = O.IN if li == 0 else O.HID
        real_out = O.OUT if li == O.LAYERS - 1 else O.HID
        for _ in range(4):
            o, i = rng.integers(real_out), rng.integers(real_in)
            for k in (wo + o * n_in + i, bo + o):
                eps = 1e-6
                pp, pm = p.copy(), p.copy()
                pp[k] += eps
                pm[k] -= eps
                fd = (O.loss(pp, f, lab, w) - O.loss(pm, f, lab, w)) / (2 * eps)
                assert abs(g[k] - fd) <= 1e-5 * max(1.0, abs(fd)), (li, k, g[k], fd)
                checked += 1
    assert checked == 40


@pytest.mark.parametrize("n", [1, 1000, 1 << 16, 3 * 100_003])
def test_epoch_order_is_a_permutation(n):
    """The restated epoch order is a permutation of [0, n) that changes with
    the epoch and the seed."""
    a = O.epoch_order(n, 7, 0)
    assert np.array_equal(np.sort(a), np.arange(n, dtype=np.uint32))
    if n > 1000:
        assert not np.array_equal(a, O.epoch_order(n, 7, 1))
        assert not np.array_equal(a, O.epoch_order(n, 8, 0))
        assert np.mean(a == np.arange(n)) < 1e-2


def test_param_layout_matches_library():
    _, total = O.layout()
    assert M.surrogate_param_count() == total == 205_840


def test_train_defaults():
    c = M.train_defaults()
    assert (c.batch, c.epochs) == (65536, 20)
    assert abs(c.lr - 1e-3) < 1e-9 and abs(c.beta1 - 0.9) < 1e-7 and abs(c.beta2 - 0.999) < 1e-7


# ------------------------------------------------------------------ GPU
def _dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.view(dtype)).cuda()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 4096])
@pytest.mark.parametrize("path", ["fused", "tiled"])
def test_forward_matches_oracle(ctx, n, path):
    """Both inference paths (the fused tcgen05 kernel and the tiled mma.sync
    GEMMs of the training path) against the BF16-emulating oracle."""
    net = M.Surrogate(ctx, seed=7)
    p = O.init_params(11)
    net.set_params(p)
    f, _ = O.random_batch(n, 12)
    fwd = net.forward if path == "fused" else net.forward_tiled
    got = fwd(_dev(f)).cpu().numpy()
    want, _ = O.forward(p, f, bf16_mode=True)
    err = np.abs(got - want)
    assert err.max() <= 2e-2 + 2e-2 * np.abs(want).max(), err.max()
    assert np.median(err) <= 1e-3
    assert np.all(got[:, O.OUT:] == 0.0)  # padding outputs
    assert net.status() == 0
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [("MGK_SURROGATE_PAIRS", "1"), ("MGK_SURROGATE_CHAIN", "tmem"),
                                     ("MGK_SURROGATE_FUSED", "0")])
def test_chain_variants_equal_default(ctx, variant):
    """The other chain kernels against the default (single CTAs, activations
    in shared memory, each tile's backward right after its forward in one
    kernel): CTA pairs (cta_group::2 MMAs of M = 256, each SM holding half of
    every weight chunk), the activations in tensor memory (tcgen05.mma with A
    from TMEM, N-halves of 128), and the forward and backward as two
    kernels.
    The same inference outputs and the same gradient, the loss to its
    summation order, on an odd tile count with a ragged last tile."""
    import os
    key, val = variant
    net = M.Surrogate(ctx, seed=7)
    net.set_params(O.init_params(41))
    f, lab = O.random_batch(70_001, 42)
    x = _dev(f)
    n = 65536
    cfg = M.train_defaults(batch=n)
    d_lab = _dev(lab[:n].view(np.int32).reshape(n, 8))
    res = {}
    try:
        for on in (False, True):
            if on:
                os.environ[key] = val
            out = net.forward(x).cpu().numpy()
            loss, g = net.gradient(cfg, x[:n].contiguous(), d_lab)
            res[on] = (out, loss, g)
    finally:
        os.environ.pop(key, None)
    (o0, l0, g0), (o1, l1, g1) = res[False], res[True]
    assert np.array_equal(o0, o1), np.abs(o0 - o1).max()
    assert np.array_equal(g0, g1), np.abs(g0 - g1).max()
    assert abs(l0 - l1) <= 1e-6 * abs(l0)
    assert net.status() == 0
    net.close()


@pytest.mark.gpu
def test_fused_forward_many_tiles_per_block(ctx):
    """300,000 rows: every block of the persistent fused kernel runs many
    tiles, so the weight ring and all barrier phases wrap around; the result
    must agree with the tiled path row for row, and follow a weight update."""
    net = M.Surrogate(ctx, seed=7)
    f, _ = O.random_batch(300_000, 13)
    x = _dev(f)
    for seed in (31, 32):
        net.set_params(O.init_params(seed))
        a = net.forward(x).cpu().numpy()
        b = net.forward_tiled(x).cpu().numpy()
        err = np.abs(a - b)
        assert err.max() <= 2e-2 + 2e-2 * np.abs(b).max() and np.median(err) <= 1e-3
    assert net.status() == 0
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1024, 8192])
def test_gradient_matches_oracle(ctx, n):
    import torch
    net = M.Surrogate(ctx, seed=7)
    p = O.init_params(21)
    net.set_params(p)
    f, lab = O.random_batch(n, 22)
    cfg = M.train_defaults(batch=n)
    loss, g = net.gradient(cfg, _dev(f), _dev(lab.view(np.int32).reshape(n, 8)))
    w = O.weights_of(cfg)
    l_b, g_b = O.loss_and_grad(p, f, lab, w, bf16_mode=True)
    l_x, g_x = O.loss_and_grad(p.astype(np.float64), f, lab, w, bf16_mode=False)
    assert abs(loss - l_b) <= 1e-3 * abs(l_b)
    L, _ = O.layout()
    for li, (wo, bo, n_out, n_in) in enumerate(L):
        for lo, hi in ((wo, wo + n_out * n_in), (bo, bo + n_out)):
            assert _rel(g[lo:hi], g_b[lo:hi]) <= 2e-2, (li, _rel(g[lo:hi], g_b[lo:hi]))
            assert _rel(g[lo:hi], g_x[lo:hi]) <= 1e-1, (li, _rel(g[lo:hi], g_x[lo:hi]))
    # the padding of the first and last layer gets no gradient
    w1 = g[: 256 * 16].reshape(256, 16)
    assert np.all(w1[:, O.IN:] == 0.0)
    w5 = g[L[4][0]: L[4][0] + 16 * 256].reshape(16, 256)
    assert np.all(w5[O.OUT:] == 0.0) and np.all(g[L[4][1] + O.OUT: L[4][1] + 16] == 0.0)
    net.close()
    del torch


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1024, 65536])
def test_tensor_core_gradient_equals_mma_path(ctx, n):
    """The tcgen05 training kernels (mlp_train_tc.cu: forward with stash,
    input gradients, split-K weight gradients) against the mma.sync GEMMs of
    mlp.cu on the same batch: both round at the same points (BF16 Z, H and
    dZ, FP32 accumulation); they differ by the SiLU evaluation (tanh.approx
    against expf) and the summation order."""
    import os
    p = O.init_params(23)
    f, lab = O.random_batch(n, 24)
    cfg = M.train_defaults(batch=n)
    grads = {}
    for path in ("mma", "tc"):
        os.environ["MGK_SURROGATE_TRAIN"] = path
        try:
            net = M.Surrogate(ctx, seed=7)
        finally:
            del os.environ["MGK_SURROGATE_TRAIN"]
        net.set_params(p)
        grads[path] = net.gradient(cfg, _dev(f), _dev(lab.view(np.int32).reshape(n, 8)))
        assert net.status() == 0
        net.close()
    (l_m, g_m), (l_t, g_t) = grads["mma"], grads["tc"]
    assert abs(l_t - l_m) <= 1e-3 * abs(l_m)
    L, _ = O.layout()
    for li, (wo, bo, n_out, n_in) in enumerate(L):
        for lo, hi in ((wo, wo + n_out * n_in), (bo, bo + n_out)):
            assert _rel(g_t[lo:hi], g_m[lo:hi]) <= 2e-2, (li, _rel(g_t[lo:hi], g_m[lo:hi]))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 1 << 24, 5 * 1_000_003])
def test_device_epoch_order_equals_restatement(ctx, n):
    """mgk_surrogate_shuffle's order on the device against the numpy
    restatement of the keyed Feistel permutation."""
    net = M.Surrogate(ctx, seed=7)
    net.shuffle(0xABCD, 3, n)
    got = net.order(n)
    assert np.array_equal(got, O.epoch_order(n, 0xABCD, 3))
    net.close()


def _samples(ctx, scene, n, seed):
    feat, lab = M.make_samples(ctx, scene, seed, n)
    return feat, lab


@pytest.mark.gpu
def test_samples_are_f64_traces_of_camera_rays(ctx):
    """Fixed-observer samples of frame `seed` equal the F64 integrator's
    classes and disk radii for the same camera rays."""
    s = small_scene(width=64, height=32, spp=1, precision=abi.PRECISION_F64)
    n = s.width * s.height
    s.seed = 99
    feat, lab = M.make_samples(ctx, s, 99, n)
    lab = lab.cpu().numpy().view(O.LABEL_DTYPE).ravel()
    rec = ctx.trace_rays(s, 0, n)
    cls = np.where(rec["cls"] == abi.RAY_DISK, 0, np.where(rec["cls"] == abi.RAY_ESCAPED, 1, 2))
    assert np.array_equal(lab["cls"], cls)
    disk = cls == 0
    assert np.allclose(lab["r"][disk], ((rec["r_hit"][disk] - 10.0) / 10.0).astype(np.float32))
    f = feat.cpu().numpy()
    n = np.stack([f[:, 4] / 2, f[:, 5] / 2, (f[:, 6] - 3) / 4], 1)  # feature scaling of the direction
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6)
    assert np.all(n[:, 2] < 0)


@pytest.mark.gpu
def test_training_reduces_loss_and_keeps_padding_zero(ctx):
    s = small_scene(width=128, height=64, spp=1, precision=abi.PRECISION_F64)
    feat, lab = _samples(ctx, s, s.width * s.height * 4, 5)
    net = M.Surrogate(ctx, seed=3)
    cfg = M.train_defaults(batch=4096, epochs=8)
    losses = net.train(cfg, feat, lab)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses
    p = net.get_params()
    L, _ = O.layout()
    assert np.all(p[: 256 * 16].reshape(256, 16)[:, O.IN:] == 0.0)
    assert np.all(p[L[4][0]: L[4][0] + 16 * 256].reshape(16, 256)[O.OUT:] == 0.0)
    net.close()


@pytest.mark.gpu
def test_data_parallel_loop_on_one_rank_is_train(ctx):
    """magik_b200.dist.train_data_parallel on one rank (shuffle, gradient step
    and Adam step through the C-ABI, the gradient in a torch buffer between
    them) takes the steps of mgk_surrogate_train from the same initial
    weights.  The backward adds its split-K partial products with atomics in
    either order, so the runs agree to FP32 summation order: epoch losses
    within 1e-3 relative, and the parameter difference within 1e-2 of the
    distance the parameters moved (L2)."""
    import torch
    from magik_b200 import dist as D
    s = small_scene(width=128, height=64, spp=1, precision=abi.PRECISION_F64)
    feat, lab = _samples(ctx, s, s.width * s.height * 2, 5)
    cfg = M.train_defaults(batch=4096, epochs=2, lr_final=1e-4)
    a, b = M.Surrogate(ctx, seed=3), M.Surrogate(ctx, seed=3)
    p0 = a.get_params()
    with pytest.raises(M.MgkError):  # no order yet
        g = torch.empty(b.param_count, dtype=torch.float32, device="cuda")
        b.gradient_step(cfg, feat, lab, 0, 4096, g, torch.zeros(1, device="cuda"))
    la = a.train(cfg, feat, lab)
    lb = D.train_data_parallel(b, cfg, feat, lab)
    torch.cuda.synchronize()
    pa, pb = a.get_params(), b.get_params()
    assert np.all(np.isfinite(lb))
    np.testing.assert_allclose(lb, la, rtol=1e-3)
    assert np.linalg.norm(pa - pb) <= 1e-2 * np.linalg.norm(pa - p0)
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("switch", ["MGK_SURROGATE_GRAPH", "MGK_SURROGATE_PDL"])
def test_counted_training_replay_equals_launches(ctx, switch):
    """mgk_surrogate_train replays epochs after the first from a CUDA graph
    and launches its kernels as programmatic dependents; with either turned
    off (the same kernels as ordinary launches) it takes the same steps: the
    same parameters bit for bit, the epoch losses to their summation order."""
    import os
    s = small_scene(width=128, height=64, spp=1, precision=abi.PRECISION_F64)
    feat, lab = _samples(ctx, s, s.width * s.height * 2, 5)
    cfg = M.train_defaults(batch=4096, epochs=3)
    runs = []
    for off in (False, True):
        net = M.Surrogate(ctx, seed=3)
        if off:
            os.environ[switch] = "0"
        try:
            losses = net.train(cfg, feat, lab)
        finally:
            os.environ.pop(switch, None)
        runs.append((net.get_params(), losses))
        assert net.status() == 0
        net.close()
    (pa, la), (pb, lb) = runs
    assert np.array_equal(pa, pb)
    np.testing.assert_allclose(la, lb, rtol=1e-5)


@pytest.mark.gpu
def test_routed_render_all_fallback_equals_integrator(ctx):
    """conf_min above 1 sends every ray to RKF45: the film must equal mgk_render's."""
    import torch
    s = small_scene(width=96, height=48, spp=2)
    stars = M.star_catalog(0x57A25, 20000)
    d_stars = torch.from_numpy(stars.view(np.uint8)).cuda()
    n_pix = s.width * s.height
    ref = torch.zeros(n_pix * 3, dtype=torch.float32, device="cuda")
    ctx.render(s, d_stars, ref)
    net = M.Surrogate(ctx, seed=3)
    film = torch.zeros_like(ref)
    st = M.render_surrogate(ctx, net, s, d_stars, film, conf_min=2.0, crit_frac=0.0)
    assert st.fallback_rays == n_pix * s.spp
    assert torch.equal(film, ref)
    # and nothing falls back with the gates open
    st = M.render_surrogate(ctx, net, s, d_stars, film, conf_min=-1.0, crit_frac=0.0)
    assert st.fallback_rays == 0 and st.attempts == 0
    net.close()


@pytest.mark.gpu
def test_trained_surrogate_render_error_and_fallback(ctx):
    """A network trained on F64 traces of the view renders the frame with part
    of the rays on RKF45; the film error against the F64 render shrinks as
    the routing gets stricter, and the strictest routing reaches the
    integrator's own film."""
    import torch
    s = small_scene(width=128, height=64, spp=2)
    base = small_scene(width=128, height=64, spp=2, precision=abi.PRECISION_F64)
    feat, lab = _samples(ctx, base, base.width * base.height * base.spp * 8, 1000)
    net = M.Surrogate(ctx, seed=3)
    net.train(M.train_defaults(batch=8192, epochs=20), feat, lab)
    stars = M.star_catalog(0x57A25, 20000)
    d_stars = torch.from_numpy(stars.view(np.uint8)).cuda()
    n_pix = s.width * s.height
    ref = torch.zeros(n_pix * 3, dtype=torch.float32, device="cuda")
    ctx.render(base, d_stars, ref)
    plain = torch.zeros_like(ref)
    plain_attempts = ctx.render(s, d_stars, plain).attempts
    errs, fb, att = [], [], []
    for conf_min in (-1.0, 0.0, 0.9, 0.99, 2.0):
        film = torch.zeros_like(ref)
        st = M.render_surrogate(ctx, net, s, d_stars, film, conf_min=conf_min, crit_frac=0.02 if conf_min >= 0 else 0.0)
        errs.append(float((film - ref).abs().view(-1, 3).mean().item()))
        fb.append(st.fallback_rays / (n_pix * s.spp))
        att.append(st.attempts)
    # what the network gains: the integrator work it takes away ...
    assert att[0] == 0 and fb[0] == 0.0
    assert fb[1] <= fb[2] <= fb[3] <= fb[4] == 1.0
    assert att[1] <= att[2] <= att[3] <= att[4] == plain_attempts
    # ... and what that costs in accuracy: the stricter the routing the closer to RKF45
    assert errs[4] <= errs[3] + 1e-6 <= errs[0] + 2e-6
