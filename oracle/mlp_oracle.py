"""CPU oracle of the deflection surrogate network (test infrastructure only).

Only the tests, the smoke check and the CPU leg of the benchmark may import
this module; the library never does.

The network is not part of the reference renderer, so there is no reference
file to follow.  This module restates, in numpy, what the library's kernels
compute:

* ``forward``/``loss_and_grad`` with ``bf16=True`` round exactly where the
  kernels round (inputs, weights, pre-activations, activations and the
  back-propagated gradients to BF16; FP32 accumulation, here done in float64
  and rounded to float32), so the GPU gradient can be compared with a tight
  tolerance;
* with ``bf16=False`` everything is float64: the mathematical gradient, used
  to pin the backward formulas by central finite differences.

Parity is pinned by those finite differences, not by a reference run.

Parameter layout (floats, weights stored [out][in], inputs padded to 16 and
outputs to 16):  W1 256x16, b1 256, W2..W4 256x256 + 256, W5 16x256, b5 16.
"""
import numpy as np

IN, IN_PAD, HID, OUT, OUT_PAD, LAYERS = 7, 16, 256, 8, 16, 5
SHAPES = [(HID, IN_PAD), (HID, HID), (HID, HID), (HID, HID), (OUT_PAD, HID)]


def layout():
    """[(w_offset, b_offset, out, in)] per layer and the total count."""
    o, res = 0, []
    for (n_out, n_in) in SHAPES:
        w = o
        o += n_out * n_in
        b = o
        o += n_out
        res.append((w, b, n_out, n_in))
    return res, o


def unpack(params):
    L, total = layout()
    p = np.asarray(params)
    assert p.size == total
    return [(p[w:w + no * ni].reshape(no, ni), p[b:b + no]) for (w, b, no, ni) in L]


def pack(grads):
    return np.concatenate([np.concatenate([g_w.ravel(), g_b.ravel()]) for (g_w, g_b) in grads])


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    out = ((u + r) & 0xFFFF0000).astype(np.uint32)
    return out.view(np.float32).reshape(a.shape)


def _f32(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, feat, bf16_mode=True):
    """Returns (out [B,16], cache).  feat: [B, 7]."""
    layers = unpack(params)
    B = feat.shape[0]
    x = np.zeros((B, IN_PAD), np.float64)
    x[:, :IN] = feat
    rnd = (lambda a: bf16(_f32(a)).astype(np.float64)) if bf16_mode else (lambda a: np.asarray(a, np.float64))
    x0 = rnd(x)
    H, Z = [x0], []
    h = x0
    for li, (W, b) in enumerate(layers):
        Wr = rnd(W)
        acc = h @ Wr.T
        if li < LAYERS - 1:
            z = (_f32(acc + b.astype(np.float64)) if bf16_mode else acc + b).astype(np.float64)
            Z.append(rnd(z))
            h = rnd(_f32(_silu(z)) if bf16_mode else _silu(z))
            H.append(h)
        else:
            out = _f32(acc + b) if bf16_mode else acc + b
    return np.asarray(out, np.float64), dict(H=H, Z=Z, layers=layers, rnd=rnd)


def loss_terms(out, lab, w):
    """Per-sample loss and d loss / d out (unscaled), restating the loss kernel:
    softmax cross-entropy over (disk, escape, horizon = logit 0), squared
    errors of radius and redshift (disk) or direction (escape), and a binary
    cross-entropy confidence head whose target is "class right and errors
    within tolerance".  lab: structured array (cls, r, g, dir)."""
    B = out.shape[0]
    d = np.zeros((B, OUT_PAD))
    z0, z1 = out[:, 0], out[:, 1]
    mx = np.maximum(np.maximum(z0, z1), 0.0)
    e0, e1, e2 = np.exp(z0 - mx), np.exp(z1 - mx), np.exp(-mx)
    se = e0 + e1 + e2
    p = np.stack([e0 / se, e1 / se, e2 / se], 1)
    c = lab["cls"].astype(np.int64)
    l = w["cls"] * -np.log(np.maximum(p[np.arange(B), c], 1e-30))
    d[:, 0] = w["cls"] * (p[:, 0] - (c == 0))
    d[:, 1] = w["cls"] * (p[:, 1] - (c == 1))
    pred = np.where((p[:, 0] >= p[:, 1]) & (p[:, 0] >= p[:, 2]), 0, np.where(p[:, 1] >= p[:, 2], 1, 2))
    good = pred == c
    disk, esc = c == 0, c == 1
    er, eg = out[:, 2] - lab["r"], out[:, 3] - lab["g"]
    l += np.where(disk, w["r"] * er * er + w["g"] * eg * eg, 0.0)
    d[:, 2] = np.where(disk, 2 * w["r"] * er, 0.0)
    d[:, 3] = np.where(disk, 2 * w["g"] * eg, 0.0)
    good &= ~disk | ((np.abs(er) < w["tol_r"]) & (np.abs(eg) < w["tol_g"]))
    ed = out[:, 4:7] - lab["dir"]
    l += np.where(esc, w["dir"] * (ed * ed).sum(1), 0.0)
    d[:, 4:7] = np.where(esc[:, None], 2 * w["dir"] * ed, 0.0)
    good &= ~esc | ((ed * ed).sum(1) < w["tol_dir"] ** 2)
    q = 1.0 / (1.0 + np.exp(-out[:, 7]))
    t = good.astype(np.float64)
    l += w["conf"] * -(t * np.log(np.maximum(q, 1e-30)) + (1 - t) * np.log(np.maximum(1 - q, 1e-30)))
    d[:, 7] = w["conf"] * (q - t)
    return l, d


def loss(params, feat, lab, w, bf16_mode=False):
    out, _ = forward(params, feat, bf16_mode)
    l, _ = loss_terms(out, lab, w)
    return l.mean()


def loss_and_grad(params, feat, lab, w, bf16_mode=True):
    """Mean batch loss and the gradient w.r.t. the flat parameter vector."""
    out, cache = forward(params, feat, bf16_mode)
    l, d = loss_terms(out, lab, w)
    B = out.shape[0]
    rnd = cache["rnd"]
    d = d / B
    d32 = _f32(d).astype(np.float64) if bf16_mode else d
    dz = rnd(d32)
    layers, H, Z = cache["layers"], cache["H"], cache["Z"]
    grads = [None] * LAYERS
    grads[LAYERS - 1] = (dz.T @ H[LAYERS - 1], d32.sum(0))
    g = dz
    for li in range(LAYERS - 1, 0, -1):
        W = rnd(layers[li][0])
        g = rnd((g @ W) * _silu_grad(Z[li - 1]))
        grads[li - 1] = (g.T @ H[li - 1], g.sum(0))
    return l.mean(), pack(grads)


def init_params(seed=1):
    """Uniform(+-1/sqrt(fan_in)) on the real inputs and outputs, zero padding
    (any seeded init serves the tests; the library's own differs)."""
    rng = np.random.default_rng(seed)
    L, total = layout()
    p = np.zeros(total, np.float32)
    for li, (w, b, no, ni) in enumerate(L):
        real_in = IN if li == 0 else HID
        real_out = OUT if li == LAYERS - 1 else HID
        W = np.zeros((no, ni), np.float32)
        k = 1.0 / np.sqrt(real_in)
        W[:real_out, :real_in] = rng.uniform(-k, k, (real_out, real_in))
        p[w:w + no * ni] = W.ravel()
        p[b:b + real_out] = rng.uniform(-k, k, real_out)
    return p


LABEL_DTYPE = np.dtype([("cls", "<i4"), ("r", "<f4"), ("g", "<f4"), ("dir", "<f4", (3,)),
                        ("reserved", "<f4", (2,))])


def random_batch(n, seed=2):
    """Features in the network's input ranges and labels of all three classes."""
    rng = np.random.default_rng(seed)
    f = np.zeros((n, IN), np.float32)
    f[:, 0] = rng.uniform(-1, 1, n)
    inc = rng.uniform(0, np.pi / 2, n)
    f[:, 1], f[:, 2] = np.cos(inc), np.sin(inc)
    f[:, 3] = rng.uniform(-1, 1, n)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[:, 2] = -np.abs(v[:, 2])
    f[:, 4:7] = v
    lab = np.zeros(n, LABEL_DTYPE)
    lab["cls"] = rng.integers(0, 3, n)
    lab["r"] = np.where(lab["cls"] == 0, rng.uniform(-0.8, 1.0, n), 0)
    lab["g"] = np.where(lab["cls"] == 0, rng.uniform(0.5, 1.5, n), 0)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    lab["dir"] = np.where((lab["cls"] == 1)[:, None], d, 0)
    return f, lab


def weights_of(cfg):
    """Loss weights of an mgk_train_config (ctypes struct or dict)."""
    get = (lambda k: cfg[k]) if isinstance(cfg, dict) else (lambda k: getattr(cfg, k))
    return dict(cls=get("w_cls"), r=get("w_r"), g=get("w_g"), dir=get("w_dir"), conf=get("w_conf"),
                tol_r=get("tol_r"), tol_g=get("tol_g"), tol_dir=get("tol_dir"))


# ----------------------------------------------------------- epoch order
def _triplet_hash(x):
    """triplet_hash (internal_math.h:2027-2037) on Python ints, 32 bits."""
    m = 0xFFFFFFFF
    x ^= x >> 17; x = (x * 0xED5AD4BB) & m; x ^= x >> 11; x = (x * 0xAC4C1B51) & m
    x ^= x >> 15; x = (x * 0x31848BAB) & m; x ^= x >> 14
    return x


def rng_u32(seed, stream, index, dim):
    """The counter-based hash chain of the library (dev_scene.cuh rng_u32)."""
    m = 0xFFFFFFFF
    h = _triplet_hash((seed & m) ^ 0x9E3779B9)
    h = _triplet_hash(h ^ ((seed >> 32) & m))
    h = _triplet_hash(h ^ stream)
    h = _triplet_hash(h ^ index)
    return _triplet_hash(h ^ ((dim * 0x85EBCA6B + 1) & m))


def epoch_order(n, seed, epoch):
    """The sample order of one epoch (a restatement of mlp.cu k_epoch_perm):
    a 4-round balanced Feistel network on the smallest even number of bits
    covering n, round function the MurmurHash3 finalizer of the right half
    xor the round key rng_u32(seed, 0x7E11, epoch, r), cycle-walked into
    [0, n).  Vectorised over the n indices."""
    bits = 2
    while bits < 32 and (1 << bits) < n:
        bits += 1
    bits += bits & 1
    hb = bits // 2
    mask = np.uint64((1 << hb) - 1)
    keys = [np.uint64(rng_u32(seed, 0x7E11, epoch, r)) for r in range(4)]

    def fmix(h):
        h = h & np.uint64(0xFFFFFFFF)
        h ^= h >> np.uint64(16); h = (h * np.uint64(0x85EBCA6B)) & np.uint64(0xFFFFFFFF)
        h ^= h >> np.uint64(13); h = (h * np.uint64(0xC2B2AE35)) & np.uint64(0xFFFFFFFF)
        h ^= h >> np.uint64(16)
        return h

    def P(x):
        L, R = x >> np.uint64(hb), x & mask
        for k in keys:
            L, R = R, L ^ (fmix(R ^ k) & mask)
        return (L << np.uint64(hb)) | R

    x = P(np.arange(n, dtype=np.uint64))
    out = x.copy()
    todo = out >= n
    while todo.any():
        out[todo] = P(out[todo])
        todo = out >= n
    return out.astype(np.uint32)
