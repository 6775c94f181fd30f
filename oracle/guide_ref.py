"""NumPy restatement of the learned path-guiding network (test infrastructure only).

The reference renderer has no guiding, so there is no reference code to follow: this module is the
FP32 CPU oracle the tests check the GPU guiding kernels against. It restates, in plain NumPy:

* the one-blob input encoding and the 224 -> 4 x 64 (ReLU) -> 40 MLP, with the GPU's BF16
  rounding points mirrored (inputs, weights and hidden activations rounded to BF16, FP32
  accumulation), see photon-v2_b200/csrc/guide.cuh and guide_mlp.cu;
* the decoding of the 40 outputs into 8 von Mises-Fisher lobes;
* the training loss -sum_i w_i log q(w_i | x_i) / sum_i w_i and its gradient with respect to every
  parameter, by reverse-mode differentiation written out by hand.
"""

from __future__ import annotations

import numpy as np

IN, HID, LOBES, OUT, BINS = 224, 64, 8, 40, 32
SHAPES = [("W0", (IN, HID)), ("b0", (HID,)), ("W1", (HID, HID)), ("b1", (HID,)), ("W2", (HID, HID)),
          ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)), ("W4", (HID, OUT)), ("b4", (OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
MIN_KAPPA, MAX_KAPPA = 1e-2, 5e3


def unpack(params):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n]).reshape(shape)
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], np.float32).reshape(-1) for name, _ in SHAPES])


def init_params(seed=0, out_scale=0.1):
    """He-initialised weights, zero biases; small output layer."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            parts[name] = rng.normal(0.0, np.sqrt(2.0 / shape[0]), shape).astype(np.float32)
        else:
            parts[name] = np.zeros(shape, np.float32)
    parts["W4"] *= out_scale
    return pack(parts)


def bf16(x):
    """Round FP32 to the nearest BF16 (ties to even), returned as FP32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def one_blob(features):
    """features [n, 7] in [0, 1] -> [n, 224]."""
    f = np.asarray(features, np.float32)
    c = (np.arange(BINS, dtype=np.float32) + 0.5) / BINS
    z = (f[:, :, None] - c[None, None, :]) * BINS
    return np.exp(-0.5 * z * z).reshape(f.shape[0], IN).astype(np.float32)


def forward(params, features, keep=False, exact=False):
    """Raw outputs [n, 40]; with keep=True also the layer inputs (for backward). exact=True drops
    the BF16 rounding and computes in FP64 (for finite-difference checks)."""
    dt = np.float64 if exact else np.float32
    rnd = (lambda a: np.asarray(a, dt)) if exact else bf16
    p = {k: np.asarray(v, dt) for k, v in unpack(params).items()}
    x = rnd(one_blob(features))
    acts = [x]
    for l in range(4):
        h = np.maximum(x @ rnd(p[f"W{l}"]) + p[f"b{l}"], 0.0).astype(dt)
        x = rnd(h)
        acts.append(x)
    out = (x @ rnd(p["W4"]) + p["b4"]).astype(dt)
    return (out, acts) if keep else out


def decode(raw):
    """raw [n, 40] -> (weights [n, 8], means [n, 8, 3], kappa [n, 8])."""
    r = np.asarray(raw, np.float64).reshape(-1, LOBES, 5)
    logits = r[:, :, 0] - r[:, :, 0].max(axis=1, keepdims=True)
    w = np.exp(logits)
    w /= w.sum(axis=1, keepdims=True)
    m = r[:, :, 1:4]
    norm = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(norm > 1e-10, m / np.maximum(norm, 1e-30), np.array([0.0, 0.0, 1.0]))
    kappa = np.clip(np.exp(r[:, :, 4]), MIN_KAPPA, MAX_KAPPA)
    return w, mu, kappa


def vmf_pdf(mu, kappa, d):
    return kappa / (2 * np.pi * (1 - np.exp(-2 * kappa))) * np.exp(kappa * (np.einsum("nlk,nk->nl", mu, d) - 1))


def mixture_pdf(raw, d):
    w, mu, kappa = decode(raw)
    return (w * vmf_pdf(mu, kappa, np.asarray(d, np.float64))).sum(axis=1)


def loss_and_output_grad(raw, dirs, weights):
    """Loss -sum w_i log q_i / sum w_i and d loss / d raw [n, 40] (FP64)."""
    raw = np.asarray(raw, np.float64).reshape(-1, LOBES, 5)
    d = np.asarray(dirs, np.float64)
    wt = np.asarray(weights, np.float64)
    total = wt.sum()
    pi, mu, kappa = decode(raw.reshape(-1, OUT))
    v = vmf_pdf(mu, kappa, d)                      # [n, 8]
    q = (pi * v).sum(axis=1)
    loss = -(wt * np.log(np.maximum(q, 1e-30))).sum() / total
    r = pi * v / np.maximum(q, 1e-30)[:, None]      # responsibilities
    g = np.zeros_like(raw)
    scale = -(wt / total)[:, None]                  # d loss / d log q
    g[:, :, 0] = scale * (r - pi)
    cos = np.einsum("nlk,nk->nl", mu, d)
    e = np.exp(-2 * kappa)
    dlogv_dkappa = 1 / kappa - 2 * e / (1 - e) + (cos - 1)
    k_raw = np.exp(raw[:, :, 4])
    inside = (k_raw > MIN_KAPPA) & (k_raw < MAX_KAPPA)
    g[:, :, 4] = scale * r * dlogv_dkappa * kappa * inside
    m = raw[:, :, 1:4]
    norm = np.maximum(np.linalg.norm(m, axis=2, keepdims=True), 1e-30)
    dmu = kappa[:, :, None] * (d[:, None, :] - cos[:, :, None] * mu) / norm
    g[:, :, 1:4] = (scale * r)[:, :, None] * dmu
    return loss, g.reshape(-1, OUT)


def gradients(params, features, dirs, weights, exact=False):
    """(loss, d loss / d params): FP32 backward through the BF16-rounded forward pass, the GPU's
    arithmetic (exact=True: FP64 throughout, no rounding)."""
    dt = np.float64 if exact else np.float32
    rnd = (lambda a: np.asarray(a, dt)) if exact else bf16
    p = {k: np.asarray(v, dt) for k, v in unpack(params).items()}
    out, acts = forward(params, features, keep=True, exact=exact)
    loss, g_out = loss_and_output_grad(out, dirs, weights)
    g = g_out.astype(dt)
    grads = {"W4": acts[4].T @ g, "b4": g.sum(axis=0)}
    dx = g @ rnd(p["W4"]).T
    for l in (3, 2, 1, 0):
        dz = dx * (acts[l + 1] > 0)
        grads[f"W{l}"] = acts[l].T @ dz
        grads[f"b{l}"] = dz.sum(axis=0)
        if l > 0:
            dx = dz @ rnd(p[f"W{l}"]).T
    return loss, np.concatenate([np.asarray(grads[name], np.float64).reshape(-1) for name, _ in SHAPES])
