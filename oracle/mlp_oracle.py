"""FP64 restatement of the learned-correction MLP (TEST INFRASTRUCTURE ONLY).

Same network as the CUDA library: 35 -> 128 -> 128 -> 128 -> 3, GELU
(0.5 x (1 + erf(x / sqrt 2))), weights rounded to BF16 before use, biases in
full precision, loss = mean over samples and outputs of (y - t)^2. Used to
check the library's tensor-core forward pass and its FP32 gradients.
"""
import numpy as np
from scipy.special import erf

IN, HID, OUT = 35, 128, 3
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, HID)), ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even)."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def _gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def _gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p, x, act_bf16=False):
    """Outputs for inputs x[n][35]; act_bf16 rounds every layer input to BF16
    (what the tensor-core path feeds its MMAs)."""
    w = unpack(p)
    h = np.asarray(x, np.float64)
    for l in (1, 2, 3):
        hin = bf16(h).astype(np.float64) if act_bf16 else h
        h = _gelu(hin @ bf16(w[f"W{l}"]).astype(np.float64).T + w[f"b{l}"])
    hin = bf16(h).astype(np.float64) if act_bf16 else h
    return hin @ bf16(w["W4"]).astype(np.float64).T + w["b4"]


def gradients(p, x, t):
    """(loss, flat gradient) in FP64 for the FP32 training path's definition."""
    w = unpack(p)
    W = {k: bf16(w[k]).astype(np.float64) for k in ("W1", "W2", "W3", "W4")}
    x = np.asarray(x, np.float64)
    zs, hs = [], [x]
    h = x
    for l in (1, 2, 3):
        z = h @ W[f"W{l}"].T + w[f"b{l}"]
        zs.append(z)
        h = _gelu(z)
        hs.append(h)
    y = h @ W["W4"].T + w["b4"]
    n = y.size
    loss = np.sum((y - t) ** 2) / n
    dz = 2.0 * (y - t) / n
    g = {"W4": dz.T @ hs[3], "b4": dz.sum(0)}
    da = (dz @ W["W4"]) * _gelu_grad(zs[2])
    for l in (3, 2, 1):
        g[f"W{l}"] = da.T @ hs[l - 1]
        g[f"b{l}"] = da.sum(0)
        if l > 1:
            da = (da @ W[f"W{l}"]) * _gelu_grad(zs[l - 2])
    flat = np.concatenate([g[name].ravel() for name, _ in SHAPES])
    return loss, flat


def init_params(seed):
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("b"):
            parts.append(rng.normal(0, 0.05, shape).ravel())
        else:
            parts.append(rng.uniform(-1, 1, shape).ravel() * np.sqrt(3.0 / shape[1]))
    return np.concatenate(parts).astype(np.float32)
