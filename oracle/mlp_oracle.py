"""ORACLE — TEST INFRASTRUCTURE ONLY.

numpy restatement of the learned closure's network, its training step and
its minibatch sampling, used by tests/ to check the GPU kernels
(phi_eng_b200/csrc/sph_mlp.cu, sph_mlp.cuh). The network has no reference
counterpart; this file states its definition:

  x_hat = bf16((x - mu) * isd)                      (float32 ops, then BF16)
  z1 = W1 x_hat + b1,  h1 = silu(z1)
  z2 = W2 h1 + b2,     h2 = silu(z2)
  y  = W3 h2 + b3,     output = y * out_scale
  W1 rounded to BF16, W2 and W3 to FP16 (the backward's W2 to BF16); biases
  FP32; products accumulated exactly here (FP32 on the tensor cores).
  loss = 1/(2B) sum_b |y_b - t_b / out_scale|^2

The kernels evaluate silu(z) = u + u tanh(u), u = z / 2 (the hidden layers
run on halved weights and biases, so the accumulators hold u), on FP16
pairs: u rounded to FP16, the hardware's FP16 tanh, one FP16 fused
multiply-add (act_f16). Layers 2 and 3 take those FP16 activations; dW2
takes them rounded to BF16.

emulate=True reproduces the GPU's BF16 rounding points (to compare against
the kernels within a tolerance: accumulation order and the hardware tanh
differ); emulate=False is the plain float64 network, used to validate the
analytic backward pass by finite differences.
"""
from __future__ import annotations

import numpy as np

FEAT, HID, OUT = 16, 64, 2
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * FEAT
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
NPARAMS = OFF_B3 + OUT
NNORM = 2 * FEAT + OUT
BETA1, BETA2, ADAM_EPS = np.float32(0.9), np.float32(0.999), np.float32(1e-8)

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)
_M3 = np.uint64(0x94D049BB133111EB)


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest bfloat16, ties to even (as float32)."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (((u + np.uint64(0x7FFF) + ((u >> np.uint64(16)) & np.uint64(1))) >> np.uint64(16)) << np.uint64(16))
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def unpack(p):
    p = np.asarray(p)
    return (p[OFF_W1:OFF_B1].reshape(HID, FEAT), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(OUT, HID), p[OFF_B3:NPARAMS])


def pack(W1, b1, W2, b2, W3, b3) -> np.ndarray:
    return np.concatenate([np.ravel(W1), b1, np.ravel(W2), b2, np.ravel(W3), b3])


def sigmoid(z):
    return 0.5 * np.tanh(0.5 * z) + 0.5


def silu(z):
    return z * sigmoid(z)


def dsilu(z):
    s = sigmoid(z)
    return s + z * s * (1.0 - s)


def f16(x) -> np.ndarray:
    """Round to the nearest FP16, ties to even (as float64)."""
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def act_f16(z):
    """silu(z) at the kernels' rounding points: u = f16(z / 2),
    f16(u + u * f16(tanh(u))) (the last a fused multiply-add)."""
    u = f16(np.clip(0.5 * z, -65504.0, 65504.0))
    t = f16(np.tanh(u))
    return f16(u + u * t)


def normalise(x, norm, emulate=True):
    x32 = np.asarray(x, dtype=np.float32)
    mu = np.asarray(norm[:FEAT], dtype=np.float32)
    isd = np.asarray(norm[FEAT:2 * FEAT], dtype=np.float32)
    xn = (x32 - mu) * isd  # float32 arithmetic, as the kernels
    return (bf16(xn) if emulate else xn).astype(np.float64)


def forward(params, norm, x, emulate=True):
    """Network output (times out_scale) and the intermediates."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(params, dtype=np.float32))
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float32))
    h = f16 if emulate else (lambda a: np.asarray(a, dtype=np.float32).astype(np.float64))
    W1b, W2b = (r(W).astype(np.float64) for W in (W1, W2))
    W2h, W3h = h(W2), h(W3)
    xh = normalise(x, norm, emulate)
    z1 = xh @ W1b.T + b1.astype(np.float64)
    h1 = act_f16(z1) if emulate else silu(z1)
    z2 = h1 @ W2h.T + b2.astype(np.float64)
    h2 = act_f16(z2) if emulate else silu(z2)
    y = h2 @ W3h.T + b3.astype(np.float64)
    os_ = np.asarray(norm[2 * FEAT:], dtype=np.float64)
    h1g = bf16(h1.astype(np.float32)).astype(np.float64) if emulate else h1
    cache = dict(xh=xh, z1=z1, h1=h1, h1g=h1g, z2=z2, h2=h2, y=y, W1b=W1b, W2b=W2b, W3b=W3h)
    return y * os_, cache


def loss_grad(params, norm, x, t, emulate=True):
    """Loss and gradient (flat, float64) of one minibatch."""
    B = x.shape[0]
    _, c = forward(params, norm, x, emulate)
    os_ = np.asarray(norm[2 * FEAT:], dtype=np.float32)
    inv_os = (np.float32(1.0) / os_)
    th = (np.asarray(t, dtype=np.float32) * inv_os).astype(np.float64)
    e = c["y"] - th
    loss = float(np.sum(e * e) / (2.0 * B))
    dy = e / B
    dW3 = dy.T @ c["h2"]
    db3 = dy.sum(0)
    dz2 = (dy @ c["W3b"]) * dsilu(c["z2"])
    dz2g = bf16(dz2.astype(np.float32)).astype(np.float64) if emulate else dz2
    dW2 = dz2g.T @ c["h1g"]
    db2 = dz2.sum(0)
    dz1 = (dz2g @ c["W2b"]) * dsilu(c["z1"])
    dz1g = bf16(dz1.astype(np.float32)).astype(np.float64) if emulate else dz1
    dW1 = dz1g.T @ c["xh"]
    db1 = dz1.sum(0)
    return loss, pack(dW1, db1, dW2, db2, dW3, db3)


def adam(w, m, v, g, t, lr):
    """One Adam step (step number t >= 1) in float32, as k_mlp_adam."""
    w, m, v, g = (np.asarray(a, dtype=np.float32) for a in (w, m, v, g))
    one = np.float32(1.0)
    mm = BETA1 * m + (one - BETA1) * g
    vv = BETA2 * v + (one - BETA2) * (g * g)
    bc1 = np.float32(1.0 - np.float64(BETA1) ** t)
    bc2 = np.float32(1.0 - np.float64(BETA2) ** t)
    upd = (mm / bc1) / (np.sqrt(vv / bc2) + ADAM_EPS)
    return w - np.float32(lr) * upd, mm, vv


def mix64(z):
    z = np.asarray(z, dtype=np.uint64) + _M1
    z = (z ^ (z >> np.uint64(30))) * _M2
    z = (z ^ (z >> np.uint64(27))) * _M3
    return z ^ (z >> np.uint64(31))


def sample_indices(seed: int, it: int, batch: int, npairs: int) -> np.ndarray:
    """Pair indices of minibatch `it`: (mix64(seed ^ (it << 32) ^ k) >> 32) * npairs >> 32."""
    with np.errstate(over="ignore"):
        k = np.arange(batch, dtype=np.uint64)
        h = mix64(np.uint64(seed) ^ (np.uint64(it) << np.uint64(32)) ^ k)
        return (((h >> np.uint64(32)) * np.uint64(npairs)) >> np.uint64(32)).astype(np.int64)


def init_params(seed: int) -> np.ndarray:
    """phieng_mlp_new's initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from
    SplitMix64(seed) for W1, b1 (fan_in 16), W2, b2 (fan_in 64); W3, b3 zero."""
    out = np.zeros(NPARAMS, dtype=np.float32)
    s = np.uint64(seed)
    vals = []
    with np.errstate(over="ignore"):
        for count, bound in ((HID * FEAT, 0.25), (HID, 0.25), (HID * HID, 0.125), (HID, 0.125)):
            k = np.arange(count, dtype=np.uint64)
            z = mix64(s + k * _M1)
            s = s + np.uint64(count) * _M1
            u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            vals.append(((2.0 * u - 1.0) * bound).astype(np.float32))
    out[OFF_W1:OFF_B1], out[OFF_B1:OFF_W2], out[OFF_W2:OFF_B2], out[OFF_B2:OFF_W3] = vals
    return out
