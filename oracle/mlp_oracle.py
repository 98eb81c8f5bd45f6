"""CPU oracle of the learned scheduler's network (test infrastructure only).

Restates, in numpy float64, what kpp_b200/csrc/kpp_sched.cu computes:
  forward   P_l = In_l W_l^T + b_l, H_l = bf16(gelu(P_l)) (erf form) for the
            hidden layers, O = H W^T + b for the output layer;
  loss      mean((O - Y)^2) over all entries; dO = 2 (O - Y) / count;
  backward  dW_l = bf16(dZ_l)^T In_l, db_l = colsum(dZ_l) (unrounded dZ),
            dZ_{l-1} = (bf16(dZ_l) W_l) * gelu'(P_{l-1});
  Adam      m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
            w -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps).
The BF16 roundings sit where the device stores BF16 (weights, inputs, hidden
activations, the gradients fed to the tensor cores), so the device and this
oracle differ only by FP32 versus float64 accumulation.  `exact=True` drops
every rounding for the finite-difference self-check of the gradients.

No reference counterpart: KPP has no learned component.  Parity here is
against the mathematics above, pinned by tests/test_sched_oracle.py
(finite differences, torch's BF16 conversion, torch.optim.Adam).
"""
from __future__ import annotations

import math

import numpy as np

_SQRT1_2 = 1.0 / math.sqrt(2.0)
_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x * _SQRT1_2))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x * _SQRT1_2))
    pdf = np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
    return cdf + x * pdf


def layer_shapes(nin: int, width: int, nhidden: int, nout: int):
    fin = [nin] + [width] * nhidden
    fout = [width] * nhidden + [nout]
    return list(zip(fout, fin))


def unpack(params: np.ndarray, shapes):
    """Split the flat parameter vector (W_l [out][in] then b_l per layer)."""
    out, off = [], 0
    for fo, fi in shapes:
        w = params[off:off + fo * fi].reshape(fo, fi)
        off += fo * fi
        b = params[off:off + fo]
        off += fo
        out.append((w, b))
    assert off == params.size
    return out


def pack(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def init_params(nin: int, width: int, nhidden: int, nout: int, seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases."""
    rng = np.random.default_rng(seed)
    layers = []
    for fo, fi in layer_shapes(nin, width, nhidden, nout):
        a = 1.0 / math.sqrt(fi)
        layers.append((rng.uniform(-a, a, (fo, fi)), rng.uniform(-a, a, fo)))
    return pack(layers).astype(np.float32)


def forward(params, shapes, x_rows, exact=False):
    """x_rows [batch][nin] (already BF16 values unless exact).  Returns the
    output and the per-layer (input, pre-activation) pairs."""
    r = (lambda a: a) if exact else bf16
    layers = unpack(np.asarray(params, dtype=np.float64), shapes)
    h = np.asarray(x_rows, dtype=np.float64)
    cache = []
    for li, (w, b) in enumerate(layers):
        wq = w if exact else r(w)
        p = h @ wq.T + b
        cache.append((h, p))
        h = r(gelu(p)) if li + 1 < len(layers) else p
    return h, cache


def loss_grad(params, shapes, x_rows, y, exact=False):
    """Loss and the flat gradient, in the parameter layout."""
    r = (lambda a: a) if exact else bf16
    layers = unpack(np.asarray(params, dtype=np.float64), shapes)
    o, cache = forward(params, shapes, x_rows, exact)
    e = o - y
    count = e.size
    loss = float((e * e).sum() / count)
    dz = 2.0 * e / count
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        w, _ = layers[li]
        h_in, _ = cache[li]
        dzq = r(dz)
        grads[li] = (dzq.T @ h_in, dz.sum(axis=0))
        if li == 0:
            break
        wq = w if exact else r(w)
        dz = (dzq @ wq) * gelu_grad(cache[li - 1][1])
    return loss, pack(grads)


def adam(w, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1.0 - b1) * g
    v = b2 * v + (1.0 - b2) * g * g
    mh = m / (1.0 - b1 ** t)
    vh = v / (1.0 - b2 ** t)
    return w - lr * mh / (np.sqrt(vh) + eps), m, v
