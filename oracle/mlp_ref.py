"""CPU reference of the picker MLP (test infrastructure).

Float64 forward and backward of the engine's MLP (csrc/bine_mlp.cu) with the
same bf16 rounding points: inputs, weights, hidden activations and the
backpropagated gradients are rounded to bf16 (round to nearest even) where
the kernels round them; everything else is float64 instead of the kernels'
fp32 accumulation.  GELU is the exact erf form.
"""
import math

import numpy as np

try:  # scipy's erf is a vectorised double-precision erf; math.erf otherwise
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def bf16(x):
    """Round float32 values to bf16 (nearest even), returned as float64."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unpack(params, layout):
    Ws, bs = [], []
    for w, b, nout, nin in layout:
        Ws.append(params[w:w + nout * nin].reshape(nout, nin).astype(np.float64))
        bs.append(params[b:b + nout].astype(np.float64))
    return Ws, bs


def forward(params, layout, x, rounding=True):
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    Ws, bs = unpack(params, layout)
    a = r(x)
    pres, acts = [], [a]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        pre = a @ r(W).T + b
        pres.append(pre)
        if l + 1 < len(Ws):
            a = r(gelu(pre).astype(np.float32)) if rounding else gelu(pre)
            acts.append(a)
    return pres, acts


def loss_and_grads(params, layout, x, t, mask, rounding=True):
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    Ws, bs = unpack(params, layout)
    pres, acts = forward(params, layout, x, rounding)
    y = pres[-1]
    cnt = max(1.0, float((mask != 0).sum()))
    d = mask * (y - t)
    loss = float((d * d).sum() / cnt)
    g = np.zeros(params.size, np.float64)
    dpre = r((2.0 * d / cnt).astype(np.float32)) if rounding else 2.0 * d / cnt
    for l in range(len(Ws) - 1, -1, -1):
        w, b, nout, nin = layout[l]
        g[w:w + nout * nin] = (dpre.T @ acts[l]).reshape(-1)
        g[b:b + nout] = dpre.sum(0)
        if l > 0:
            dact = dpre @ r(Ws[l])
            dp = dact * gelu_grad(pres[l - 1])
            dpre = r(dp.astype(np.float32)) if rounding else dp
    return loss, g
