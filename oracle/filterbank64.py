"""FP64 numpy restatement of the batched FIR -> cascaded-biquad filter bank and
its adjoint, the oracle the CUDA path is checked against.  TEST INFRASTRUCTURE
ONLY (imported by tests/, __graft_entry__.smoke() and bench.py's CPU leg).

FIR: u[j] = sum_{c<T} x[j+c] h[T-1-c] (src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54),
i.e. ``np.convolve(x, h, "valid")``.  Each stage is the direct-form-II
section of src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_cn.cpp with natural
coefficients [b0 b1 b2 a1 a2] and a zero initial state, i.e.
``scipy.signal.lfilter([b0, b1, b2], [1, a1, a2], u)``.
"""
from __future__ import annotations

import numpy as np
from scipy.signal import lfilter


def stable_sections(rng, S, radius=(0.3, 0.9)):
    """S random stable sections: complex pole pairs of radius in ``radius``,
    zeros anywhere in the unit disc, gain normalised to about 1 at DC."""
    out = np.zeros((S, 5))
    for s in range(S):
        r = rng.uniform(*radius)
        th = rng.uniform(0.05, np.pi - 0.05)
        a1, a2 = -2 * r * np.cos(th), r * r
        rz = rng.uniform(0.0, 1.0)
        tz = rng.uniform(0.0, np.pi)
        b = np.array([1.0, -2 * rz * np.cos(tz), rz * rz])
        g = (1 + a1 + a2) / max(abs(b.sum()), 0.2)
        out[s] = [b[0] * g, b[1] * g, b[2] * g, a1, a2]
    return out


def channel_forward(x, h, coefs):
    """Returns (y, stage inputs list) in FP64; coefs (S, 5)."""
    u = np.convolve(np.asarray(x, np.float64), np.asarray(h, np.float64), "valid")
    acts = [u]
    for b0, b1, b2, a1, a2 in np.asarray(coefs, np.float64).reshape(-1, 5):
        acts.append(lfilter([b0, b1, b2], [1.0, a1, a2], acts[-1]))
    return acts[-1], acts


def channel_adjoint(x, h, coefs, gy):
    """dLoss/dx, dLoss/dh, dLoss/dcoefs (S, 5) for dLoss/dy = gy, in FP64."""
    x = np.asarray(x, np.float64)
    h = np.asarray(h, np.float64)
    coefs = np.asarray(coefs, np.float64).reshape(-1, 5)
    _, acts = channel_forward(x, h, coefs)
    g = np.asarray(gy, np.float64).copy()
    gc = np.zeros_like(coefs)
    for s in range(len(coefs) - 1, -1, -1):
        b0, b1, b2, a1, a2 = coefs[s]
        u, y = acts[s], acts[s + 1]
        v = lfilter([1.0], [1.0, a1, a2], g[::-1])[::-1]
        vp = np.concatenate([v, [0.0, 0.0]])
        g = b0 * vp[:-2] + b1 * vp[1:-1] + b2 * vp[2:]
        gc[s] = [v @ u, v[1:] @ u[:-1], v[2:] @ u[:-2], -(v[1:] @ y[:-1]), -(v[2:] @ y[:-2])]
    gx = np.convolve(g, h[::-1], "full")
    gh = np.correlate(x, g, "valid")[::-1]
    return gx, gh, gc


def bank_forward(lengths, taps, stages, x, h, c):
    """Packed FP64 forward over all channels (y tail samples zero)."""
    y = np.zeros(len(x))
    xo = ho = co = 0
    for L, T, S in zip(lengths, taps, stages):
        yc, _ = channel_forward(x[xo:xo + L], h[ho:ho + T], c[co:co + 5 * S])
        y[xo:xo + L - T + 1] = yc
        xo, ho, co = xo + L, ho + T, co + 5 * S
    return y


def bank_adjoint(lengths, taps, stages, x, h, c, gy):
    gx = np.zeros(len(x))
    gh = np.zeros(len(h))
    gc = np.zeros(len(c))
    xo = ho = co = 0
    for L, T, S in zip(lengths, taps, stages):
        a, b, d = channel_adjoint(x[xo:xo + L], h[ho:ho + T], c[co:co + 5 * S], gy[xo:xo + L - T + 1])
        gx[xo:xo + L], gh[ho:ho + T], gc[co:co + 5 * S] = a, b, d.reshape(-1)
        xo, ho, co = xo + L, ho + T, co + 5 * S
    return gx, gh, gc
