"""CPU timing baseline for the batched FIR -> cascaded-biquad filter bank step
(forward, MSE loss gradient, adjoint), composed of the reference's own
natural-C kernels (oracle/_ref): test and benchmark infrastructure only.

Per channel (length L, T taps, S direct-form-II stages, natural [b0 b1 b2 a1 a2]):
  forward   u = DSPLIB_fir_cn(x, h)                      (src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54)
            y_s = DSPLIB_cascadeBiquad_cn DF2, one stage at a time (every stage
                  output is kept for the adjoint)          (src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_cn.cpp)
  loss      gy = 2 (y - target) / n
  adjoint   per stage, last first:
              v  = the same biquad kernel with [1 0 0 a1 a2] on time-reversed g, reversed back
              gu = FIR of [v 0 0] with taps [b2 b1 b0]
              d[b0 b1 b2] = (v.u, v[1:].u[:-1], v[2:].u[:-2]); d[a1 a2] = -(v[1:].y[:-1], v[2:].y[:-2])
            gx = FIR of [0^(T-1) g 0^(T-1)] with the taps reversed
            gh = FIR of x with "taps" g reversed, reversed
Channels are spread over a thread pool (the kernels release the GIL).
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import biquad, fir


def _fir1(x, taps):
    """Valid correlation y[j] = sum_c x[j+c] taps[T-1-c] by the reference FIR kernel (one channel)."""
    T = len(taps)
    return fir(x[None, :], np.asarray(taps, np.float32)[None, :], T, nch=0, impl="ref")[0]


def _df2_1(u, row):
    st = np.zeros((2, 1), np.float32)
    return biquad(2, u[:, None], np.asarray(row, np.float32)[None, :], st, nch=0, impl="ref")[:, 0]


def channel_step(x, h, coefs, target, n_total):
    """One channel's forward + adjoint; returns (loss part, gx, gh, gcoefs)."""
    x = np.asarray(x, np.float32)
    acts = [_fir1(x, h)]
    for row in coefs:
        acts.append(_df2_1(acts[-1], row))
    y = acts[-1]
    d = y - target
    loss = float(d @ d) / n_total
    g = (d * (2.0 / n_total)).astype(np.float32)
    gc = np.zeros_like(coefs)
    z2 = np.zeros(2, np.float32)
    for s in range(len(coefs) - 1, -1, -1):
        b0, b1, b2, a1, a2 = coefs[s]
        u, ys = acts[s], acts[s + 1]
        v = _df2_1(np.ascontiguousarray(g[::-1]), [1.0, 0.0, 0.0, a1, a2])[::-1]
        v = np.ascontiguousarray(v)
        gc[s] = [v @ u, v[1:] @ u[:-1], v[2:] @ u[:-2], -(v[1:] @ ys[:-1]), -(v[2:] @ ys[:-2])]
        g = _fir1(np.concatenate([v, z2]), [b2, b1, b0])
    T = len(h)
    zt = np.zeros(T - 1, np.float32)
    gx = _fir1(np.concatenate([zt, g, zt]), np.asarray(h[::-1]))
    gh = _fir1(x, np.ascontiguousarray(g[::-1]))[::-1]
    return loss, gx, gh, gc


def bank_step_sample(lengths, taps, stages, x, h, c, target, channels, threads, n_total):
    """Run channel_step over ``channels`` (indices) on ``threads`` workers; returns (seconds, samples)."""
    xo = np.concatenate([[0], np.cumsum(lengths)])
    ho = np.concatenate([[0], np.cumsum(taps)])
    co = np.concatenate([[0], 5 * np.cumsum(stages)])

    def one(ch):
        L, T, S = int(lengths[ch]), int(taps[ch]), int(stages[ch])
        return channel_step(x[xo[ch]:xo[ch] + L], h[ho[ch]:ho[ch] + T], c[co[ch]:co[ch] + 5 * S].reshape(S, 5),
                            target[xo[ch]:xo[ch] + L - T + 1], n_total)

    t0 = time.perf_counter()
    if threads > 1:
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(one, channels))
    else:
        for ch in channels:
            one(ch)
    return time.perf_counter() - t0, int(sum(int(lengths[ch]) for ch in channels))
