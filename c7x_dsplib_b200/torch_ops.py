"""PyTorch operators over the C ABI: ``torch.ops.dsplib_gpu.*``.

    import c7x_dsplib_b200.torch_ops          # registers the operators
    y = torch.ops.dsplib_gpu.fir(x, h, False, 0, False, 0)
    y = torch.ops.dsplib_gpu.cascade_biquad(x, coef, state, form, nch)   # updates state in place
    q = torch.ops.dsplib_gpu.fltoq15(x, 1)
    f = torch.ops.dsplib_gpu.q15tofl(q, torch.float32)

Each operator launches the library's kernels on the caller's current CUDA stream
without synchronising (the asynchronous mode of the C ABI), so the ops compose with
other stream work and with CUDA-graph capture; the fake (meta) implementations give
output shapes and dtypes for tracing.  Inputs must be CUDA tensors; the arithmetic
contract of each op is that of the DSPLIB entry point it calls.
"""
from __future__ import annotations

import torch

import c7x_dsplib_b200 as D

_LIB = "dsplib_gpu"


def _cuda(*ts):
    for t in ts:
        if not t.is_cuda:
            raise ValueError("dsplib_gpu operators take CUDA tensors")


@torch.library.custom_op(f"{_LIB}::fir", mutates_args=())
def fir(x: torch.Tensor, h: torch.Tensor, nch: bool, precision: int, qmode: bool, shift: int) -> torch.Tensor:
    """DSPLIB_fir (OPTIMIZED) over channel-major rows x [batch, N] with stored taps
    h [1 or batch, T]; returns [batch, N - T + 1] in x's dtype.  precision: 0 FP32
    CUDA cores, 1 split-BF16x3 tensor cores (FLOAT32); qmode: integer Q-mode output."""
    _cuda(x, h)
    x, h = x.contiguous(), h.contiguous()
    batch, n = x.shape
    T = h.shape[1]
    out = torch.empty((batch, n - T + 1), dtype=x.dtype, device=x.device)
    D.fir(x, h, T, nch=nch, precision=precision, qmode=qmode, shift=shift, out=out,
          stream=torch.cuda.current_stream())
    return out


@fir.register_fake
def _(x, h, nch, precision, qmode, shift):
    return x.new_empty((x.shape[0], x.shape[1] - h.shape[1] + 1))


@torch.library.custom_op(f"{_LIB}::cascade_biquad", mutates_args=("state",))
def cascade_biquad(x: torch.Tensor, coef: torch.Tensor, state: torch.Tensor, form: int, nch: bool) -> torch.Tensor:
    """DSPLIB_cascadeBiquad (OPTIMIZED) over time-major x [N, C] (FLOAT32) with the
    optimized coefficient buffer; state [S * nv, C] is read and updated in place."""
    _cuda(x, coef, state)
    out = torch.empty_like(x)
    D.cascade_biquad(x.contiguous(), coef.contiguous(), state, form=form, nch=nch, out=out,
                     stream=torch.cuda.current_stream())
    return out


@cascade_biquad.register_fake
def _(x, coef, state, form, nch):
    return torch.empty_like(x)


@torch.library.custom_op(f"{_LIB}::fltoq15", mutates_args=())
def fltoq15(x: torch.Tensor, func_style: int) -> torch.Tensor:
    """DSPLIB_fltoq15: FLOAT32 / FLOAT64 -> Q.15 int16 (flattened)."""
    _cuda(x)
    out = torch.empty(x.numel(), dtype=torch.int16, device=x.device)
    D.fltoq15(x.contiguous().view(-1), func_style=func_style, out=out, stream=torch.cuda.current_stream())
    return out


@fltoq15.register_fake
def _(x, func_style):
    return x.new_empty(x.numel(), dtype=torch.int16)


@torch.library.custom_op(f"{_LIB}::q15tofl", mutates_args=())
def q15tofl(x: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """DSPLIB_q15tofl: Q.15 int16 -> FLOAT32 / FLOAT64 (flattened)."""
    _cuda(x)
    out = torch.empty(x.numel(), dtype=dtype, device=x.device)
    npdt = {torch.float32: "float32", torch.float64: "float64"}[dtype]
    import numpy as np

    D.q15tofl(x.contiguous().view(-1), np.dtype(npdt), out=out, stream=torch.cuda.current_stream())
    return out


@q15tofl.register_fake
def _(x, dtype):
    return x.new_empty(x.numel(), dtype=dtype)
