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


# ---------------------------------------------------------------- autograd

def _fir_setup(ctx, inputs, output):
    x, h, nch, precision, qmode, shift = inputs
    ctx.save_for_backward(x, h)
    ctx.nch = nch


def _fir_backward(ctx, gy):
    """y[l, j] = sum_c x[l, j + c] h[T - 1 - c]  (FLOAT32 only):
    dx = FIR of gy zero-padded by T - 1 on both sides with the taps flipped (a full
    convolution with the taps), dh[T - 1 - c] = sum_j gy[j] x[j + c], the FIR of x
    with each channel's flipped gradient as its taps.  Both on the library's kernels."""
    x, h = ctx.saved_tensors
    if x.dtype != torch.float32:
        raise RuntimeError("dsplib_gpu::fir is differentiable for FLOAT32 only")
    T = h.shape[1]
    gy = gy.contiguous()
    gx = gh = None
    if ctx.needs_input_grad[0]:
        pad = torch.nn.functional.pad(gy, (T - 1, T - 1))
        hf = torch.flip(h, dims=[1]).contiguous()
        gx = torch.ops.dsplib_gpu.fir(pad, hf, bool(ctx.nch), 0, False, 0)
    if ctx.needs_input_grad[1]:
        lag = torch.ops.dsplib_gpu.fir(x.contiguous(), torch.flip(gy, dims=[1]).contiguous(), True, 0, False, 0)
        gh = torch.flip(lag, dims=[1])
        if not ctx.nch:
            gh = gh.sum(dim=0, keepdim=True)
    return gx, gh, None, None, None, None


fir.register_autograd(_fir_backward, setup_context=_fir_setup)


_PLANS = {}


def _bank_plan(C, N, S, device):
    """A filter-bank plan of C channels of N samples, one tap, S stages: the cascade alone."""
    from .filterbank import RaggedFilterBank

    key = (C, N, S, str(device))
    if key not in _PLANS:
        _PLANS[key] = RaggedFilterBank([N] * C, [1] * C, [S] * C, device=device)
    return _PLANS[key]


@torch.library.custom_op(f"{_LIB}::cascade_biquad_natural", mutates_args=())
def cascade_biquad_natural(x: torch.Tensor, coef: torch.Tensor, form: int) -> torch.Tensor:
    """Differentiable DSPLIB_cascadeBiquad (OPTIMIZED) from a zero state over time-major
    x [N, C] (FLOAT32) with natural coefficients coef [1 or C, 5 S] ([b0 b1 b2 a1 a2] per
    stage); the optimized buffer comes from DSPLIB_cascadeBiquad_get_coefficients on the
    device.  Gradients w.r.t. x and coef (every form has the transfer function of the
    natural coefficients; the adjoint is the filter-bank adjoint)."""
    _cuda(x, coef)
    x, coef = x.contiguous(), coef.contiguous()
    N, C = x.shape
    S = coef.shape[1] // 5
    nch = coef.shape[0] > 1
    nv = 4 if form == D.DF1 else 2
    state = torch.zeros((S * nv, C), device=x.device)
    if form == D.TIF or nch:
        import ctypes

        args, pin, pout, pvar, pcn, popt = D.biquad_descs(C, N, S, form, nch)
        opt = torch.zeros(popt.dim_y * popt.stride_y // 4, device=x.device)
        st = D.lib().DSPLIB_cascadeBiquad_get_coefficients(form, int(nch), ctypes.byref(pcn), ctypes.byref(popt),
                                                           coef.data_ptr(), opt.data_ptr())
        if st != D.SUCCESS:
            raise D.DsplibError("DSPLIB_cascadeBiquad_get_coefficients", st)
    else:
        opt = coef
    out = torch.empty_like(x)
    D.cascade_biquad(x, opt, state, form=form, nch=nch, out=out, stream=torch.cuda.current_stream())
    return out


@cascade_biquad_natural.register_fake
def _(x, coef, form):
    return torch.empty_like(x)


def _bq_setup(ctx, inputs, output):
    x, coef, form = inputs
    ctx.save_for_backward(x, coef)


def _bq_backward(ctx, gy):
    x, coef = ctx.saved_tensors
    N, C = x.shape
    S = coef.shape[1] // 5
    bank = _bank_plan(C, N, S, x.device)
    coefs = (coef if coef.shape[0] == C else coef.expand(C, -1)).contiguous().view(-1)
    xp = x.t().contiguous().view(-1)
    taps = torch.ones(C, device=x.device)
    y = torch.empty(bank.sizes[0], device=x.device)
    work = torch.empty(bank.sizes[3], device=x.device)
    bank.forward_raw(xp, taps, coefs, y, work)
    gx = torch.empty_like(xp)
    gt = torch.empty_like(taps)
    gc = torch.empty_like(coefs)
    scratch = torch.empty(bank.sizes[4], device=x.device)
    bank.backward_raw(xp, taps, coefs, work, gy.t().contiguous().view(-1), gx, gt, gc, scratch)
    gc = gc.view(C, 5 * S)
    if coef.shape[0] == 1:
        gc = gc.sum(dim=0, keepdim=True)
    return gx.view(C, N).t().contiguous(), gc, None


cascade_biquad_natural.register_autograd(_bq_backward, setup_context=_bq_setup)
