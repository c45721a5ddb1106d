"""Batched FIR -> cascaded-biquad filter bank over channels of uneven length,
with gradients, on the C ABI's ``DSPLIB_gpu_firBiquadBatched_fwd/bwd``.

Per channel c: ``u_c = DSPLIB_fir(x_c, h_c)`` (valid correlation, the tap
order of src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54) followed by ``S_c`` direct-form-II
biquads from a zero state (the DF2 recurrence of
src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_cn.cpp, natural coefficients
[b0 b1 b2 a1 a2] per stage).  Channels are packed back to back (see
``include/dsplib_gpu.h``); ``RaggedFilterBank.pack`` / ``unpack`` convert from
and to lists of per-channel tensors.

``RaggedFilterBank.apply(x, taps, coefs)`` is differentiable in all three
inputs (``torch.autograd.Function`` whose forward and backward are one C-ABI
call each, queued on torch's current stream).  ``graph_step`` captures a
forward + backward into a CUDA graph for a fixed plan.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import DsplibError, SUCCESS, lib

SAMPLES, TAPS, COEFS, WORK, SCRATCH, OUTPUTS = 0, 1, 2, 3, 4, 5


def _stream_ptr():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class RaggedFilterBank:
    """Plan for a fixed set of channel lengths, tap counts and stage counts."""

    def __init__(self, lengths, taps, stages, device=None):
        import torch

        self.lengths = np.asarray(lengths, dtype=np.int32)
        self.taps = np.asarray(taps, dtype=np.int32)
        self.stages = np.asarray(stages, dtype=np.int32)
        C = len(self.lengths)
        if not (len(self.taps) == C and len(self.stages) == C):
            raise ValueError("lengths, taps and stages must have one entry per channel")
        self.device = torch.device(device if device is not None else "cuda")
        L = lib()
        self._plan = ctypes.c_void_p()
        i32 = ctypes.POINTER(ctypes.c_int32)
        with torch.cuda.device(self.device):
            st = L.DSPLIB_gpu_raggedPlanCreate(ctypes.byref(self._plan), C, self.lengths.ctypes.data_as(i32),
                                               self.taps.ctypes.data_as(i32), self.stages.ctypes.data_as(i32))
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_raggedPlanCreate", st)
        self.x_off = np.concatenate([[0], np.cumsum(self.lengths.astype(np.int64))])
        self.h_off = np.concatenate([[0], np.cumsum(self.taps.astype(np.int64))])
        self.c_off = np.concatenate([[0], 5 * np.cumsum(self.stages.astype(np.int64))])
        self.out_lengths = self.lengths - self.taps + 1
        self.sizes = {k: int(L.DSPLIB_gpu_raggedPlanSize(self._plan, k)) for k in (SAMPLES, TAPS, COEFS, WORK,
                                                                                   SCRATCH, OUTPUTS)}

    def __del__(self):
        if getattr(self, "_plan", None) is not None and self._plan.value:
            try:
                lib().DSPLIB_gpu_raggedPlanDestroy(self._plan)
            except Exception:
                pass
            self._plan = None

    @property
    def num_channels(self):
        return len(self.lengths)

    # ---------------------------------------------------------------- packing
    def pack(self, parts, kind="x"):
        """Concatenate per-channel tensors (x: length L_c; taps: T_c; coefs: (S_c, 5))."""
        import torch

        return torch.cat([p.reshape(-1) for p in parts]).contiguous()

    def unpack(self, flat, kind="y"):
        """Split a packed tensor back into per-channel views (y: first L_c - T_c + 1 samples)."""
        if kind in ("x", "y"):
            out = [flat[self.x_off[c]:self.x_off[c + 1]] for c in range(self.num_channels)]
            if kind == "y":
                out = [o[:self.out_lengths[c]] for c, o in enumerate(out)]
            return out
        if kind == "taps":
            return [flat[self.h_off[c]:self.h_off[c + 1]] for c in range(self.num_channels)]
        if kind == "coefs":
            return [flat[self.c_off[c]:self.c_off[c + 1]].reshape(-1, 5) for c in range(self.num_channels)]
        raise ValueError(kind)

    # ---------------------------------------------------------------- raw calls
    def _check(self, t, n, name):
        import torch

        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.numel() == n):
            raise ValueError(f"{name}: need a contiguous float32 CUDA tensor of {n} elements")

    def forward_raw(self, x, taps, coefs, y, work):
        self._check(x, self.sizes[SAMPLES], "x")
        self._check(taps, self.sizes[TAPS], "taps")
        self._check(coefs, self.sizes[COEFS], "coefs")
        self._check(y, self.sizes[SAMPLES], "y")
        self._check(work, self.sizes[WORK], "work")
        st = lib().DSPLIB_gpu_firBiquadBatched_fwd(self._plan, x.data_ptr(), taps.data_ptr(), coefs.data_ptr(),
                                                  y.data_ptr(), work.data_ptr(), _stream_ptr())
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_firBiquadBatched_fwd", st)

    def backward_raw(self, x, taps, coefs, work, gy, gx, gtaps, gcoefs, scratch):
        self._check(gy, self.sizes[SAMPLES], "gy")
        self._check(gx, self.sizes[SAMPLES], "gx")
        self._check(gtaps, self.sizes[TAPS], "gtaps")
        self._check(gcoefs, self.sizes[COEFS], "gcoefs")
        self._check(scratch, self.sizes[SCRATCH], "scratch")
        st = lib().DSPLIB_gpu_firBiquadBatched_bwd(self._plan, x.data_ptr(), taps.data_ptr(), coefs.data_ptr(),
                                                  work.data_ptr(), gy.data_ptr(), gx.data_ptr(), gtaps.data_ptr(),
                                                  gcoefs.data_ptr(), scratch.data_ptr(), _stream_ptr())
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_firBiquadBatched_bwd", st)

    def mse_grad_raw(self, y, target, gy, loss, scratch):
        """loss[0] = mean over valid samples of (y - target)^2; gy = its gradient (zero on tails)."""
        self._check(y, self.sizes[SAMPLES], "y")
        self._check(target, self.sizes[SAMPLES], "target")
        self._check(gy, self.sizes[SAMPLES], "gy")
        self._check(loss, 1, "loss")
        self._check(scratch, self.sizes[SCRATCH], "scratch")
        st = lib().DSPLIB_gpu_raggedMseGrad(self._plan, y.data_ptr(), target.data_ptr(), gy.data_ptr(),
                                           loss.data_ptr(), scratch.data_ptr(), _stream_ptr())
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_raggedMseGrad", st)

    def step_mse_raw(self, x, taps, coefs, target, y, gy, loss, gx, gtaps, gcoefs, work, scratch):
        """Forward + MSE loss + adjoint in one call (DSPLIB_gpu_firBiquadBatched_stepMse)."""
        self._check(target, self.sizes[SAMPLES], "target")
        self._check(y, self.sizes[SAMPLES], "y")
        self._check(gy, self.sizes[SAMPLES], "gy")
        self._check(loss, 1, "loss")
        self._check(gx, self.sizes[SAMPLES], "gx")
        self._check(gtaps, self.sizes[TAPS], "gtaps")
        self._check(gcoefs, self.sizes[COEFS], "gcoefs")
        self._check(work, self.sizes[WORK], "work")
        self._check(scratch, self.sizes[SCRATCH], "scratch")
        st = lib().DSPLIB_gpu_firBiquadBatched_stepMse(
            self._plan, x.data_ptr(), taps.data_ptr(), coefs.data_ptr(), target.data_ptr(), y.data_ptr(),
            gy.data_ptr(), loss.data_ptr(), gx.data_ptr(), gtaps.data_ptr(), gcoefs.data_ptr(), work.data_ptr(),
            scratch.data_ptr(), _stream_ptr())
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_firBiquadBatched_stepMse", st)

    def set_async(self, on: bool):
        """True: step_mse_host returns once queued on the current stream (page-locked
        tensors; synchronise the stream, then check status()); False: it returns complete."""
        return lib().DSPLIB_gpu_raggedPlanSetAsync(self._plan, int(bool(on)))

    def status(self) -> int:
        """DSPLIB_gpu_raggedPlanStatus: nonzero if a bounded tensor-core wait expired."""
        return lib().DSPLIB_gpu_raggedPlanStatus(self._plan)

    def step_mse_host(self, x, taps, coefs, target, y, gy, loss, gx, gtaps, gcoefs):
        """The training step on host tensors (DSPLIB_gpu_firBiquadBatched_stepMseHost):
        inputs copied in and results copied out by the library, channel segments
        pipelined over three streams; returns once the results are in host memory.
        Page-locked tensors let the copies overlap; gy may be None."""
        def check(t, n, name):
            import torch

            if not (t.dtype == torch.float32 and t.is_contiguous() and t.numel() == n):
                raise ValueError(f"{name}: need a contiguous float32 tensor of {n} elements")

        n, nh, nk = self.sizes[SAMPLES], self.sizes[TAPS], self.sizes[COEFS]
        for t, m, name in ((x, n, "x"), (taps, nh, "taps"), (coefs, nk, "coefs"), (target, n, "target"),
                           (y, n, "y"), (loss, 1, "loss"), (gx, n, "gx"), (gtaps, nh, "gtaps"),
                           (gcoefs, nk, "gcoefs")):
            check(t, m, name)
        if gy is not None:
            check(gy, n, "gy")
        st = lib().DSPLIB_gpu_firBiquadBatched_stepMseHost(
            self._plan, x.data_ptr(), taps.data_ptr(), coefs.data_ptr(), target.data_ptr(), y.data_ptr(),
            None if gy is None else gy.data_ptr(), loss.data_ptr(), gx.data_ptr(), gtaps.data_ptr(),
            gcoefs.data_ptr(), _stream_ptr())
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_firBiquadBatched_stepMseHost", st)

    # ---------------------------------------------------------------- autograd
    def apply(self, x, taps, coefs):
        """Differentiable y = filterbank(x; taps, coefs) on packed tensors."""
        return _FirBiquadFn.apply(x, taps, coefs, self)

    def graph_step(self, x, taps, coefs, target):
        """Capture one training step (forward, MSE loss, adjoint: DSPLIB_gpu_firBiquadBatched_stepMse)
        for this plan in a CUDA graph.

        Returns ``(replay, outputs)``: ``replay()`` reruns the captured work on
        the same input tensors (refill them in place between replays);
        ``outputs`` holds the loss, y, gx, gtaps and gcoefs tensors the graph writes."""
        import torch

        dev = x.device
        y = torch.empty(self.sizes[SAMPLES], device=dev)
        work = torch.empty(self.sizes[WORK], device=dev)
        gy = torch.empty(self.sizes[SAMPLES], device=dev)
        gx = torch.empty_like(x)
        gtaps = torch.empty_like(taps)
        gcoefs = torch.empty_like(coefs)
        scratch = torch.empty(self.sizes[SCRATCH], device=dev)
        loss = torch.empty(1, device=dev)

        def body():
            self.step_mse_raw(x, taps, coefs, target, y, gy, loss, gx, gtaps, gcoefs, work, scratch)

        s = torch.cuda.Stream(device=dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(s):
            body()  # warm-up outside capture
        torch.cuda.current_stream(dev).wait_stream(s)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            body()
        outputs = {"loss": loss, "y": y, "gx": gx, "gtaps": gtaps, "gcoefs": gcoefs}
        return g.replay, outputs

    def output_mask(self, device):
        """1 on the valid output samples of every channel, 0 on the T_c - 1 tail samples."""
        import torch

        m = np.zeros(self.sizes[SAMPLES], dtype=np.float32)
        for c in range(self.num_channels):
            m[self.x_off[c]:self.x_off[c] + self.out_lengths[c]] = 1.0
        return torch.from_numpy(m).to(device)


def _autograd_base():
    import torch

    return torch.autograd.Function


class _FirBiquadFn(_autograd_base()):
    @staticmethod
    def forward(ctx, x, taps, coefs, bank):
        import torch

        x, taps, coefs = x.contiguous(), taps.contiguous(), coefs.contiguous()
        y = torch.empty(bank.sizes[SAMPLES], device=x.device, dtype=torch.float32)
        work = torch.empty(bank.sizes[WORK], device=x.device, dtype=torch.float32)
        bank.forward_raw(x, taps, coefs, y, work)
        ctx.save_for_backward(x, taps, coefs, work)
        ctx.bank = bank
        return y

    @staticmethod
    def backward(ctx, gy):
        import torch

        x, taps, coefs, work = ctx.saved_tensors
        bank = ctx.bank
        gy = gy.contiguous()
        gx = torch.empty_like(x)
        gtaps = torch.empty_like(taps)
        gcoefs = torch.empty_like(coefs)
        scratch = torch.empty(bank.sizes[SCRATCH], device=x.device, dtype=torch.float32)
        bank.backward_raw(x, taps, coefs, work, gy, gx, gtaps, gcoefs, scratch)
        return gx, gtaps, gcoefs, None
