#!/usr/bin/env python
"""Benchmark of the DSPLIB filtering hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Default workload (N = 1): the batched, differentiable FIR -> cascaded-biquad
filter bank the metric ("FIR+biquad Gsamples/s") is quoted on: 2048 channels of
lengths log-uniform in [256, 262144] (75.4 M samples), FIR taps uniform in
{32..512}, 2-8 DF2 stages (poles r <= 0.98), one training step = forward, MSE
loss gradient against a fixed target bank's output and the adjoint w.r.t. the
input, the taps and the biquad coefficients, replayed from one CUDA graph.
Other workloads (--workload): the plain DSPLIB_cascadeBiquad configuration
(32 channels x 8192 samples x 4 stages, and its 4096-channel scaled shape),
the FIR configurations (int16 Q15, FP32 plain and split-BF16x3, int8 / int16
tensor-core in Q mode and in the natural-C wrap mode) and the next-row kernels.

One step = one pass of the hot path over the whole batch, inputs resident in
HBM.  L2 is flushed (256 MiB write) between steps, outside the CUDA events that
time each step.  ``value`` = samples processed by all ranks / max-over-ranks
device time.  ``e2e`` = the same metric through the library's public calls with
page-locked host buffers (host->device copies of every input and device->host
copies of every result inside the timed region).  Multi-GPU: one process per
GPU (torchrun), each rank runs its own copy of the workload (no data-path
collective), weak scaling.

``--impl reference`` times the reference's natural-C kernels (compiled from
the reference sources into oracle/_ref) on the host cores with all threads,
on the same workload, and prints the same JSON line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, FALLBACK_BF16_TFLOPS, "fallback"


def profile_traffic(name):
    """dram bytes per launch recorded from an ncu capture in profiles/<name>.md."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch"):
            try:
                return int(float(line.split("=")[1].split()[0]))
            except Exception:
                return None
    return None


# ----------------------------------------------------------- workloads


def biquad_coefficients(rng, rows, S):
    """Natural [rows, S*5] per the default-workload rule (module docstring)."""
    out = np.zeros((rows, S, 5), np.float64)
    for r_ in range(rows):
        for s in range(S):
            r = rng.uniform(0.5, 0.95)
            th = rng.uniform(0, math.pi)
            ph = rng.uniform(0, math.pi)
            b = np.array([1.0, -2 * math.cos(ph), 1.0])
            a = np.array([1.0, -2 * r * math.cos(th), r * r])
            z = np.exp(-1j * th * np.arange(3))
            g = 1.0 / max(abs(np.dot(b, z) / np.dot(a, z)), 1e-12)
            out[r_, s] = [g * b[0], g * b[1], g * b[2], a[1], a[2]]
    return out.reshape(rows, S * 5).astype(np.float32)


def lowpass_taps(rng, rows, T):
    """Hamming-windowed sinc low-pass, cutoff ~ U[0.05, 0.45] of Nyquist, unit DC gain; stored order."""
    n = np.arange(T) - (T - 1) / 2.0
    out = np.zeros((rows, T), np.float32)
    for r_ in range(rows):
        fc = rng.uniform(0.05, 0.45)
        h = fc * np.sinc(fc * n) * np.hamming(T)
        out[r_] = (h / h.sum())[::-1]
    return out


class Workload:
    name = ""
    metric = "Gsamples/s"
    dtype = "f32"
    e2e_in_flight = 1  # independent calls the end-to-end loop keeps in flight

    def bind_stream(self, stream):
        self.h.set_stream(stream)

    def e2e_drain(self):
        """Wait for the calls the end-to-end loop left in flight."""


class BiquadWorkload(Workload):
    def __init__(self, C=32, N=8192, S=4, form=2, seed=2):
        import c7x_dsplib_b200 as D

        self.D = D
        self.C, self.N, self.S, self.form = C, N, S, form
        self.name = f"cascadeBiquad_DF2_{C}ch_x_{N}_x_{S}stages"
        rng = np.random.default_rng(seed)
        self.x = rng.standard_normal((N, C)).astype(np.float32)
        self.nat = biquad_coefficients(rng, 1, S)
        self.opt = None  # the OPT layout comes from the library's get_coefficients (setup_device)
        self.samples = N * C
        nv = 4 if form == 1 else 2
        self.alg_bytes = 4 * (2 * N * C) + 4 * 5 * S + 2 * 4 * (S * nv * C)
        self.bound = "hbm"
        # up to 16 channels: one CTA per channel along time; beyond: lane = channel
        self.kernel = "biquad_chan_kernel" if C <= 16 else "biquad_scan_kernel"

    def config(self):
        return {"workload": self.name, "channels": self.C, "samples_per_channel": self.N, "stages": self.S,
                "form": "DF2", "funcStyle": "OPTIMIZED", "coefficients": "shared"}

    def setup_device(self, torch, func_style=None):
        D = self.D
        fs = D.OPTIMIZED if func_style is None else func_style
        if self.opt is None:
            self.opt, _ = D.opt_coefficients(self.nat, self.form, 0, self.C)
        self.xd = torch.from_numpy(self.x).cuda()
        self.yd = torch.zeros_like(self.xd)
        self.sd = torch.zeros((self.S * 2, self.C), device="cuda")
        self.cd = torch.from_numpy(self.opt if fs == D.OPTIMIZED else self.nat).cuda()
        args, pin, pout, pvar, pcn, popt = D.biquad_descs(self.C, self.N, self.S, self.form, 0, func_style=fs)
        self.h = D.BiquadHandle()
        st = self.h.init(args, pin, popt if fs == D.OPTIMIZED else pcn, pvar, pout)
        assert st == D.SUCCESS, self.h.last_error()
        self.h.set_async(True)

    def step(self):
        st = self.h.exec(self.xd, self.cd, self.sd, self.yd)
        if st != self.D.SUCCESS:
            raise RuntimeError(self.h.last_error())

    def e2e_setup(self, torch):
        D = self.D
        self.hx = torch.from_numpy(self.x).pin_memory()
        self.hy = torch.zeros_like(self.hx).pin_memory()
        self.hs = torch.zeros((self.S * 2, self.C)).pin_memory()
        self.hc = torch.from_numpy(self.opt).pin_memory()
        args, pin, pout, pvar, pcn, popt = D.biquad_descs(self.C, self.N, self.S, self.form, 0)
        self.he = D.BiquadHandle()
        assert self.he.init(args, pin, popt, pvar, pout) == D.SUCCESS
        self.h2d = self.hx.numel() * 4 + self.hc.numel() * 4 + self.hs.numel() * 4
        self.d2h = self.hy.numel() * 4 + self.hs.numel() * 4
        # Independent signals in flight on their own handles and streams with asynchronous
        # completion on page-locked buffers (DSPLIB_gpu_setAsync level 2): one call's PCIe
        # reads overlap another's kernel and writes.  Each call still reads its input and
        # writes its output and state across PCIe; a slot is reused once its call completed.
        # Signals of 4 MB or more go through the library's staged block pipeline, whose calls
        # complete before returning, so they run one at a time.
        self.e2e_in_flight = 3 if (self.C >= 32 and self.x.nbytes < (4 << 20)) else 1
        self.slots = []
        for _ in range(self.e2e_in_flight):
            h, stream = D.BiquadHandle(), torch.cuda.Stream()
            assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
            assert h.set_stream(stream) == D.SUCCESS and h.set_async(2) == D.SUCCESS
            self.slots.append((h, stream, torch.zeros_like(self.hx).pin_memory(),
                               torch.zeros((self.S * 2, self.C)).pin_memory()))
        self.slot_next = 0

    def e2e_step(self):
        h, stream, hy, hs = self.slots[self.slot_next % self.e2e_in_flight]
        if self.slot_next >= self.e2e_in_flight:
            stream.synchronize()  # this slot's previous call is complete
        self.slot_next += 1
        st = h.exec(self.hx, self.hc, hs, hy)
        if st != self.D.SUCCESS:
            raise RuntimeError(h.last_error())

    def e2e_drain(self):
        for _, stream, _, _ in self.slots:
            stream.synchronize()

    def e2e_sync_step(self):
        """One synchronous call (the reference's calling pattern)."""
        st = self.he.exec(self.hx, self.hc, self.hs, self.hy)
        if st != self.D.SUCCESS:
            raise RuntimeError(self.he.last_error())

    def cpu_reference(self, threads, budget_s):
        import oracle

        reps, t_total = 0, 0.0
        while t_total < budget_s or reps < 2:
            st = np.zeros((self.S * 2, self.C), np.float32)
            t0 = time.perf_counter()
            oracle.biquad(self.form, self.x, self.nat, st, nch=0, impl="ref", threads=threads)
            t_total += time.perf_counter() - t0
            reps += 1
        return self.samples * reps / t_total / 1e9, f"{reps} full passes of the workload ({self.C} ch x {self.N})"


class FirWorkload(Workload):
    def __init__(self, name, dtype, B, N, T, *, nch, precision=0, qmode=False, shift=0, seed=3):
        import c7x_dsplib_b200 as D

        self.D = D
        self.name = name
        self.B, self.N, self.T, self.nch, self.precision, self.qmode, self.shift = B, N, T, nch, precision, qmode, shift
        rng = np.random.default_rng(seed)
        self.npdt = dtype
        if dtype == np.float32:
            self.x = rng.standard_normal((B, N)).astype(np.float32)
            self.hh = lowpass_taps(rng, B if nch else 1, T)
            self.dtype = "f32"
        else:
            info = np.iinfo(dtype)
            lo, hi = (-4096, 4095) if (dtype == np.int16 and name.startswith("fir_int16_16ch")) else (info.min,
                                                                                                      info.max)
            self.x = rng.integers(lo, hi, size=(B, N), endpoint=True).astype(dtype)
            self.hh = rng.integers(lo, hi, size=(B if nch else 1, T), endpoint=True).astype(dtype)
            self.dtype = {np.int8: "i8", np.int16: "i16", np.int32: "i32"}[dtype]
        elt = np.dtype(dtype).itemsize
        self.out_size = N - T + 1
        self.samples = B * self.out_size
        self.alg_bytes = elt * (B * N + B * self.out_size + self.hh.size)
        self.alg_flops = 2.0 * T * self.samples
        self.bound = "tensor" if precision == 1 else "hbm"
        if dtype == np.float32:
            self.kernel = "fir_bf16x3_tc_kernel" if precision == 1 else "fir_f32_simt_kernel"
        else:
            self.kernel = "fir_int_tc_kernel" if T <= 2048 else "fir_direct_kernel"

    def config(self):
        return {"workload": self.name, "channels": self.B, "samples_per_channel": self.N, "taps": self.T,
                "coefficients": "per-channel" if self.nch else "shared",
                "precision": ["simt_fp32", "bf16x3"][self.precision] if self.dtype == "f32" else
                ("q_mode shift=%d" % self.shift if self.qmode else "wrap (natural-C)")}

    def setup_device(self, torch, func_style=None):
        D = self.D
        fs = D.OPTIMIZED if func_style is None else func_style
        self.xd = torch.from_numpy(self.x).cuda()
        self.hd = torch.from_numpy(self.hh).cuda()
        self.yd = torch.zeros((self.B, self.out_size), dtype=self.xd.dtype, device="cuda")
        code = {"f32": D.FLOAT32, "i8": D.INT8, "i16": D.INT16, "i32": D.INT32}[self.dtype]
        args, pin, pf, po = D.fir_setup(code, self.B, self.N, self.T, nch=self.nch, func_style=fs, shift=self.shift)
        self.h = D.FirHandle()
        assert self.h.init(args, pin, pf, po) == D.SUCCESS
        self.h.set_precision(self.precision)
        self.h.set_qmode(self.qmode)
        self.h.set_async(True)
        self.args = (args, pin, pf, po)

    def step(self):
        st = self.h.exec(self.xd, self.hd, self.yd)
        if st != self.D.SUCCESS:
            raise RuntimeError(self.h.last_error())

    def e2e_setup(self, torch):
        self.hx = torch.from_numpy(self.x).pin_memory()
        self.hhp = torch.from_numpy(self.hh).pin_memory()
        self.hy = torch.zeros((self.B, self.out_size), dtype=self.hx.dtype).pin_memory()
        self.he = self.D.FirHandle()
        args, pin, pf, po = self.args
        assert self.he.init(args, pin, pf, po) == self.D.SUCCESS
        self.he.set_precision(self.precision)
        self.he.set_qmode(self.qmode)
        elt = np.dtype(self.npdt).itemsize
        self.h2d = (self.x.size + self.hh.size) * elt
        self.d2h = self.samples * elt

    def e2e_step(self):
        st = self.he.exec(self.hx, self.hhp, self.hy)
        if st != self.D.SUCCESS:
            raise RuntimeError(self.he.last_error())

    def cpu_reference(self, threads, budget_s):
        import oracle

        # bounded sample: a channel subset sized to the budget, scaled by samples
        rows = self.B
        per_row_s = None
        reps, t_total, done = 0, 0.0, 0
        sub = min(self.B, max(threads, 1))
        while t_total < budget_s or reps < 1:
            xs = np.ascontiguousarray(self.x[:sub])
            hs = np.ascontiguousarray(self.hh[:sub] if self.nch else self.hh)
            t0 = time.perf_counter()
            oracle.fir(xs, hs, self.T, nch=self.nch, impl="ref", threads=threads)
            dt = time.perf_counter() - t0
            t_total += dt
            done += sub * self.out_size
            reps += 1
            if per_row_s is None:
                per_row_s = dt / sub
                if dt < budget_s / 20 and sub < rows:
                    sub = min(rows, max(sub, int(sub * (budget_s / 10) / max(dt, 1e-6))))
        return done / t_total / 1e9, f"{done // self.out_size} channel passes of {self.N} samples (subset of the " \
                                     f"{self.B}-channel workload)"


def random_sections(rng, S, rmin=0.5, rmax=0.98):
    """S stable sections [b0 b1 b2 a1 a2]: conjugate poles r ~ U[rmin, rmax], angle ~ U[0.05, pi - 0.05],
    zeros r ~ U[0, 1], gain normalised to about 1 at DC."""
    out = np.zeros((S, 5))
    for s in range(S):
        r = rng.uniform(rmin, rmax)
        th = rng.uniform(0.05, math.pi - 0.05)
        a1, a2 = -2 * r * math.cos(th), r * r
        rz, tz = rng.uniform(0, 1), rng.uniform(0, math.pi)
        b = np.array([1.0, -2 * rz * math.cos(tz), rz * rz])
        g = (1 + a1 + a2) / max(abs(b.sum()), 0.2)
        out[s] = [b[0] * g, b[1] * g, b[2] * g, a1, a2]
    return out


class FilterBankWorkload(Workload):
    """Batched uneven FIR -> cascaded-biquad bank, one training step: forward,
    MSE loss against a fixed target filter bank's output, adjoint w.r.t. input,
    taps and coefficients, captured in one CUDA graph.  2048 channels, lengths
    log-uniform in [256, 262144], taps uniform in {32..512} (N(0, 1/taps), at
    most the channel length), 2-8 stages with poles of radius <= 0.98, input N(0, 1).

    Algorithmic work of one step (the roofline's numerator):
      HBM     20 bytes per input sample: x in and y out (forward), target in and the
              output gradient (loss), x and the gradient in and gx out (adjoint), FP32,
              each touched once; activations a design keeps or recomputes are not counted.
      tensor  6 T Lu flops per channel: the FIR forward, its input gradient and its taps
              gradient, 2 T flops per output each.
    The bound is whichever of the two takes longer at the measured peaks."""

    BYTES_PER_SAMPLE = 20

    def __init__(self, C=2048, seed=5):
        import c7x_dsplib_b200 as D

        self.D = D
        rng = np.random.default_rng(seed)
        self.lengths = np.exp(rng.uniform(math.log(256), math.log(262144), C)).astype(np.int64)
        self.taps = np.minimum(rng.integers(32, 512, size=C, endpoint=True), self.lengths)
        self.stages = rng.integers(2, 8, size=C, endpoint=True)
        self.C = C
        self.name = f"fir_biquad_bank_{C}ch_ragged_fwd_bwd"
        self.samples = int(self.lengths.sum())
        self.x = rng.standard_normal(self.samples).astype(np.float32)
        self.h = np.concatenate([rng.standard_normal(T) / math.sqrt(T) for T in self.taps]).astype(np.float32)
        self.c = np.concatenate([random_sections(rng, S).reshape(-1) for S in self.stages]).astype(np.float32)
        self.ht = np.concatenate([rng.standard_normal(T) / math.sqrt(T) for T in self.taps]).astype(np.float32)
        self.ct = np.concatenate([random_sections(rng, S).reshape(-1) for S in self.stages]).astype(np.float32)
        Lu = self.lengths - self.taps + 1
        self.alg_bytes = self.BYTES_PER_SAMPLE * self.samples
        self.alg_flops = float(np.sum(6.0 * self.taps * Lu))
        hbm, bf16, _ = peaks()
        t_hbm, t_tensor = self.alg_bytes / (hbm * 1e9), self.alg_flops / (bf16 * 1e12)
        self.bound = "hbm" if t_hbm >= t_tensor else "tensor"
        self.bound_times_ms = {"hbm": t_hbm * 1e3, "tensor": t_tensor * 1e3}
        self.issued_flops = self._issued_tensor_flops()
        self.kernel = "fir_biquad_bank_step"
        self.launches_per_step = None

    def _issued_tensor_flops(self):
        """Tensor-core flops the split-BF16 kernels issue per step (Toeplitz inflation and
        the hi/lo products included): 8 * K flops per output, K = round16(T + 63), for the
        forward (Lu outputs), the input gradient (L outputs) and the taps gradient."""
        K = ((self.taps + 63 + 15) // 16) * 16
        Lu = self.lengths - self.taps + 1
        return float(np.sum(8.0 * K * (Lu + self.lengths + Lu)))

    def config(self):
        return {"workload": self.name, "channels": self.C, "total_samples": self.samples,
                "lengths": "log-uniform [256, 262144]", "taps": "uniform {32..512}", "stages": "uniform {2..8}",
                "pole_radius": "U[0.5, 0.98]", "loss": "MSE vs fixed target bank output",
                "graph": "one fused training-step call (forward + loss + adjoint) in one CUDA graph"}

    def bind_stream(self, stream):
        pass

    def setup_device(self, torch, func_style=None):
        from c7x_dsplib_b200.filterbank import RaggedFilterBank

        self.bank = RaggedFilterBank(self.lengths, self.taps, self.stages)
        dev = "cuda"
        self.xd = torch.from_numpy(self.x).to(dev)
        self.hd = torch.from_numpy(self.h).to(dev)
        self.cd = torch.from_numpy(self.c).to(dev)
        self.target = self.bank.apply(self.xd, torch.from_numpy(self.ht).to(dev),
                                      torch.from_numpy(self.ct).to(dev)).detach()
        torch.cuda.synchronize()
        n0 = self.D.kernel_launch_count()
        self.replay, self.out = self.bank.graph_step(self.xd, self.hd, self.cd, self.target)
        # graph_step runs the body once eagerly, then once under capture
        self.launches_per_step = (self.D.kernel_launch_count() - n0) // 2

    def step(self):
        self.replay()

    def phase_times(self, torch, reps=3):
        """Event-timed C-ABI calls, run eagerly: forward, loss and adjoint as separate calls, and the
        fused step the timed graph replays; median ms each."""
        b, dev = self.bank, "cuda"
        y = torch.empty(b.sizes[0], device=dev)
        work = torch.empty(b.sizes[3], device=dev)
        gy = torch.empty_like(y)
        gx, gh, gc = torch.empty_like(self.xd), torch.empty_like(self.hd), torch.empty_like(self.cd)
        scratch = torch.empty(b.sizes[4], device=dev)
        loss = torch.empty(1, device=dev)
        calls = {"forward": lambda: b.forward_raw(self.xd, self.hd, self.cd, y, work),
                 "loss": lambda: b.mse_grad_raw(y, self.target, gy, loss, scratch),
                 "adjoint": lambda: b.backward_raw(self.xd, self.hd, self.cd, work, gy, gx, gh, gc, scratch),
                 "fused_step": lambda: b.step_mse_raw(self.xd, self.hd, self.cd, self.target, y, gy, loss, gx, gh,
                                                      gc, work, scratch)}
        times = {k: [] for k in calls}
        s = torch.cuda.current_stream()
        for _ in range(reps):
            for k, f in calls.items():
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                f()
                e1.record(s)
                torch.cuda.synchronize()
                times[k].append(e0.elapsed_time(e1))
        return {k: statistics.median(v) for k, v in times.items()}

    def e2e_setup(self, torch):
        # every input of the step from page-locked host memory, every result back, through
        # the library's host-buffer step (channel segments pipelined over three streams);
        # two independent calls in flight (two plans of the bank, DSPLIB_gpu_raggedPlanSetAsync),
        # so that one call's copies out overlap the next one's copies in
        from c7x_dsplib_b200.filterbank import RaggedFilterBank

        self.hx = torch.from_numpy(self.x).pin_memory()
        self.htg = self.target.cpu().pin_memory()
        self.hh = torch.from_numpy(self.h).pin_memory()
        self.hc = torch.from_numpy(self.c).pin_memory()
        self.h_out = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in self.out.items()}
        self.h2d = 4 * (self.hx.numel() + self.htg.numel() + self.hh.numel() + self.hc.numel())
        self.d2h = sum(4 * t.numel() for t in self.h_out.values())
        self.e2e_in_flight = 2
        self.slots = []
        for _ in range(self.e2e_in_flight):
            bank = RaggedFilterBank(self.lengths, self.taps, self.stages)
            bank.set_async(True)
            outs = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in self.out.items()}
            self.slots.append((bank, torch.cuda.Stream(), outs))
        self.slot_next = 0

    def _host_step(self, bank, o):
        bank.step_mse_host(self.hx, self.hh, self.hc, self.htg, o["y"], None, o["loss"], o["gx"], o["gtaps"],
                           o["gcoefs"])

    def e2e_step(self):
        import torch

        bank, st, o = self.slots[self.slot_next % self.e2e_in_flight]
        self.slot_next += 1
        st.synchronize()  # this slot's previous call has finished: its buffers may be reused
        with torch.cuda.stream(st):
            self._host_step(bank, o)

    def e2e_drain(self):
        for bank, st, _ in self.slots:
            st.synchronize()
            if bank.status() != 0:
                raise RuntimeError("a bounded tensor-core wait expired in an end-to-end step")

    def e2e_sync_step(self):
        """The same step one synchronous call at a time."""
        self._host_step(self.bank, self.h_out)

    def e2e_check(self, torch):
        """The host-buffer steps' results equal the device step's (bitwise; the loss to
        its summation order)."""
        self.replay()
        torch.cuda.synchronize()
        for outs in [self.h_out] + [o for _, _, o in self.slots]:
            for k, t in outs.items():
                d = self.out[k].cpu()
                ok = torch.allclose(t, d, rtol=1e-6, atol=0) if k == "loss" else torch.equal(t, d)
                if not ok:
                    raise RuntimeError(f"end-to-end result {k} differs from the device step")

    def cpu_reference(self, threads, budget_s):
        from oracle.filterbank import bank_step_sample

        n_total = int((self.lengths - self.taps + 1).sum())
        order = np.random.default_rng(0).permutation(self.C)
        t_total, done, i = 0.0, 0, 0
        tgt = getattr(self, "_target_host", None)
        if tgt is None:
            tgt = np.zeros(self.samples, np.float32)
        while (t_total < budget_s or done == 0) and i < self.C:
            chunk = order[i:i + max(threads, 1)]
            dt, n = bank_step_sample(self.lengths, self.taps, self.stages, self.x, self.h, self.c, tgt, chunk,
                                     threads, n_total)
            t_total += dt
            done += n
            i += len(chunk)
        return done / t_total / 1e9, f"{i} of {self.C} channels (random order), {done} samples, forward + loss + " \
                                     f"adjoint composed of the reference's FIR and biquad natural-C kernels"


def stream_name(kind, n, channels, inputs):
    return {"fltoq15": f"fltoq15_f32_{n >> 20}M", "q15tofl": f"q15tofl_f32_{n >> 20}M",
            "interleave": f"interleave_{channels}ch_f32_{n >> 20}M",
            "deinterleave": f"deinterleave_{channels}ch_f32_{n >> 20}M",
            "addnch": f"addNCh_f32_{inputs}in_{channels}ch_{n >> 20}M"}[kind]


def _ref_chunks(fn, n, threads):
    """Run fn(lo, hi) over [0, n) split into `threads` contiguous ranges on host threads
    (ctypes releases the GIL during the foreign call, so the ranges run in parallel)."""
    from concurrent.futures import ThreadPoolExecutor

    threads = max(1, min(threads, n))
    bounds = [(n * k // threads, n * (k + 1) // threads) for k in range(threads)]
    if threads == 1:
        fn(0, n)
        return
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda b: fn(*b), bounds))


class StreamWorkload(Workload):
    """The Q.15 conversions and layout kernels next to the filters (DSPLIB_fltoq15,
    DSPLIB_q15tofl, DSPLIB_interleave, DSPLIB_deinterleave, DSPLIB_addNCh): one exec over
    arrays far larger than L2 per step, metric = elements (output samples) per second."""

    bound = "hbm"
    metric = "Gsamples/s"

    def __init__(self, kind, n, *, channels=2, inputs=12, seed=6):
        import c7x_dsplib_b200 as D

        self.D, self.kind, self.n = D, kind, n
        rng = np.random.default_rng(seed)
        self.C, self.L = channels, inputs
        if kind == "fltoq15":
            self.x = rng.uniform(-1, 1, n).astype(np.float32)
            self.out_dtype, self.samples, self.alg_bytes = np.int16, n, 6 * n
            self.kernel, self.dtype = "fltoq15_vec_kernel", "f32"
        elif kind == "q15tofl":
            self.x = rng.integers(-32768, 32767, n, endpoint=True).astype(np.int16)
            self.out_dtype, self.samples, self.alg_bytes = np.float32, n, 6 * n
            self.kernel, self.dtype = "q15tofl_vec_kernel", "i16"
        elif kind in ("interleave", "deinterleave"):
            # interleave: C channel rows of n samples -> n rows of C; deinterleave the reverse
            self.x = rng.standard_normal(n * channels).astype(np.float32)
            self.out_dtype, self.samples, self.alg_bytes = np.float32, n * channels, 8 * n * channels
            self.W, self.H = (n, channels) if kind == "interleave" else (channels, n)
            self.kernel, self.dtype = ("interleave_k_kernel" if kind == "interleave" else "deinterleave_k_kernel"), "f32"
        else:  # addNCh: `inputs` stacked inputs of `channels` rows of n samples
            self.x = rng.uniform(-10, 10, n * channels * inputs).astype(np.float32)
            self.out_dtype, self.samples = np.float32, n * channels
            self.alg_bytes = 4 * n * channels * (inputs + 1)
            self.kernel, self.dtype = "addnch_kernel", "f32"
        self.name = stream_name(kind, n, channels, inputs)

    def config(self):
        c = {"workload": self.name, "elements_out": self.samples, "funcStyle": "OPTIMIZED"}
        if self.kind in ("interleave", "deinterleave", "addnch"):
            c["channels"] = self.C
        if self.kind == "addnch":
            c["inputs"] = self.L
        return c

    def _call(self, x, y, h):
        D = self.D
        if self.kind == "fltoq15":
            D.fltoq15(x, out=y, handle=h)
        elif self.kind == "q15tofl":
            D.q15tofl(x, np.float32, out=y, handle=h)
        elif self.kind in ("interleave", "deinterleave"):
            D.transpose(x, y, self.W, self.H, self.W * 4, self.H * 4, kind=self.kind, handle=h)
        else:
            D.add_nch(x, y, self.n, self.C, self.L, self.n, self.n * self.C, self.n, handle=h)

    def _handle(self):
        D = self.D
        if self.kind == "fltoq15":
            return D.Fltoq15Handle()
        if self.kind == "q15tofl":
            return D.Q15toflHandle()
        return D.LayoutHandle({"interleave": "DSPLIB_interleave", "deinterleave": "DSPLIB_deinterleave",
                               "addnch": "DSPLIB_addNCh"}[self.kind])

    def setup_device(self, torch, func_style=None):
        self.h = self._handle()
        self.xd = torch.from_numpy(self.x).cuda()
        self.yd = torch.zeros(self.samples, dtype=getattr(torch, np.dtype(self.out_dtype).name), device="cuda")
        self.h.set_async(True)
        self._call(self.xd, self.yd, self.h)

    def step(self):
        self._call(self.xd, self.yd, self.h)

    def e2e_setup(self, torch):
        self.hx = torch.from_numpy(self.x).pin_memory()
        self.hy = torch.zeros(self.samples, dtype=self.yd.dtype).pin_memory()
        self.h2d = self.x.nbytes
        self.d2h = self.samples * np.dtype(self.out_dtype).itemsize
        self.he = self._handle()

    def e2e_step(self):
        self._call(self.hx, self.hy, self.he)

    def cpu_reference(self, threads, budget_s):
        import ctypes

        import oracle

        R = oracle.ref()
        m = min(self.n, 1 << 22)  # bounded sample: the first 4 Mi samples per channel
        y = np.zeros(self.samples, self.out_dtype)
        vp = ctypes.c_void_p
        e = self.x.itemsize
        if self.kind == "fltoq15":
            fn = lambda lo, hi: R.ref_fltoq15_cn(12, vp(self.x.ctypes.data + lo * 4), vp(y.ctypes.data + lo * 2),
                                                 hi - lo)
            units, per = m, 1
        elif self.kind == "q15tofl":
            fn = lambda lo, hi: R.ref_q15tofl_cn(12, vp(self.x.ctypes.data + lo * 2), vp(y.ctypes.data + lo * 4),
                                                 hi - lo)
            units, per = m, 1
        elif self.kind == "interleave":  # column ranges of the C x n matrix
            fn = lambda lo, hi: R.ref_transpose_cn(12, vp(self.x.ctypes.data + lo * e), vp(y.ctypes.data + lo * e * self.C),
                                                   hi - lo, self.C, self.n * e, self.C * e)
            units, per = m, self.C
        elif self.kind == "deinterleave":  # row ranges of the n x C matrix
            fn = lambda lo, hi: R.ref_transpose_cn(12, vp(self.x.ctypes.data + lo * e * self.C), vp(y.ctypes.data + lo * e),
                                                   self.C, hi - lo, self.C * e, self.n * e)
            units, per = m, self.C
        else:  # addNCh: one channel row per task
            fn = lambda lo, hi: R.ref_addnch_cn(12, vp(self.x.ctypes.data + lo * self.n * e), vp(y.ctypes.data + lo * self.n * e),
                                                m, hi - lo, self.L, self.n, self.n * self.C, self.n)
            units, per = self.C, m
        reps, t_total = 0, 0.0
        while t_total < budget_s or reps < 1:
            t0 = time.perf_counter()
            _ref_chunks(fn, units, threads)
            t_total += time.perf_counter() - t0
            reps += 1
        done = reps * units * per
        return done / t_total / 1e9, f"{reps} passes over the first {m} samples per channel (of {self.n})"


WORKLOADS = {
    "fir_biquad_bank_2048ch_ragged": lambda: FilterBankWorkload(),
    "fir_biquad_bank_256ch_ragged": lambda: FilterBankWorkload(C=256),
    "biquad_32x8192x4": lambda: BiquadWorkload(),
    "biquad_4096x8192x4": lambda: BiquadWorkload(C=4096),
    "fir_int16_16ch_4096_64taps": lambda: FirWorkload("fir_int16_16ch_4096_64taps", np.int16, 16, 4096, 64, nch=0,
                                                      qmode=True, shift=15, seed=1),
    "fir_f32_1024ch_65536_256taps_simt": lambda: FirWorkload("fir_f32_1024ch_65536_256taps_simt", np.float32, 1024,
                                                             65536, 256, nch=1, precision=0),
    "fir_f32_1024ch_65536_256taps_bf16x3": lambda: FirWorkload("fir_f32_1024ch_65536_256taps_bf16x3", np.float32,
                                                               1024, 65536, 256, nch=1, precision=1),
    "fir_int8_4096ch_16384_128taps": lambda: FirWorkload("fir_int8_4096ch_16384_128taps", np.int8, 4096, 16384, 128,
                                                         nch=0, qmode=True, shift=7, seed=4),
    "fir_int16_4096ch_16384_128taps": lambda: FirWorkload("fir_int16_4096ch_16384_128taps", np.int16, 4096, 16384,
                                                          128, nch=0, qmode=True, shift=15, seed=4),
    # the natural-C wrap mode (modulo 2^bits, bit-exact to the reference _cn kernel)
    "fir_int8_4096ch_16384_128taps_wrap": lambda: FirWorkload("fir_int8_4096ch_16384_128taps_wrap", np.int8, 4096,
                                                              16384, 128, nch=0, qmode=False, seed=4),
    "fir_int16_4096ch_16384_128taps_wrap": lambda: FirWorkload("fir_int16_4096ch_16384_128taps_wrap", np.int16,
                                                               4096, 16384, 128, nch=0, qmode=False, seed=4),
    "fir_int16_16ch_4096_64taps_wrap": lambda: FirWorkload("fir_int16_16ch_4096_64taps_wrap", np.int16, 16, 4096,
                                                           64, nch=0, qmode=False, seed=1),
}
for _k, _n, _c in (("fltoq15", 64 << 20, 2), ("q15tofl", 64 << 20, 2), ("interleave", 16 << 20, 2),
                   ("deinterleave", 16 << 20, 2), ("addnch", 1 << 20, 16)):
    WORKLOADS[stream_name(_k, _n, _c, 12)] = (lambda k=_k, n=_n, c=_c: StreamWorkload(k, n, channels=c))
DEFAULT = "fir_biquad_bank_2048ch_ragged"
TUNE_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c7x_dsplib_b200", "tune_b200.json")


# ----------------------------------------------------------- clocks


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ----------------------------------------------------------- main


def best_threads(wl):
    """All host threads, unless thread start-up outweighs the work (tiny workloads): then one."""
    n = os.cpu_count() or 1
    if n == 1:
        return 1
    v1, _ = wl.cpu_reference(1, budget_s=0.2)
    vn, _ = wl.cpu_reference(n, budget_s=0.2)
    return n if vn >= v1 else 1


def run_reference(a, wl):
    threads = best_threads(wl)
    try:
        import oracle

        if not oracle.ref_available():
            print(json.dumps({"impl": "reference", "unavailable": "reference natural-C library oracle/_ref not built"}))
            return
        value, sample = wl.cpu_reference(threads, budget_s=2.0)
        # K timed steps of the same bounded sample, after W warm-up steps
        for _ in range(a.warmup):
            wl.cpu_reference(threads, budget_s=0.0)
        vals = []
        t0 = time.perf_counter()
        per_step = min(0.05, 60.0 / max(a.steps, 1))
        for _ in range(a.steps):
            v, _ = wl.cpu_reference(threads, budget_s=per_step)
            vals.append(v)
            if time.perf_counter() - t0 > 120.0:  # keep the arm within a few minutes
                break
        elapsed = time.perf_counter() - t0
        value = statistics.median(vals)
    except Exception as e:  # the reference arm must always print its line
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {e}"}))
        return
    line = {"metric": f"{wl.name} {wl.metric}", "value": value, "unit": wl.metric, "n_gpus": a.gpus,
            "steps": len(vals), "warmup": a.warmup, "ms_per_step": elapsed * 1e3 / max(len(vals), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype,
            "data": "synthetic (seeded)", "config": wl.config(), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": wl.metric, "cores": threads, "kind": "reference",
                             "sample": sample + "; reference _cn compiled from the reference sources, channels split "
                                                "over std::threads"},
            "e2e": {"value": value, "unit": wl.metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner cache file (default: $DSPLIB_GPU_TUNE_CACHE, else the package's tune_b200.json)")
    ap.add_argument("--autotune", action="store_true",
                    help="measure launch shapes missing from the cache at set-up and save them to it")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank == 0:
            run_reference(a, WORKLOADS[a.workload]())
        return

    import torch

    import c7x_dsplib_b200 as D

    torch.cuda.set_device(local)
    # launch shapes measured on this GPU model by the library's autotuner (CACHED mode:
    # problem classes without an entry keep the built-in rules)
    tune = a.tune_cache or os.environ.get("DSPLIB_GPU_TUNE_CACHE") or TUNE_CACHE
    shapes = "built-in rules"
    if tune and (os.path.exists(tune) or a.autotune):
        D.lib().DSPLIB_gpu_autotuneSetCachePath(tune.encode())
        shapes = f"autotuner cache {os.path.basename(tune)}" + (" (measured in this run where missing)" if a.autotune
                                                                 else "")
    if a.autotune:
        D.lib().DSPLIB_gpu_autotuneSetMode(2)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = WORKLOADS[a.workload]()
    wl.setup_device(torch)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    wl.bind_stream(stream)

    for _ in range(a.warmup):
        wl.step()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = D.kernel_launch_count()
    for i in range(a.steps):
        flush.zero_()
        starts[i].record(stream)
        wl.step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    launches = D.kernel_launch_count() - n0
    if getattr(wl, "launches_per_step", None):  # CUDA-graph replays bypass the library's launch counter
        launches = wl.launches_per_step * a.steps
    if dist:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / a.steps
    value = wl.samples * world / (ms_per_step * 1e-3) / 1e9

    hbm, bf16, peak_kind = peaks()
    kernel_ms = statistics.median(step_ms)
    if wl.bound == "hbm":
        achieved = wl.alg_bytes / (kernel_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6650 GB/s", "algorithmic_bytes_per_launch": wl.alg_bytes}
    else:
        achieved = wl.alg_flops / (kernel_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                "peak_source": f"{peak_kind} bf16_tflops", "algorithmic_flops_per_launch": wl.alg_flops}
    traffic = profile_traffic(f"{wl.kernel}_{wl.name}")
    roof["traffic"] = traffic
    roof["kernel"] = wl.kernel
    roof["median_launch_ms"] = kernel_ms
    if isinstance(wl, FilterBankWorkload):
        # a step is one graph of several kernels: both floors, the issued tensor work, and
        # the event-timed C-ABI calls of an eager step (outside the timed region)
        roof["algorithmic_bytes_per_launch"] = wl.alg_bytes
        roof["algorithmic_flops_per_launch"] = wl.alg_flops
        roof["floor_ms"] = {"hbm": wl.alg_bytes / (hbm * 1e9) * 1e3, "tensor": wl.alg_flops / (bf16 * 1e12) * 1e3}
        roof["issued_tensor_flops_per_step"] = wl.issued_flops
        roof["issued_tensor_tflops"] = wl.issued_flops / (kernel_ms * 1e-3) / 1e12
        roof["kernel"] = f"{wl.kernel} ({wl.launches_per_step} launches in one CUDA graph)"
        roof["phases_ms"] = wl.phase_times(torch)

    # end to end through the C ABI with pinned host buffers
    wl.e2e_setup(torch)

    def e2e_time(step, drain):
        for _ in range(3):
            step()
        drain()
        n = max(10, min(a.steps, 200))
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(n):
            step()
        drain()
        s = (time.perf_counter() - t0) / n
        if dist:
            t = torch.tensor([s], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            s = float(t.item())
        return s

    e2e_s = e2e_time(wl.e2e_step, wl.e2e_drain)
    e2e = {"value": wl.samples * world / e2e_s / 1e9, "unit": wl.metric, "h2d_bytes_per_step": wl.h2d,
           "d2h_bytes_per_step": wl.d2h, "ms_per_step": e2e_s * 1e3, "in_flight": wl.e2e_in_flight}
    if hasattr(wl, "e2e_sync_step"):
        sync_s = e2e_time(wl.e2e_sync_step, lambda: None)
        e2e["sync_value"] = wl.samples * world / sync_s / 1e9
        e2e["sync_ms_per_step"] = sync_s * 1e3
    if hasattr(wl, "e2e_check"):
        wl.e2e_check(torch)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            import oracle

            if oracle.ref_available():
                threads = best_threads(wl)
                v, sample = wl.cpu_reference(threads, budget_s=3.0)
                cpu = {"value": v, "unit": wl.metric, "cores": threads, "kind": "reference",
                       "sample": sample + "; reference _cn compiled from the reference sources"}
        except Exception as e:
            cpu = {"value": None, "unit": wl.metric, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": f"{wl.name} {wl.metric}", "value": value, "unit": wl.metric, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic (seeded)",
                "config": dict(wl.config(), l2="flushed between steps (256 MiB write outside the timed events)",
                               parallelism=f"channel blocks x{world}, no collective", launch_shapes=shapes),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
