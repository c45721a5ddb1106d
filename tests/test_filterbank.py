"""Batched ragged FIR -> cascaded-biquad filter bank (forward + adjoint).

CPU: the FP64 restatement's adjoint against central finite differences (pins
the reference the GPU path is compared with), and the plan entry points'
export.  GPU: the C-ABI forward/backward against the FP64 restatement, bitwise
repeatability, autograd, and CUDA-graph replay."""
import numpy as np
import pytest

from filterbank_ref import bank_adjoint, bank_forward, channel_adjoint, channel_forward, stable_sections


def _loss(x, h, c, w):
    y, _ = channel_forward(x, h, c)
    return float(w @ y)


@pytest.mark.parametrize("L,T,S", [(40, 5, 2), (17, 1, 3), (9, 9, 1), (30, 4, 0)])
def test_fp64_adjoint_matches_finite_differences(L, T, S):
    rng = np.random.default_rng(L * 100 + T * 10 + S)
    x = rng.standard_normal(L)
    h = rng.standard_normal(T)
    c = stable_sections(rng, S).reshape(-1)
    w = rng.standard_normal(L - T + 1)
    gx, gh, gc = channel_adjoint(x, h, c, w)
    eps = 1e-6
    for vec, grad in ((x, gx), (h, gh), (c, gc.reshape(-1))):
        fd = np.zeros_like(vec)
        for i in range(len(vec)):
            vp = vec.copy()
            vm = vec.copy()
            vp[i] += eps
            vm[i] -= eps
            args_p = [vp if vec is a else a for a in (x, h, c)]
            args_m = [vm if vec is a else a for a in (x, h, c)]
            fd[i] = (_loss(*args_p, w) - _loss(*args_m, w)) / (2 * eps)
        np.testing.assert_allclose(grad, fd, rtol=1e-6, atol=1e-7)


def test_reference_composed_step_matches_fp64():
    """The CPU baseline step built from the reference's natural-C kernels computes the same gradients."""
    import oracle
    from oracle.filterbank import channel_step

    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(11)
    L, T, S = 3000, 37, 3
    x = rng.standard_normal(L).astype(np.float32)
    h = (rng.standard_normal(T) / np.sqrt(T)).astype(np.float32)
    c = stable_sections(rng, S).astype(np.float32)
    target = rng.standard_normal(L - T + 1).astype(np.float32)
    n = L - T + 1
    loss, gx, gh, gc = channel_step(x, h, c, target, n)
    y64, _ = channel_forward(x, h, c)
    gy64 = 2.0 * (y64 - target) / n
    gx64, gh64, gc64 = channel_adjoint(x, h, c, gy64)
    assert loss == pytest.approx(float((y64 - target) @ (y64 - target)) / n, rel=1e-5)
    for got, want in ((gx, gx64), (gh, gh64), (gc, gc64)):
        assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()


def test_plan_symbols_exported():
    from c7x_dsplib_b200 import lib

    L = lib()
    for n in ("DSPLIB_gpu_raggedPlanCreate", "DSPLIB_gpu_raggedPlanSize", "DSPLIB_gpu_raggedPlanDestroy",
              "DSPLIB_gpu_firBiquadBatched_fwd", "DSPLIB_gpu_firBiquadBatched_bwd"):
        assert hasattr(L, n)


# ---------------------------------------------------------------------------------- GPU


def _bank_case(seed, C, Lrange=(64, 20000), Tmax=64, Smax=6, force=()):
    rng = np.random.default_rng(seed)
    lengths, taps, stages = [], [], []
    for _ in range(C):
        T = int(rng.integers(1, Tmax + 1))
        L = int(rng.integers(max(T, Lrange[0]), Lrange[1] + 1))
        lengths.append(L)
        taps.append(T)
        stages.append(int(rng.integers(0, Smax + 1)))
    for L, T, S in force:
        lengths.append(L)
        taps.append(T)
        stages.append(S)
    x = rng.standard_normal(sum(lengths))
    h = np.concatenate([rng.standard_normal(T) / np.sqrt(T) for T in taps])
    c = np.concatenate([stable_sections(rng, S).reshape(-1) for S in stages] + [np.zeros(0)])
    return lengths, taps, stages, x, h, c


def _per_channel_err(lengths, offsets_len, got, want):
    """max |got - want| / max(|want|) per channel segment."""
    worst = 0.0
    o = 0
    for n in offsets_len:
        if n:
            peak = max(np.abs(want[o:o + n]).max(), 1e-30)
            worst = max(worst, np.abs(got[o:o + n] - want[o:o + n]).max() / peak)
        o += n
    return worst


# Tolerance (FP32 kernels against the FP64 restatement, max error relative to
# each channel's peak magnitude, for y, gx, gtaps and gcoefs): 1e-4.
Y_TOL = 1e-4
G_TOL = 1e-4


def _run_bank(lengths, taps, stages, x, h, c, gy):
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    bank = RaggedFilterBank(lengths, taps, stages)
    dev = "cuda"
    xt = torch.tensor(x, dtype=torch.float32, device=dev)
    ht = torch.tensor(h, dtype=torch.float32, device=dev)
    ct = torch.tensor(c, dtype=torch.float32, device=dev)
    gyt = torch.tensor(gy, dtype=torch.float32, device=dev)
    y = torch.empty(bank.sizes[0], device=dev)
    work = torch.empty(bank.sizes[3], device=dev)
    bank.forward_raw(xt, ht, ct, y, work)
    gx, gh, gc = torch.empty_like(xt), torch.empty_like(ht), torch.empty_like(ct)
    scratch = torch.empty(bank.sizes[4], device=dev)
    bank.backward_raw(xt, ht, ct, work, gyt, gx, gh, gc, scratch)
    torch.cuda.synchronize()
    return bank, [t.cpu().numpy().astype(np.float64) for t in (y, gx, gh, gc)]


def _check_bank(lengths, taps, stages, x, h, c, seed=0):
    rng = np.random.default_rng(seed + 99)
    # inputs as the GPU sees them (FP32-rounded), reference in FP64
    x = x.astype(np.float32).astype(np.float64)
    h = h.astype(np.float32).astype(np.float64)
    c = c.astype(np.float32).astype(np.float64)
    gy = rng.standard_normal(len(x)).astype(np.float32).astype(np.float64)
    out_len = [L - T + 1 for L, T in zip(lengths, taps)]
    gy_masked = gy.copy()
    o = 0
    for L, n in zip(lengths, out_len):
        gy_masked[o + n:o + L] = 0.0
        o += L
    bank, (y, gx, gh, gc) = _run_bank(lengths, taps, stages, x, h, c, gy)
    y64 = bank_forward(lengths, taps, stages, x, h, c)
    gx64, gh64, gc64 = bank_adjoint(lengths, taps, stages, x, h, c, gy_masked)
    # tail samples of y are zero
    o = 0
    for L, n in zip(lengths, out_len):
        assert np.all(y[o + n:o + L] == 0.0)
        o += L
    ey = _per_channel_err(lengths, lengths, y, y64)
    egx = _per_channel_err(lengths, lengths, gx, gx64)
    egh = _per_channel_err(lengths, taps, gh, gh64)
    egc = _per_channel_err(lengths, [5 * s for s in stages], gc, gc64)
    assert ey <= Y_TOL, ey
    assert egx <= G_TOL, egx
    assert egh <= G_TOL, egh
    assert egc <= G_TOL, egc
    return bank


@pytest.mark.gpu
def test_bank_small_mixed():
    _check_bank(*_bank_case(1, 12, Lrange=(16, 3000), Tmax=32, Smax=4,
                            force=[(1, 1, 2), (5, 5, 0), (7, 1, 0), (33, 32, 3), (200, 7, 1)]))


@pytest.mark.gpu
def test_bank_multi_window_long_channels():
    # channels longer than one 8192-sample scan window, deep cascades
    _check_bank(*_bank_case(2, 6, Lrange=(8000, 70000), Tmax=128, Smax=10,
                            force=[(8192 + 63, 64, 8), (16384, 1, 12), (8193, 2, 1)]))


@pytest.mark.gpu
def test_bank_long_taps():
    _check_bank(*_bank_case(3, 5, Lrange=(600, 5000), Tmax=512, Smax=3, force=[(512, 512, 2), (2600, 300, 1)]))


@pytest.mark.gpu
def test_bank_many_channels():
    _check_bank(*_bank_case(4, 300, Lrange=(256, 4000), Tmax=64, Smax=6))


@pytest.mark.gpu
def test_backward_bitwise_repeatable():
    import torch

    lengths, taps, stages, x, h, c = _bank_case(5, 20, Lrange=(100, 9000), Tmax=48, Smax=5)
    gy = np.random.default_rng(7).standard_normal(len(x))
    _, a = _run_bank(lengths, taps, stages, x, h, c, gy)
    _, b = _run_bank(lengths, taps, stages, x, h, c, gy)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    del torch


@pytest.mark.gpu
def test_autograd_and_graph_replay():
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages, x, h, c = _bank_case(6, 16, Lrange=(100, 12000), Tmax=40, Smax=4)
    bank = RaggedFilterBank(lengths, taps, stages)
    dev = "cuda"
    xt = torch.tensor(x, dtype=torch.float32, device=dev, requires_grad=True)
    ht = torch.tensor(h, dtype=torch.float32, device=dev, requires_grad=True)
    ct = torch.tensor(c, dtype=torch.float32, device=dev, requires_grad=True)
    target = torch.randn(bank.sizes[0], device=dev)
    mask = bank.output_mask(dev)
    n = mask.sum()
    y = bank.apply(xt, ht, ct)
    loss = (((y - target) * mask) ** 2).sum() / n
    loss.backward()
    # same step captured in a CUDA graph
    xs, hs, cs = xt.detach().clone(), ht.detach().clone(), ct.detach().clone()
    replay, out = bank.graph_step(xs, hs, cs, target)
    replay()
    torch.cuda.synchronize()
    assert torch.allclose(out["loss"], loss.detach(), rtol=1e-5, atol=0)
    assert torch.allclose(out["gx"], xt.grad, rtol=1e-5, atol=1e-9)
    assert torch.allclose(out["gtaps"], ht.grad, rtol=1e-5, atol=1e-9)
    assert torch.allclose(out["gcoefs"], ct.grad, rtol=1e-5, atol=1e-9)
    # replay after refilling the inputs in place follows the new values
    xs.mul_(0.5)
    replay()
    torch.cuda.synchronize()
    y2 = bank.apply(xs, hs, cs).detach()
    assert torch.allclose(out["y"], y2, rtol=0, atol=0)


@pytest.mark.gpu
def test_mse_grad():
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages = [5000, 64, 3000, 9000], [16, 64, 1, 200], [1, 0, 2, 3]
    bank = RaggedFilterBank(lengths, taps, stages)
    rng = np.random.default_rng(12)
    y = rng.standard_normal(bank.sizes[0]).astype(np.float32)
    t = rng.standard_normal(bank.sizes[0]).astype(np.float32)
    yd, td = torch.from_numpy(y).cuda(), torch.from_numpy(t).cuda()
    gy = torch.full_like(yd, 7.0)
    loss = torch.empty(1, device="cuda")
    scratch = torch.empty(bank.sizes[4], device="cuda")
    bank.mse_grad_raw(yd, td, gy, loss, scratch)
    torch.cuda.synchronize()
    mask = bank.output_mask("cpu").numpy() > 0
    n = int(mask.sum())
    assert n == bank.sizes[5]
    d = (y - t).astype(np.float32)
    want_gy = np.where(mask, np.float32(2.0 / n) * d, np.float32(0.0))
    assert np.array_equal(gy.cpu().numpy(), want_gy)
    want = float(np.sum(d[mask].astype(np.float64) ** 2) / n)
    assert float(loss.item()) == pytest.approx(want, rel=1e-6)


# ------------------------------------------------------------------ poles near the unit circle


def _fp32_channel_step(x, h, c, gy):
    """The same step in sequential FP32 (numpy / scipy single-precision recursions): the
    error an FP32 implementation of this filter makes anyway, the yardstick for the
    bound below."""
    from scipy.signal import lfilter

    f = np.float32
    u = np.convolve(x.astype(f), h.astype(f), "valid").astype(f)
    coefs = np.asarray(c, f).reshape(-1, 5)
    acts = [u]
    for b0, b1, b2, a1, a2 in coefs:
        acts.append(lfilter(np.array([b0, b1, b2], f), np.array([1, a1, a2], f), acts[-1]).astype(f))
    g = gy.astype(f)
    gc = np.zeros_like(coefs)
    for s in range(len(coefs) - 1, -1, -1):
        b0, b1, b2, a1, a2 = coefs[s]
        uu, yy = acts[s], acts[s + 1]
        v = lfilter(np.array([1], f), np.array([1, a1, a2], f), g[::-1]).astype(f)[::-1]
        vp = np.concatenate([v, np.zeros(2, f)])
        g = (b0 * vp[:-2] + b1 * vp[1:-1] + b2 * vp[2:]).astype(f)
        gc[s] = [v @ uu, v[1:] @ uu[:-1], v[2:] @ uu[:-2], -(v[1:] @ yy[:-1]), -(v[2:] @ yy[:-2])]
    gx = np.convolve(g, h.astype(f)[::-1], "full").astype(f)
    gh = np.correlate(x.astype(f), g, "valid")[::-1].astype(f)
    return acts[-1], gx, gh, gc.reshape(-1)


def _rel(got, want):
    return float(np.abs(np.asarray(got, np.float64) - want).max() / max(np.abs(want).max(), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("radius", [0.99, 0.995, 0.999])
def test_bank_poles_near_unit_circle(radius):
    """Every pole at radius 0.99 / 0.995 / 0.999 (the regime the FP64-formed transition
    powers exist for), channels of many scan segments, against FP64.  Bound per channel
    and quantity: max(1e-4, 4 x the error of the sequential FP32 step), the FP32
    recursion's own error growing like 1 / (1 - r)."""
    rng = np.random.default_rng(int(radius * 1000))
    lengths, taps, stages = [70000, 23000, 9000, 4200], [64, 17, 200, 1], [2, 3, 4, 1]
    x = rng.standard_normal(sum(lengths)).astype(np.float32).astype(np.float64)
    h = np.concatenate([rng.standard_normal(T) / np.sqrt(T) for T in taps]).astype(np.float32).astype(np.float64)
    c = np.concatenate([stable_sections(rng, S, radius=(radius, radius)).reshape(-1) for S in stages])
    c = c.astype(np.float32).astype(np.float64)
    gy = rng.standard_normal(len(x)).astype(np.float32).astype(np.float64)
    o = 0
    for L, T in zip(lengths, taps):
        gy[o + L - T + 1:o + L] = 0.0
        o += L
    bank, (y, gx, gh, gc) = _run_bank(lengths, taps, stages, x, h, c, gy)
    xo = ho = co = 0
    for L, T, S in zip(lengths, taps, stages):
        xs, hs, cs = x[xo:xo + L], h[ho:ho + T], c[co:co + 5 * S]
        gys = gy[xo:xo + L - T + 1]
        y64, _ = channel_forward(xs, hs, cs)
        gx64, gh64, gc64 = channel_adjoint(xs, hs, cs, gys)
        y32, gx32, gh32, gc32 = _fp32_channel_step(xs, hs, cs, gys)
        for name, got, want, seq in (("y", y[xo:xo + L - T + 1], y64, y32), ("gx", gx[xo:xo + L], gx64, gx32),
                                     ("gtaps", gh[ho:ho + T], gh64, gh32),
                                     ("gcoefs", gc[co:co + 5 * S], gc64.reshape(-1), gc32)):
            bound = max(1e-4, 4 * _rel(seq, want))
            assert _rel(got, want) <= bound, (radius, L, name, _rel(got, want), _rel(seq, want))
        xo, ho, co = xo + L, ho + T, co + 5 * S


@pytest.mark.gpu
def test_bank_deep_cascades_beyond_shared_memory():
    """24 and 22 stages beside shallow ones: the unit transitions of deep cascades
    (48 x 48 state) and the adjoint's per-stage sequences in shared memory."""
    lengths, taps, stages, x, h, c = _bank_case(8, 5, Lrange=(2000, 12000), Tmax=32, Smax=4,
                                                force=[(9000, 16, 24), (3000, 3, 22)])
    _check_bank(lengths, taps, stages, x, h, c)


@pytest.mark.gpu
def test_fused_step_equals_separate_calls():
    """DSPLIB_gpu_firBiquadBatched_stepMse against forward + MSE + adjoint as three calls:
    y, gy and every gradient bitwise equal, the loss to FP64 summation order."""
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages, x, h, c = _bank_case(13, 20, Lrange=(100, 30000), Tmax=96, Smax=6,
                                                force=[(70000, 33, 4), (600, 1, 0)])
    bank = RaggedFilterBank(lengths, taps, stages)
    dev = "cuda"
    xt, ht, ct = (torch.tensor(a, dtype=torch.float32, device=dev) for a in (x, h, c))
    target = torch.randn(bank.sizes[0], device=dev, generator=torch.Generator(dev).manual_seed(3))
    n = bank.sizes[0]
    sep = {k: torch.empty(n, device=dev) for k in ("y", "gy", "gx")}
    sep["gtaps"], sep["gcoefs"] = torch.empty_like(ht), torch.empty_like(ct)
    sep["loss"] = torch.empty(1, device=dev)
    work = torch.empty(bank.sizes[3], device=dev)
    scratch = torch.empty(bank.sizes[4], device=dev)
    bank.forward_raw(xt, ht, ct, sep["y"], work)
    bank.mse_grad_raw(sep["y"], target, sep["gy"], sep["loss"], scratch)
    bank.backward_raw(xt, ht, ct, work, sep["gy"], sep["gx"], sep["gtaps"], sep["gcoefs"], scratch)
    fus = {k: torch.full_like(v, 7.0) for k, v in sep.items()}
    work2 = torch.empty_like(work)
    scratch2 = torch.empty_like(scratch)
    bank.step_mse_raw(xt, ht, ct, target, fus["y"], fus["gy"], fus["loss"], fus["gx"], fus["gtaps"],
                      fus["gcoefs"], work2, scratch2)
    torch.cuda.synchronize()
    for k in ("y", "gy", "gx", "gtaps", "gcoefs"):
        assert torch.equal(fus[k], sep[k]), k
    assert float(fus["loss"]) == pytest.approx(float(sep["loss"]), rel=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [True, False])
def test_host_step_equals_device_step(pinned):
    """DSPLIB_gpu_firBiquadBatched_stepMseHost on host tensors (several pipelined channel
    segments: 7.3 M samples at 2 M samples per segment) against the device call:
    y, gy and every gradient bitwise equal, the loss to FP64 summation order; twice in a
    row, then with gy omitted and the taps / coefficients left on the device."""
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages, x, h, c = _bank_case(21, 60, Lrange=(1000, 240000), Tmax=300, Smax=8,
                                                force=[(262144, 512, 8), (300, 300, 0)])
    bank = RaggedFilterBank(lengths, taps, stages)
    assert bank.sizes[0] > 6_000_000
    dev = "cuda"
    xt, ht, ct = (torch.tensor(a, dtype=torch.float32, device=dev) for a in (x, h, c))
    target = torch.randn(bank.sizes[0], device=dev, generator=torch.Generator(dev).manual_seed(5))
    n = bank.sizes[0]
    ref = {k: torch.empty(n, device=dev) for k in ("y", "gy", "gx")}
    ref["gtaps"], ref["gcoefs"], ref["loss"] = torch.empty_like(ht), torch.empty_like(ct), torch.empty(1, device=dev)
    bank.step_mse_raw(xt, ht, ct, target, ref["y"], ref["gy"], ref["loss"], ref["gx"], ref["gtaps"], ref["gcoefs"],
                      torch.empty(bank.sizes[3], device=dev), torch.empty(bank.sizes[4], device=dev))
    torch.cuda.synchronize()
    ref = {k: v.cpu() for k, v in ref.items()}

    def host(t):
        t = t.cpu()
        return t.pin_memory() if pinned else t.clone()

    hx, hh, hc, ht_ = host(xt), host(ht), host(ct), host(target)
    for rep in range(3):
        out = {k: host(torch.full_like(v, 7.0)) for k, v in ref.items()}
        taps_in, coefs_in, gy_out = (hh, hc, out["gy"]) if rep < 2 else (ht, ct, None)
        if rep == 2:
            out["gtaps"], out["gcoefs"] = torch.full_like(ht, 7.0), torch.full_like(ct, 7.0)
        bank.step_mse_host(hx, taps_in, coefs_in, ht_, out["y"], gy_out, out["loss"], out["gx"], out["gtaps"],
                           out["gcoefs"])
        for k in ("y", "gy", "gx", "gtaps", "gcoefs"):
            if k == "gy" and gy_out is None:
                continue
            assert torch.equal(out[k].cpu(), ref[k]), (rep, k)
        assert float(out["loss"]) == pytest.approx(float(ref["loss"]), rel=1e-6)


@pytest.mark.gpu
def test_host_step_async_two_plans_in_flight():
    """Two plans of the same bank, each DSPLIB_gpu_raggedPlanSetAsync(plan, 1), calls queued
    on two streams before either finishes (one call's copies out overlap the next's copies
    in), three rounds: every result bitwise equal to the device step's."""
    import torch

    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages, x, h, c = _bank_case(22, 40, Lrange=(1000, 240000), Tmax=300, Smax=6)
    dev = "cuda"
    xt, ht, ct = (torch.tensor(a, dtype=torch.float32, device=dev) for a in (x, h, c))
    ref_bank = RaggedFilterBank(lengths, taps, stages)
    target = torch.randn(ref_bank.sizes[0], device=dev, generator=torch.Generator(dev).manual_seed(9))
    n = ref_bank.sizes[0]
    ref = {k: torch.empty(n, device=dev) for k in ("y", "gy", "gx")}
    ref["gtaps"], ref["gcoefs"], ref["loss"] = torch.empty_like(ht), torch.empty_like(ct), torch.empty(1, device=dev)
    ref_bank.step_mse_raw(xt, ht, ct, target, ref["y"], ref["gy"], ref["loss"], ref["gx"], ref["gtaps"],
                          ref["gcoefs"], torch.empty(ref_bank.sizes[3], device=dev),
                          torch.empty(ref_bank.sizes[4], device=dev))
    torch.cuda.synchronize()
    ref = {k: v.cpu() for k, v in ref.items()}
    hx, hh, hc, htg = (t.cpu().pin_memory() for t in (xt, ht, ct, target))
    banks = [RaggedFilterBank(lengths, taps, stages) for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    outs = []
    for b in banks:
        assert b.set_async(True) == 0
        outs.append({k: torch.full(v.shape, 7.0).pin_memory() for k, v in ref.items() if k != "gy"})
    for rnd in range(3):
        for b, st, o in zip(banks, streams, outs):
            st.synchronize()  # this slot's previous call finished: its buffers may be reused
            with torch.cuda.stream(st):
                b.step_mse_host(hx, hh, hc, htg, o["y"], None, o["loss"], o["gx"], o["gtaps"], o["gcoefs"])
        for b, st, o in zip(banks, streams, outs):
            st.synchronize()
            assert b.status() == 0
            for k in ("y", "gx", "gtaps", "gcoefs"):
                assert torch.equal(o[k], ref[k]), (rnd, k)
            assert float(o["loss"]) == pytest.approx(float(ref["loss"]), rel=1e-6)
