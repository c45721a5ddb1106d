"""torch.ops.dsplib_gpu.*: the C ABI registered as PyTorch operators (queued on the current
stream, fake implementations for tracing).  GPU tests compare each operator with the
synchronous library call on the same inputs."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_operators_registered():
    import c7x_dsplib_b200.torch_ops  # noqa: F401

    for name in ("fir", "cascade_biquad", "fltoq15", "q15tofl"):
        assert hasattr(torch.ops.dsplib_gpu, name)


def test_fake_shapes():
    import c7x_dsplib_b200.torch_ops  # noqa: F401
    from torch._subclasses.fake_tensor import FakeTensorMode

    with FakeTensorMode():
        x = torch.empty(4, 100, dtype=torch.int16, device="cuda")
        h = torch.empty(1, 9, dtype=torch.int16, device="cuda")
        assert torch.ops.dsplib_gpu.fir(x, h, False, 0, True, 3).shape == (4, 92)
        f = torch.empty(10, 3, device="cuda")
        assert torch.ops.dsplib_gpu.fltoq15(f, 1).dtype == torch.int16
        assert torch.ops.dsplib_gpu.q15tofl(torch.empty(7, dtype=torch.int16, device="cuda"),
                                            torch.float64).dtype == torch.float64


@pytest.mark.gpu
def test_ops_match_library_calls_on_a_side_stream():
    import c7x_dsplib_b200 as D
    import c7x_dsplib_b200.torch_ops  # noqa: F401

    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.integers(-2000, 2000, (6, 5000)).astype(np.int16)).cuda()
    h = torch.from_numpy(rng.integers(-2000, 2000, (1, 31)).astype(np.int16)).cuda()
    xf = torch.from_numpy(rng.standard_normal((3000, 40)).astype(np.float32)).cuda()
    nat = np.array([[0.2, 0.1, 0.2, -0.9, 0.5, 0.3, -0.1, 0.3, -0.5, 0.4]], np.float32)
    opt, _ = D.opt_coefficients(nat, D.DF2, 0, 40)
    cd = torch.from_numpy(opt).cuda()
    want_fir = D.fir(x, h, nch=False, qmode=True, shift=4)
    st_ref = torch.zeros(4, 40, device="cuda")
    want_bq = D.cascade_biquad(xf, cd, st_ref, form=D.DF2, nch=0)
    side = torch.cuda.Stream()
    st = torch.zeros(4, 40, device="cuda")
    with torch.cuda.stream(side):
        y = torch.ops.dsplib_gpu.fir(x, h, False, 0, True, 4)
        yb = torch.ops.dsplib_gpu.cascade_biquad(xf, cd, st, D.DF2, False)
        q = torch.ops.dsplib_gpu.fltoq15(xf * 0.1, 1)
        back = torch.ops.dsplib_gpu.q15tofl(q, torch.float32)
    side.synchronize()
    assert torch.equal(y, want_fir)
    assert torch.equal(yb, want_bq) and torch.equal(st, st_ref)
    assert torch.equal(q, D.fltoq15((xf * 0.1).view(-1)))
    assert torch.equal(back, D.q15tofl(q, np.float32))


@pytest.mark.gpu
def test_ops_capture_in_cuda_graph():
    import c7x_dsplib_b200 as D
    import c7x_dsplib_b200.torch_ops  # noqa: F401

    x = torch.randn(128, 4096, device="cuda")
    h = torch.randn(1, 17, device="cuda") / 4
    y0 = torch.ops.dsplib_gpu.fir(x, h, False, 0, False, 0)  # eager call first
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        torch.ops.dsplib_gpu.fir(x, h, False, 0, False, 0)
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        yg = torch.ops.dsplib_gpu.fir(x, h, False, 0, False, 0)
    x.mul_(2.0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(yg, 2.0 * y0, rtol=1e-5, atol=1e-5)
    del D


@pytest.mark.gpu
@pytest.mark.parametrize("nch", [False, True])
def test_fir_operator_gradients_match_fp64(nch):
    """dx and dh of torch.ops.dsplib_gpu.fir (FLOAT32) against float64 autograd of the same
    correlation (y[j] = sum_c x[j + c] h[T - 1 - c])."""
    import c7x_dsplib_b200.torch_ops  # noqa: F401

    g = torch.Generator().manual_seed(5)
    B, N, T = 3, 400, 23
    x = torch.randn(B, N, generator=g)
    h = torch.randn(B if nch else 1, T, generator=g) / 5
    w = torch.randn(B, N - T + 1, generator=g)
    xd, hd = x.cuda().requires_grad_(), h.cuda().requires_grad_()
    (torch.ops.dsplib_gpu.fir(xd, hd, nch, 0, False, 0) * w.cuda()).sum().backward()
    x64, h64 = x.double().requires_grad_(), h.double().requires_grad_()
    hh = h64 if nch else h64.expand(B, T)
    y64 = torch.stack([torch.nn.functional.conv1d(x64[l].view(1, 1, -1), hh[l].flip(0).view(1, 1, -1)).view(-1)
                       for l in range(B)])
    (y64 * w.double()).sum().backward()
    for got, want in ((xd.grad, x64.grad), (hd.grad, h64.grad)):
        err = (got.double().cpu() - want).abs().max() / want.abs().max()
        assert err <= 1e-5, float(err)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [0, 1, 2, 3])
@pytest.mark.parametrize("nch", [False, True])
def test_cascade_operator_gradients_match_fp64(form, nch):
    """torch.ops.dsplib_gpu.cascade_biquad_natural: output and the gradients w.r.t. the
    input and the natural coefficients against the FP64 restatement of the adjoint."""
    import c7x_dsplib_b200.torch_ops  # noqa: F401
    from oracle.filterbank64 import channel_adjoint, channel_forward, stable_sections

    rng = np.random.default_rng(30 + form + 4 * nch)
    N, C, S = 3000, 6, 3
    x = rng.standard_normal((N, C)).astype(np.float32)
    rows = C if nch else 1
    nat = np.stack([stable_sections(rng, S).reshape(-1) for _ in range(rows)]).astype(np.float32)
    gy = rng.standard_normal((N, C)).astype(np.float32)
    xd = torch.from_numpy(x).cuda().requires_grad_()
    cd = torch.from_numpy(nat).cuda().requires_grad_()
    y = torch.ops.dsplib_gpu.cascade_biquad_natural(xd, cd, form)
    (y * torch.from_numpy(gy).cuda()).sum().backward()
    gc64 = np.zeros((C, 5 * S))
    for ch in range(C):
        c64 = nat[ch if nch else 0].astype(np.float64)
        y64, _ = channel_forward(x[:, ch].astype(np.float64), np.ones(1), c64)
        assert np.abs(y.detach().cpu().numpy()[:, ch] - y64).max() <= 1e-4 * np.abs(y64).max()
        gx64, _, gcc = channel_adjoint(x[:, ch].astype(np.float64), np.ones(1), c64, gy[:, ch].astype(np.float64))
        got = xd.grad.cpu().numpy()[:, ch]
        assert np.abs(got - gx64).max() <= 1e-4 * np.abs(gx64).max()
        gc64[ch] = gcc.reshape(-1)
    want = gc64 if nch else gc64.sum(axis=0, keepdims=True)
    got = cd.grad.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()
