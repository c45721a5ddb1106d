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
