"""Failure paths of exec, made on the host (no GPU fault): DSPLIB_gpu_injectFault makes
the n-th CUDA operation an exec queues report a failure after it was queued.  Every
such call must return DSPLIB_ERR_FAILURE with a reason in DSPLIB_gpu_lastError, let the
copies and kernels it had queued finish (they touch the caller's buffers), and leave
the handle usable: the next call without injection computes the right result.

Covered: the host-buffer block pipelines of the FIR (pageable buffers of 8 MB and
more), the cascade biquad (page-locked signals of 4 MB and more) and the Q.15
conversion (8 MB and more staged), and the single-block paths of small buffers.
Also the error words of the tensor-core kernels: clear after normal calls."""
import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _fir_case(B, N, T, seed):
    rng = np.random.default_rng(seed)
    x = rng.integers(-4096, 4096, size=(B, N)).astype(np.int16)
    h = rng.integers(-4096, 4096, size=(1, T)).astype(np.int16)
    return x, h


@pytest.mark.parametrize("B,N", [(8, 300000), (3, 2000)])
def test_fir_injected_failures_drain_and_recover(B, N):
    T = 64
    x, h = _fir_case(B, N, T, 1)
    want = oracle.fir(x, h, T, nch=0)
    args, pin, pf, po = D.fir_setup(D.INT16, B, N, T, nch=0)
    hd = D.FirHandle()
    assert hd.init(args, pin, pf, po) == D.SUCCESS
    failed = 0
    for n in range(1, 12):
        y = np.zeros((B, N - T + 1), np.int16)
        assert hd.inject_fault(n) == D.SUCCESS
        st = hd.exec(x, h, y)
        if st == D.SUCCESS:  # fewer operations than n: nothing was injected
            assert np.array_equal(y, want)
            break
        assert st == D.ERR_FAILURE, (n, st)
        assert hd.last_error() != ""
        failed += 1
        y = np.zeros_like(y)
        assert hd.exec(x, h, y) == D.SUCCESS, hd.last_error()  # the handle is usable again
        assert np.array_equal(y, want), n
    assert failed >= 3


@pytest.mark.parametrize("N,pinned", [(65536, True), (1000, False)])
def test_biquad_injected_failures_drain_and_recover(N, pinned):
    C, S = 32, 4
    rng = np.random.default_rng(2)
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = np.tile(np.array([[0.3, 0.2, 0.1, -0.9, 0.4]], np.float32), (1, S))
    opt, _ = D.opt_coefficients(nat, D.DF2, 0, C)
    args, pin, pout, pvar, pcn, popt = D.biquad_descs(C, N, S, D.DF2, 0)
    hd = D.BiquadHandle()
    assert hd.init(args, pin, popt, pvar, pout) == D.SUCCESS
    mk = (lambda a: torch.from_numpy(a).pin_memory()) if pinned else (lambda a: torch.from_numpy(a))
    xs = mk(x)
    cs = mk(opt)

    def run(inject):
        st0 = np.zeros((2 * S, C), np.float32)
        y = mk(np.zeros_like(x))
        sv = mk(st0)
        if inject:
            hd.inject_fault(inject)
        return hd.exec(xs, cs, sv, y), y.numpy().copy(), sv.numpy().copy()

    st, want_y, want_s = run(0)
    assert st == D.SUCCESS
    failed = 0
    for n in range(1, 14):
        st, _, _ = run(n)
        if st == D.SUCCESS:
            break
        assert st == D.ERR_FAILURE and hd.last_error() != ""
        failed += 1
        st, y, sv = run(0)
        assert st == D.SUCCESS
        assert np.array_equal(y, want_y) and np.array_equal(sv, want_s), n
    assert failed >= 3


@pytest.mark.parametrize("n", [(1 << 23) + 5, 1000])
def test_q15_injected_failures_drain_and_recover(n):
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    hd = D.Fltoq15Handle()
    want = D.fltoq15(x, handle=hd)  # initialises the handle (reference call sequence) and runs once
    failed = 0
    for k in range(1, 14):
        out = np.zeros(n, np.int16)
        assert hd.inject_fault(k) == D.SUCCESS
        st = hd.exec(x, out)
        if st == D.SUCCESS:
            assert np.array_equal(out, want)
            break
        assert st == D.ERR_FAILURE and hd.last_error() != ""
        failed += 1
        out = np.zeros(n, np.int16)
        assert hd.exec(x, out) == D.SUCCESS
        assert np.array_equal(out, want), k
    assert failed >= 2


def test_tensor_core_error_words_clear_after_normal_calls():
    rng = np.random.default_rng(4)
    x = rng.integers(-128, 128, size=(4, 9000)).astype(np.int8)
    h = rng.integers(-128, 128, size=(1, 128)).astype(np.int8)
    hd = D.FirHandle()
    args, pin, pf, po = D.fir_setup(D.INT8, 4, 9000, 128, nch=0, shift=7)
    assert hd.init(args, pin, pf, po) == D.SUCCESS
    hd.set_qmode(True)
    hd.set_async(True)
    y = torch.zeros((4, 9000 - 127), dtype=torch.int8, device="cuda")
    xd, hdev = torch.from_numpy(x).cuda(), torch.from_numpy(h).cuda()
    for _ in range(3):
        assert hd.exec(xd, hdev, y) == D.SUCCESS
    torch.cuda.synchronize()
    assert hd.status() == D.SUCCESS
    assert np.array_equal(y.cpu().numpy(), oracle.fir_q(x, h, 128, 7, nch=0))
    from c7x_dsplib_b200 import lib
    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    bank = RaggedFilterBank([3000, 900], [31, 7], [2, 1])
    xt = torch.randn(3900, device="cuda")
    ht = torch.randn(38, device="cuda")
    ct = torch.tensor([0.5, 0.1, 0.0, -0.5, 0.2] * 3, dtype=torch.float32, device="cuda")
    bank.apply(xt, ht, ct)
    torch.cuda.synchronize()
    assert lib().DSPLIB_gpu_raggedPlanStatus(bank._plan) == D.SUCCESS
