"""FIR parity on the GPU, through the C ABI, against the CPU oracle.

NATC must be bit-exact to the reference natural-C kernel (integers wrap,
floats summed in tap order).  OPTIMIZED floats are checked against the FP64
oracle with a stated tolerance and against the reference criterion (abs
2^-10, test/DSPLIB_fir/DSPLIB_fir_d.c:315-317).  Q mode is bit-exact to the
oracle's output-stage restatement.
"""
import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle
from conftest import case_keys

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL_REF = 2.0 ** -10


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def rand(dt, shape, rng):
    if dt == np.float32:
        return rng.standard_normal(shape).astype(dt)
    info = np.iinfo(dt)
    return rng.integers(info.min, info.max, size=shape, endpoint=True).astype(dt)


SHAPES = [(1, 1, 1), (1, 17, 17), (3, 300, 37), (2, 2048, 1), (4, 5000, 256), (2, 3000, 1500), (5, 1025, 64)]


@pytest.mark.parametrize("dt", [np.int8, np.int16, np.int32, np.float32])
@pytest.mark.parametrize("nch", [0, 1])
@pytest.mark.parametrize("on_device", [False, True])
def test_natc_bitexact(dt, nch, on_device):
    rng = np.random.default_rng(11)
    for (B, N, T) in SHAPES:
        x = rand(dt, (B, N), rng)
        h = rand(dt, (B if nch else 1, T), rng)
        want = oracle.fir(x, h, T, nch=nch)
        if on_device:
            got = host(D.fir(dev(x), dev(h), T, nch=nch, func_style=D.NATC))
        else:
            got = D.fir(x, h, T, nch=nch, func_style=D.NATC)
        assert np.array_equal(got, want), (B, N, T)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference _cn library not built")
@pytest.mark.parametrize("dt", [np.int16, np.float32])
def test_natc_bitexact_vs_reference_cn(dt):
    rng = np.random.default_rng(5)
    x = rand(dt, (16, 4096), rng)
    h = rand(dt, (1, 64), rng)
    got = host(D.fir(dev(x), dev(h), 64, nch=0, func_style=D.NATC))
    assert np.array_equal(got, oracle.fir(x, h, 64, nch=0, impl="ref"))


@pytest.mark.parametrize("dt", [np.int8, np.int16, np.int32])
def test_opt_integer_default_is_wrap(dt):
    rng = np.random.default_rng(3)
    x, h = rand(dt, (3, 700, ), rng), rand(dt, (3, 50), rng)
    got = host(D.fir(dev(x), dev(h), 50, nch=1, func_style=D.OPTIMIZED))
    assert np.array_equal(got, oracle.fir(x, h, 50, nch=1))


@pytest.mark.parametrize("dt,shift", [(np.int8, 7), (np.int8, 0), (np.int16, 15), (np.int16, 3), (np.int32, 31),
                                      (np.int32, 0), (np.int8, 26), (np.int8, 31), (np.int8, 32), (np.int8, 62),
                                      (np.int16, 40), (np.int16, 62), (np.int32, 62)])
def test_qmode_bitexact(dt, shift):
    rng = np.random.default_rng(shift + 1)
    for (B, N, T) in [(2, 700, 64), (3, 4096, 128), (1, 40, 40)]:
        x, h = rand(dt, (B, N), rng), rand(dt, (B, T), rng)
        got = host(D.fir(dev(x), dev(h), T, nch=1, func_style=D.OPTIMIZED, qmode=True, shift=shift))
        assert np.array_equal(got, oracle.fir_q(x, h, T, shift, nch=1)), (B, N, T)


@pytest.mark.parametrize("dt", [np.int8, np.int16, np.int32])
def test_qmode_shift_beyond_accumulator_rejected(dt):
    """Q mode takes shifts up to 62; beyond, exec refuses with DSPLIB_ERR_INVALID_VALUE and
    leaves the output untouched (the wrap mode ignores the shift, as the natural-C kernel)."""
    B, N, T = 2, 300, 16
    rng = np.random.default_rng(23)
    x, hh = rand(dt, (B, N), rng), rand(dt, (1, T), rng)
    args, pin, pfilt, pout = D.fir_setup(_NP_CODE[dt], B, N, T, nch=0, shift=63)
    h = D.FirHandle()
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    out = dev(np.full((B, N - T + 1), 5, dt))
    h.set_qmode(True)
    assert h.exec(dev(x), dev(hh), out) == D.ERR_INVALID_VALUE
    assert "shift" in h.last_error()
    assert np.all(host(out) == 5)
    h.set_qmode(False)
    assert h.exec(dev(x), dev(hh), out) == D.SUCCESS
    assert np.array_equal(host(out), oracle.fir(x, hh, T, nch=0))


_NP_CODE = {np.int8: D.INT8, np.int16: D.INT16, np.int32: D.INT32}


@pytest.mark.parametrize("dt", [np.int8, np.int16])
@pytest.mark.parametrize("shift", [30, 31, 32, 33, 47, 62])
def test_qmode_boundary_shifts(dt, shift):
    """Q-mode shifts around and beyond the 32-bit accumulator of the int8 output stage and up
    to the 62 accepted: bit-exact to the restatement (large shifts round every output to 0
    or -1 exactly as the exact accumulator does), on the tensor-core kernel."""
    rng = np.random.default_rng(shift)
    info = np.iinfo(dt)
    x = rng.integers(info.min, info.max, size=(3, 5000), endpoint=True).astype(dt)
    h = rng.integers(info.min, info.max, size=(1, 128), endpoint=True).astype(dt)
    got = host(D.fir(dev(x), dev(h), 128, nch=0, func_style=D.OPTIMIZED, qmode=True, shift=shift))
    assert np.array_equal(got, oracle.fir_q(x, h, 128, shift, nch=0))


@pytest.mark.parametrize("dt", [np.int8, np.int16])
@pytest.mark.parametrize("qmode", [False, True])
def test_int_tensor_core_edges(dt, qmode):
    """Tensor-core integer path: partial tiles, odd pitches, extreme values, long filters
    (T <= 2048 on the tensor cores, beyond that the CUDA-core kernel)."""
    rng = np.random.default_rng(21)
    info = np.iinfo(dt)
    for (B, N, T, nch) in [(1, 16, 1, 0), (2, 2047 + 30, 31, 1), (3, 5000, 2048, 0), (2, 4500, 2100, 1),
                           (5, 2049 + 127, 128, 1), (1, 70000, 97, 0)]:
        x = rand(dt, (B, N), rng)
        h = rand(dt, (B if nch else 1, T), rng)
        x[:, :8] = info.min  # the hi/lo split must handle the extremes
        h[:, :3] = info.min
        h[:, -2:] = info.max
        shift = 7 if dt == np.int8 else 15
        got = host(D.fir(dev(x), dev(h), T, nch=nch, func_style=D.OPTIMIZED, qmode=qmode, shift=shift))
        want = oracle.fir_q(x, h, T, shift, nch=nch) if qmode else oracle.fir(x, h, T, nch=nch)
        assert np.array_equal(got, want), (B, N, T, nch)


def test_int_tensor_core_unaligned_rows():
    """Row pitch not a multiple of 16 bytes (vector loads must not be used)."""
    rng = np.random.default_rng(22)
    B, N, T, pitch = 3, 3001, 64, 3003
    x = np.zeros((B, pitch), np.int8)
    x[:, :N] = rand(np.int8, (B, N), rng)
    hh = rand(np.int8, (1, T), rng)
    args, pin, pfilt, pout = D.fir_setup(D.INT8, B, N, T, nch=0, in_pitch=pitch, out_pitch=N - T + 5)
    out = np.zeros((B, N - T + 5), np.int8)
    h = D.FirHandle()
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    h.set_qmode(True)
    xd, hd, od = dev(x), dev(hh), dev(out)
    assert h.exec(xd, hd, od) == D.SUCCESS, h.last_error()
    want = oracle.fir_q(np.ascontiguousarray(x[:, :N]), hh, T, 0, nch=0)
    assert np.array_equal(host(od)[:, : N - T + 1], want)


def _relerr(y, y64):
    return np.max(np.abs(y.astype(np.float64) - y64), axis=1) / np.maximum(np.max(np.abs(y64), axis=1), 1e-30)


@pytest.mark.parametrize("nch", [0, 1])
def test_simt_float_accuracy(nch):
    rng = np.random.default_rng(9)
    for (B, N, T) in [(4, 5000, 256), (2, 3000, 1500), (3, 100, 1), (2, 9000, 33)]:
        x = rng.standard_normal((B, N)).astype(np.float32)
        h = (rng.standard_normal((B if nch else 1, T)) / np.sqrt(T)).astype(np.float32)
        y = host(D.fir(dev(x), dev(h), T, nch=nch, precision=D.FIR_SIMT))
        y64 = oracle.fir_f64(x, h, T, nch=nch)
        assert np.max(_relerr(y, y64)) <= 2e-6, (B, N, T)
        assert np.max(np.abs(y - oracle.fir(x, h, T, nch=nch))) <= TOL_REF


def lowpass(rng, rows, T):
    """Hamming-windowed sinc low-pass, cutoff U[0.05, 0.45], unit DC gain (stored tap order)."""
    n = np.arange(T) - (T - 1) / 2.0
    out = np.zeros((rows, T), np.float32)
    for r in range(rows):
        fc = rng.uniform(0.05, 0.45)
        hh = fc * np.sinc(fc * n) * np.hamming(T) if T > 1 else np.ones(1)
        out[r] = (hh / hh.sum())[::-1]
    return out


@pytest.mark.parametrize("nch", [0, 1])
def test_bf16x3_accuracy(nch):
    """Split-BF16x3 tensor-core FIR: max |y - y64| / max |y64| <= 1e-5 per channel
    (N(0,1) input, windowed-sinc taps as in the FP32 FIR workload), and the
    reference criterion abs 2^-10 against the natural-C result."""
    rng = np.random.default_rng(31 + nch)
    for (B, N, T) in [(2, 9000, 1), (3, 70000, 256), (2, 5000, 512), (2, 3000, 100), (1, 300, 255)]:
        x = rng.standard_normal((B, N)).astype(np.float32)
        hh = lowpass(rng, B if nch else 1, T)
        y = host(D.fir(dev(x), dev(hh), T, nch=nch, precision=D.FIR_BF16X3))
        y64 = oracle.fir_f64(x, hh, T, nch=nch)
        assert np.max(_relerr(y, y64)) <= 1e-5, (B, N, T)
        assert np.max(np.abs(y - oracle.fir(x, hh, T, nch=nch))) <= TOL_REF


def test_bf16x3_tile_runs_per_cta():
    """Enough channels that each CTA filters a run of four consecutive 8192-output tiles of
    one channel (raw tiles two ahead in the ring, barrier phases carried across tiles);
    per-channel taps, rows whose starts alternate between 16-byte aligned and not."""
    rng = np.random.default_rng(41)
    B, T = 300, 251
    N = 4 * 8192 + T - 1
    x = rng.standard_normal((B, N)).astype(np.float32)
    hh = lowpass(rng, B, T)
    y = host(D.fir(dev(x), dev(hh), T, nch=1, precision=D.FIR_BF16X3))
    assert np.max(_relerr(y, oracle.fir_f64(x, hh, T, nch=1))) <= 1e-5


def test_bf16x3_long_filter_uses_fp32_kernel():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 3000)).astype(np.float32)
    hh = (rng.standard_normal((2, 700)) / 30).astype(np.float32)
    y = host(D.fir(dev(x), dev(hh), 700, nch=1, precision=D.FIR_BF16X3))
    assert np.max(_relerr(y, oracle.fir_f64(x, hh, 700, nch=1))) <= 2e-6


def test_bf16x3_unaligned_rows():
    rng = np.random.default_rng(6)
    B, N, T, pitch = 3, 20001, 64, 20003
    x = np.zeros((B, pitch), np.float32)
    x[:, :N] = rng.standard_normal((B, N))
    hh = lowpass(rng, 1, T)
    args, pin, pfilt, pout = D.fir_setup(D.FLOAT32, B, N, T, nch=0, in_pitch=pitch, out_pitch=N - T + 3)
    out = np.zeros((B, N - T + 3), np.float32)
    h = D.FirHandle()
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    h.set_precision(D.FIR_BF16X3)
    xd, hd, od = dev(x), dev(hh), dev(out)
    assert h.exec(xd, hd, od) == D.SUCCESS, h.last_error()
    y64 = oracle.fir_f64(np.ascontiguousarray(x[:, :N]), hh, T, nch=0)
    assert np.max(_relerr(host(od)[:, : N - T + 1], y64)) <= 1e-5


def _golden_cases():
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "fir_golden.npz"))
    return case_keys(d, "f")


@pytest.mark.parametrize("key", _golden_cases())
@pytest.mark.parametrize("style", [D.NATC, D.OPTIMIZED])
def test_reference_flow_golden(golden_fir, key, style):
    """The reference driver's call sequence (DSPLIB_fir_d.c:101-305) including
    the padded MMA filter layout, checked against the reference golden output."""
    meta = golden_fir[key + "_meta"]
    _, N, T, B, nch, mma = (int(v) for v in meta)
    x, taps, yg = golden_fir[key + "_x"], golden_fir[key + "_h"], golden_fir[key + "_y"]
    args, pin, pfilt, pout = D.fir_setup(D.FLOAT32, B, N, T, nch=nch, func_style=style, mma=mma)
    M = args.MMA_SIZE
    rows = B if nch else 1
    if mma:  # taps at offset 2*MMA_SIZE of zeroed padded rows (DSPLIB_fir_d.c:195-208)
        fbuf = np.zeros((rows, pfilt.stride_y // 4), np.float32)
        fbuf[:, 2 * M: 2 * M + T] = taps
    else:
        fbuf = np.ascontiguousarray(taps)
    h = D.FirHandle()
    assert h.init_check(args, pin, pfilt, pout) == D.SUCCESS
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    out = np.zeros((B, pout.stride_y // 4), np.float32)
    fptr = fbuf.ctypes.data + (2 * M * 4 if (mma and style == D.NATC) else 0)  # DSPLIB_fir_d.c:303-305
    assert D.lib().DSPLIB_fir_exec(h.h, x.ctypes.data, fptr, out.ctypes.data) == D.SUCCESS, h.last_error()
    y = out[:, : N - T + 1]
    assert np.max(np.abs(y - yg)) <= TOL_REF
    if style == D.NATC:
        assert np.array_equal(y, oracle.fir(x, taps, T, nch=nch))


def test_strided_rows_keep_gaps():
    """Host buffers with pitch > row width: bytes between rows are left untouched."""
    rng = np.random.default_rng(2)
    B, N, T, pin_p, pout_p = 3, 200, 9, 256, 250
    x = np.zeros((B, pin_p), np.float32)
    x[:, :N] = rng.standard_normal((B, N))
    hh = rng.standard_normal((1, T)).astype(np.float32)
    args, pin, pfilt, pout = D.fir_setup(D.FLOAT32, B, N, T, nch=0, in_pitch=pin_p, out_pitch=pout_p)
    out = np.full((B, pout_p), 7.0, np.float32)
    h = D.FirHandle()
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    # out dim_x = pout_p from the descriptor, as the reference driver sets it (DSPLIB_fir_d.c:128)
    assert h.exec(x, hh, out) == D.SUCCESS
    want = oracle.fir(np.ascontiguousarray(x[:, :N]), hh, T, nch=0)
    assert np.max(np.abs(out[:, : N - T + 1] - want)) <= TOL_REF
    assert np.all(out[:, N - T + 1:] == 7.0)


def test_async_stream_device():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((8, 10000)).astype(np.float32)
    hh = rng.standard_normal((1, 100)).astype(np.float32)
    xd, hd = dev(x), dev(hh)
    yd = torch.zeros((8, 10000 - 99), device="cuda")
    args, pin, pfilt, pout = D.fir_setup(D.FLOAT32, 8, 10000, 100, nch=0)
    h = D.FirHandle()
    assert h.init(args, pin, pfilt, pout) == D.SUCCESS
    s = torch.cuda.Stream()
    h.set_stream(s)
    h.set_async(True)
    n0 = D.kernel_launch_count()
    with torch.cuda.stream(s):
        assert h.exec(xd, hd, yd) == D.SUCCESS
    s.synchronize()
    assert D.kernel_launch_count() == n0 + 1
    assert np.max(np.abs(host(yd) - oracle.fir(x, hh, 100, nch=0))) <= TOL_REF


@pytest.mark.parametrize("dt,precision,qmode,B,N,T", [
    (np.int16, D.FIR_SIMT, False, 96, 65536, 64),   # tensor-core wrap, even blocks
    (np.int8, D.FIR_SIMT, True, 130, 65536, 128),   # tensor-core Q mode
    (np.float32, D.FIR_SIMT, False, 37, 65536, 33),  # odd batch: unequal blocks
    (np.float32, D.FIR_BF16X3, False, 37, 65536, 256),
])
@pytest.mark.parametrize("pinned", [False, True])
def test_host_buffers_pipelined(dt, precision, qmode, B, N, T, pinned):
    """Host buffers of 8 MB and more run as a copy-in / compute / copy-out
    pipeline over channel blocks: results equal the device-buffer call bit for bit."""
    rng = np.random.default_rng(B + T)
    x = rand(dt, (B, N), rng)
    h = rand(dt, (B, T), rng) if dt != np.float32 else (rng.standard_normal((B, T)) / T).astype(np.float32)
    shift = 7 if dt == np.int8 else 0
    want = host(D.fir(dev(x), dev(h), T, nch=1, precision=precision, qmode=qmode, shift=shift))
    if pinned:
        xh = torch.from_numpy(x).pin_memory()
        hh = torch.from_numpy(h).pin_memory()
        out = torch.zeros((B, N - T + 1), dtype=xh.dtype).pin_memory()
        got = D.fir(xh, hh, T, nch=1, precision=precision, qmode=qmode, shift=shift, out=out).numpy()
    else:
        got = D.fir(x, h, T, nch=1, precision=precision, qmode=qmode, shift=shift)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("dt,style,precision,qmode,C,T,N,blocks", [
    (np.int16, D.NATC, D.FIR_SIMT, False, 5, 37, 100, 6),       # bit-exact natural C
    (np.int8, D.OPTIMIZED, D.FIR_SIMT, True, 3, 64, 16, 9),     # block shorter than the history, tensor cores
    (np.float32, D.OPTIMIZED, D.FIR_BF16X3, False, 4, 256, 4096, 3),
])
@pytest.mark.parametrize("on_device", [False, True])
def test_fir_stream_matches_one_call(dt, style, precision, qmode, C, T, N, blocks, on_device):
    """Streaming FIR: blocks filtered one call at a time equal one call over the
    whole signal preceded by T - 1 zeros."""
    rng = np.random.default_rng(C * T + N)
    x = rand(dt, (C, N * blocks), rng)
    h = rand(dt, (C, T), rng) if dt != np.float32 else (rng.standard_normal((C, T)) / T).astype(np.float32)
    shift = 7 if qmode else 0
    code = {np.int8: D.INT8, np.int16: D.INT16, np.float32: D.FLOAT32}[dt]
    st = D.FirStream(code, C, N, T, nch=1, func_style=style, shift=shift, precision=precision, qmode=qmode)
    padded = np.concatenate([np.zeros((C, T - 1), dt), x], axis=1)
    if dt == np.float32:
        want64 = oracle.fir_f64(padded, h, T, nch=1)
    elif qmode:
        want = oracle.fir_q(padded, h, T, shift, nch=1)
    else:
        want = oracle.fir(padded, h, T, nch=1)
    hd = dev(h) if on_device else h
    got = []
    for b in range(blocks):
        xb = np.ascontiguousarray(x[:, b * N:(b + 1) * N])
        if on_device:
            out = torch.zeros((C, N), dtype=dev(xb).dtype, device="cuda")
            got.append(host(st.exec(dev(xb), hd, out)))
        else:
            out = np.zeros((C, N), dt)
            got.append(st.exec(xb, hd, out))
    got = np.concatenate(got, axis=1)
    if dt == np.float32:
        peak = np.abs(want64).max(axis=1, keepdims=True)
        assert np.max(np.abs(got - want64) / peak) <= 1e-5
    else:
        assert np.array_equal(got, want)
    # reset starts a new signal: the first block again
    st.reset()
    xb = np.ascontiguousarray(x[:, :N])
    out = np.zeros((C, N), dt)
    again = st.exec(xb, h, out)
    assert np.array_equal(again, got[:, :N])


def test_handles_on_concurrent_host_threads():
    """Handles are independent: host threads filtering pageable host buffers at the same
    time (per-thread staging buffers and copy pipelines) give the oracle's results."""
    import threading

    rng = np.random.default_rng(21)
    jobs = []
    for k in range(4):
        x = rng.integers(-1000, 1000, (64, 40000)).astype(np.int16)
        h = rng.integers(-1000, 1000, (64, 33)).astype(np.int16)
        jobs.append((x, h))
    results, errors = [None] * len(jobs), []

    def work(k):
        try:
            x, h = jobs[k]
            hd = D.FirHandle()
            s = torch.cuda.Stream()
            ys = []
            for _ in range(3):
                args, pin, pf, po = D.fir_setup(D.INT16, 64, 40000, 33, nch=True)
                assert hd.init(args, pin, pf, po) == D.SUCCESS
                hd.set_stream(s)
                y = np.zeros((64, 40000 - 32), np.int16)
                assert hd.exec(x, h, y) == D.SUCCESS, hd.last_error()
                ys.append(y)
            results[k] = ys
        except Exception as e:  # reported below
            errors.append(repr(e))

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (x, h), ys in zip(jobs, results):
        want = oracle.fir(x, h, 33, nch=True)
        for y in ys:
            assert np.array_equal(y, want)


# ------------------------------------------------------------------ float Q mode


@pytest.mark.parametrize("Q", [0, 8, 15, 24, 31])
@pytest.mark.parametrize("nch", [0, 1])
def test_float_q_mode_bitexact(Q, nch):
    """FLOAT32 with InitArgs.enableQ: quantised to int32 at scale 2^Q, exact integer sums,
    rounding shift and saturation (the C7x fixed-point MMA path), bit-exact to the
    restatement; the saturation at large Q included (|x| 2^31 overflows int32)."""
    rng = np.random.default_rng(40 + Q + nch)
    for (B, N, T) in [(1, 17, 17), (3, 2000, 64), (2, 5000, 1500)]:
        x = rng.standard_normal((B, N)).astype(np.float32)
        h = (rng.standard_normal((B if nch else 1, T)) / np.sqrt(T)).astype(np.float32)
        x[0, :3] = [np.inf, -np.inf, np.nan]
        got = host(D.fir(dev(x), dev(h), T, nch=nch, float_q=Q))
        want = oracle.fir_floatq(x, h, T, Q, nch=nch)
        assert np.array_equal(got, want, equal_nan=True), (B, N, T)


def test_float_q_mode_tracks_fp64_and_rejects_large_q():
    rng = np.random.default_rng(44)
    x = rng.uniform(-1, 1, (2, 4096)).astype(np.float32)
    h = (rng.standard_normal((1, 128)) / 16).astype(np.float32)
    got = host(D.fir(dev(x), dev(h), 128, nch=0, float_q=20)).astype(np.float64)
    w = oracle.fir_f64(x, h, 128, nch=0)
    # each operand carries at most 2^-21 of quantisation error: |err| <= T 2^-20 max|x| max|h| roughly
    assert np.abs(got - w).max() <= 128 * 2.0 ** -20 * float(np.abs(h).max() + 1)
    args, pin, pf, po = D.fir_setup(D.FLOAT32, 2, 4096, 128, nch=0, float_q=32)
    hd = D.FirHandle()
    assert hd.init(args, pin, pf, po) == D.SUCCESS
    out = dev(np.zeros((2, 4096 - 127), np.float32))
    assert hd.exec(dev(x), dev(h), out) == D.ERR_INVALID_VALUE
    assert "Q" in hd.last_error()
