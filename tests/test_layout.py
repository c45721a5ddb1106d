"""DSPLIB_interleave / DSPLIB_deinterleave / DSPLIB_addNCh: the layout conversions between
channel-major FIR buffers and time-major biquad buffers, and the channel sum after a
filter bank.

CPU: the C restatement against the golden fixtures (tests/golden/layout_golden.npz:
outputs of the reference's own DSPLIB_matTrans_cn.cpp / DSPLIB_addNCh_cn.cpp at the
shapes and strides of the reference test tables, plus the addNCh generator's float64
goldens); the reference coverage cases (DSPLIB_interleave_d.c, DSPLIB_deinterleave_d.c,
DSPLIB_addNCh_d.c coverage_test_main) on the C ABI.
GPU: the CUDA kernels through the C ABI, bit-exact against the golden outputs and the
oracle, device and host buffers, large and odd shapes.
"""
import ctypes
import os

import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "layout_golden.npz")
INT128 = 4  # DSPLIB_INT128


def _cases(prefix):
    d = np.load(GOLDEN)
    return sorted((k[:-5] for k in d if k.endswith("_meta") and k.startswith(prefix)), key=lambda k: int(k[1:]))


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


# ------------------------------------------------------------------ CPU: oracle pinning


def test_fixture_coverage(golden):
    kinds = {k[0] for k in golden if k.endswith("_meta")}
    assert kinds == {"i", "d", "a"}
    dts = {str(golden[k[:-5] + "_x"].dtype) for k in golden if k.endswith("_meta") and k[0] in "id"}
    assert dts == {"int8", "uint8", "int16", "uint16", "int32", "uint32", "int64", "uint64", "float32", "float64"}


@pytest.mark.parametrize("key", _cases("i") + _cases("d"))
def test_oracle_transpose_matches_golden(golden, key):
    _, W, H, s_in, s_out = (int(v) for v in golden[key + "_meta"])
    x, want = golden[key + "_x"], golden[key + "_y"]
    got = np.zeros_like(want)
    oracle.transpose(x, W, H, s_in, s_out, got)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("key", _cases("a"))
def test_oracle_addnch_matches_golden(golden, key):
    _, S, C, L, sY, sZ, sO = (int(v) for v in golden[key + "_meta"])
    x, want, g64 = golden[key + "_x"], golden[key + "_y"], golden[key + "_golden"]
    got = np.zeros_like(want)
    oracle.addnch(x, S, C, L, sY, sZ, sO, got)
    assert np.array_equal(got, want)  # the reference natural-C result, bit for bit
    # and the generator's float64 golden within the driver's 2^-10 (DSPLIB_addNCh_d.c:244-252)
    assert np.max(np.abs(got.reshape(C, sO)[:, :S] - g64)) <= 2.0 ** -10


# ------------------------------------------------------------------ CPU: API semantics


def _bp(t, x=16, y=16, stride=16):
    return D.bp(t, x, y, stride)


def test_interleave_coverage_cases():
    """DSPLIB_interleave_d.c coverage cases 1000-1006 (in 16 x 16, out dim_x 16, stride 16 bytes)."""
    L = D.lib()
    h = D.LayoutHandle("DSPLIB_interleave")
    a = D.StyleInitArgs(funcStyle=D.NATC)
    r = ctypes.byref
    chk = L.DSPLIB_interleave_init_checkParams
    assert chk(None, r(_bp(D.INT32)), r(_bp(D.INT32)), r(a)) == D.ERR_NULL_POINTER  # 1000
    assert chk(h.h, r(_bp(INT128)), r(_bp(D.INT32)), r(a)) == D.ERR_INVALID_TYPE  # 1001 / 1005
    assert chk(h.h, r(_bp(D.INT32)), r(_bp(D.INT16)), r(a)) == D.ERR_INVALID_TYPE  # 1002
    buf = (ctypes.c_char * 64)()
    assert L.DSPLIB_interleave_exec_checkParams(h.h, None, buf) == D.ERR_NULL_POINTER  # 1003
    assert L.DSPLIB_interleave_exec_checkParams(h.h, buf, None) == D.ERR_NULL_POINTER  # 1004
    assert chk(h.h, r(_bp(D.INT8, x=9)), r(_bp(D.INT8, x=9)), r(a)) == D.ERR_INVALID_VALUE  # 1006
    assert chk(h.h, r(_bp(D.INT16, x=9)), r(_bp(D.INT16, x=9)), r(a)) == D.ERR_INVALID_VALUE
    # two packed rows: only the type list applies (DSPLIB_interleave.cpp:42-44)
    assert chk(h.h, r(_bp(D.INT8, x=9, y=2)), r(_bp(D.INT8, x=2, y=9, stride=2)), r(a)) == D.SUCCESS
    # kept quirk: outside that case the second test's verdict replaces the type-list verdict
    assert chk(h.h, r(_bp(INT128)), r(_bp(INT128)), r(a)) == D.SUCCESS
    assert L.DSPLIB_interleave_init(h.h, r(_bp(INT128)), r(_bp(INT128)), r(a)) == D.ERR_INVALID_TYPE


def test_deinterleave_coverage_cases():
    L = D.lib()
    h = D.LayoutHandle("DSPLIB_deinterleave")
    r = ctypes.byref
    chk = L.DSPLIB_deinterleave_init_checkParams
    for style in (D.NATC, D.OPTIMIZED):
        a = D.StyleInitArgs(funcStyle=style)
        assert chk(None, r(_bp(D.INT32)), r(_bp(D.INT32)), r(a)) == D.ERR_NULL_POINTER  # 1000
        assert chk(h.h, r(_bp(INT128)), r(_bp(D.INT32)), r(a)) == D.ERR_INVALID_TYPE  # 1001
        assert chk(h.h, r(_bp(D.INT32)), r(_bp(D.INT16)), r(a)) == D.ERR_INVALID_TYPE  # 1002
        assert L.DSPLIB_deinterleave_init(h.h, r(_bp(INT128)), r(_bp(D.INT32)), r(a)) == D.ERR_INVALID_TYPE  # 1005
    buf = (ctypes.c_char * 64)()
    assert L.DSPLIB_deinterleave_exec_checkParams(h.h, None, buf) == D.ERR_NULL_POINTER  # 1003
    assert L.DSPLIB_deinterleave_exec_checkParams(h.h, buf, None) == D.ERR_NULL_POINTER  # 1004
    a = D.StyleInitArgs(funcStyle=D.NATC)
    assert chk(h.h, r(_bp(D.INT8, x=17)), r(_bp(D.INT8, x=17)), r(a)) == D.ERR_INVALID_VALUE  # 1006
    # one channel, or two packed channels, pass whatever the types (DSPLIB_deinterleave.cpp:30-33)
    assert chk(h.h, r(_bp(INT128, x=1)), r(_bp(D.INT32)), r(a)) == D.SUCCESS
    assert chk(h.h, r(_bp(D.INT32, x=2, stride=8)), r(_bp(D.INT8)), r(a)) == D.SUCCESS


def test_addnch_coverage_cases():
    L = D.lib()
    h = D.LayoutHandle("DSPLIB_addNCh")
    r = ctypes.byref

    def b3(t):
        return D.BufParams3D(t, 16, 16, 64, 16, 1024)

    chk = L.DSPLIB_addNCh_init_checkParams
    for style in (D.NATC, D.OPTIMIZED):
        a = D.StyleInitArgs(funcStyle=style)
        assert chk(None, r(b3(D.INT32)), r(_bp(D.INT32)), r(a)) == D.ERR_NULL_POINTER  # 1000
        assert chk(h.h, r(b3(INT128)), r(_bp(D.INT32)), r(a)) == D.ERR_INVALID_TYPE  # 1001
        assert chk(h.h, r(b3(D.FLOAT32)), r(_bp(D.INT16)), r(a)) == D.ERR_INVALID_TYPE  # 1002
        assert L.DSPLIB_addNCh_init(h.h, r(b3(D.INT64)), r(_bp(D.INT16)), r(a)) == D.ERR_INVALID_TYPE  # 1005
        assert chk(h.h, r(b3(D.FLOAT64)), r(_bp(D.FLOAT64)), r(a)) == D.SUCCESS
    buf = (ctypes.c_char * 64)()
    assert L.DSPLIB_addNCh_exec_checkParams(h.h, None, buf) == D.ERR_NULL_POINTER  # 1003
    assert L.DSPLIB_addNCh_exec_checkParams(h.h, buf, None) == D.ERR_NULL_POINTER  # 1004


def test_exec_without_init_fails():
    for prefix in ("DSPLIB_interleave", "DSPLIB_deinterleave", "DSPLIB_addNCh"):
        h = D.LayoutHandle(prefix)
        x = np.zeros(16, np.float32)
        assert h.exec(x, x) == D.ERR_FAILURE


# ------------------------------------------------------------------ GPU


def _torch():
    return pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.parametrize("style", [D.NATC, D.OPTIMIZED])
def test_transpose_golden_cases_on_device(golden, style):
    torch = _torch()
    for key in _cases("i") + _cases("d"):
        _, W, H, s_in, s_out = (int(v) for v in golden[key + "_meta"])
        x, want = golden[key + "_x"], golden[key + "_y"]
        # sentinel-filled output: bytes between the output rows must stay untouched
        xd = torch.from_numpy(x.view(np.uint8).copy()).cuda()
        yd = torch.full((want.nbytes,), 0xA5, dtype=torch.uint8, device="cuda")
        kind = "interleave" if key[0] == "i" else "deinterleave"
        D.transpose(_typed(torch, xd, x.dtype), _typed(torch, yd, want.dtype), W, H, s_in, s_out, kind=kind,
                    func_style=style)
        got = yd.cpu().numpy().view(want.dtype)
        ref = np.frombuffer(np.full(want.nbytes, 0xA5, np.uint8).tobytes(), want.dtype).copy()
        oracle.transpose(x, W, H, s_in, s_out, ref)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), key
        # the golden output's element positions
        mask = _written_mask(W, H, s_out, want.itemsize, want.size)
        assert np.array_equal(got[mask].view(np.uint8), want[mask].view(np.uint8)), key


def _typed(torch, t, dt):
    """A uint8 device tensor viewed as the numpy dtype's torch counterpart (same bytes)."""
    m = {np.dtype(np.int8): torch.int8, np.dtype(np.uint8): torch.uint8, np.dtype(np.int16): torch.int16,
         np.dtype(np.uint16): torch.uint16, np.dtype(np.int32): torch.int32, np.dtype(np.uint32): torch.uint32,
         np.dtype(np.int64): torch.int64, np.dtype(np.uint64): torch.uint64, np.dtype(np.float32): torch.float32,
         np.dtype(np.float64): torch.float64}
    return t.view(m[np.dtype(dt)])


def _written_mask(W, H, s_out, e, n):
    mask = np.zeros(n, bool)
    for i in range(W):
        o = (i * s_out) // e
        mask[o:o + H] = True
    return mask


@pytest.mark.gpu
def test_transpose_large_and_host_buffers():
    torch = _torch()
    rng = np.random.default_rng(3)
    # few-channel register kernels (2-4 channels, packed side) with ragged tails, and the tiled kernel
    for (W, H, dt) in [(2, 1 << 20, np.float32), (1 << 20, 2, np.int16), (3, 100003, np.int8),
                       (100003, 4, np.uint64), (4, 77777, np.float32), (77779, 3, np.int16), (2, 15, np.int8),
                       (8, 300001, np.float64), (3000, 3000, np.int8), (1, 4097, np.uint64), (4097, 1, np.int32),
                       (33, 65, np.uint16)]:
        e = np.dtype(dt).itemsize
        s_in, s_out = W * e, H * e
        x = rng.integers(0, 200, size=W * H).astype(dt)
        want = np.zeros(W * H, dt)
        oracle.transpose(x, W, H, s_in, s_out, want)
        got = _typed(torch, torch.zeros(W * H * e, dtype=torch.uint8, device="cuda"), dt)
        xd = _typed(torch, torch.from_numpy(x.view(np.uint8)).cuda(), dt)
        D.transpose(xd, got, W, H, s_in, s_out)
        assert np.array_equal(got.view(torch.uint8).cpu().numpy().view(dt), want), (W, H, dt)
        # pageable host buffers (staged)
        hy = np.zeros_like(want)
        D.transpose(x, hy, W, H, s_in, s_out, kind="deinterleave")
        assert np.array_equal(hy, want), (W, H, dt)


@pytest.mark.gpu
def test_async_level_one_completes_with_pinned_host_buffers():
    """DSPLIB_gpu_setAsync(h, 1) applies to device buffers only: page-locked host buffers,
    which the kernel reads and writes in place, hold the result when exec returns."""
    torch = _torch()
    rng = np.random.default_rng(8)
    W, H = 2, 1 << 21
    x = rng.standard_normal(W * H).astype(np.float32)
    want = np.zeros(W * H, np.float32)
    oracle.transpose(x, W, H, W * 4, H * 4, want)
    hx, hy = torch.from_numpy(x).pin_memory(), torch.zeros(W * H).pin_memory()
    h = D.LayoutHandle("DSPLIB_interleave")
    args = D.StyleInitArgs(funcStyle=D.OPTIMIZED)
    assert h.init(args, D.bp(D.FLOAT32, W, H, W * 4), D.bp(D.FLOAT32, H, W, H * 4)) == D.SUCCESS
    assert h.set_async(1) == D.SUCCESS
    assert h.exec(hx, hy) == D.SUCCESS
    assert np.array_equal(hy.numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("style", [D.NATC, D.OPTIMIZED])
def test_addnch_golden_cases_on_device(golden, style):
    torch = _torch()
    for key in _cases("a"):
        _, S, C, L, sY, sZ, sO = (int(v) for v in golden[key + "_meta"])
        x, want = golden[key + "_x"], golden[key + "_y"]
        yd = torch.zeros(want.size, dtype=torch.float32 if want.dtype == np.float32 else torch.float64, device="cuda")
        D.add_nch(torch.from_numpy(x).cuda(), yd, S, C, L, sY, sZ, sO, func_style=style)
        assert np.array_equal(yd.cpu().numpy(), want), key


@pytest.mark.gpu
def test_addnch_large_strided_and_host():
    torch = _torch()
    rng = np.random.default_rng(4)
    for dt in (np.float32, np.float64):
        S, C, L, sY, sO = 100003, 7, 12, 100040, 100016
        sZ = sY * C + 8
        x = rng.uniform(-10, 10, size=L * sZ).astype(dt)
        x[5] = -0.0  # 0 + (-0) is +0 in the reference's order of additions
        want = np.zeros(C * sO, dt)
        oracle.addnch(x, S, C, L, sY, sZ, sO, want)
        y = torch.zeros(C * sO, dtype=torch.float32 if dt == np.float32 else torch.float64, device="cuda")
        D.add_nch(torch.from_numpy(x).cuda(), y, S, C, L, sY, sZ, sO)
        assert np.array_equal(y.cpu().numpy().view(np.uint8), want.view(np.uint8))
        hy = np.zeros_like(want)
        D.add_nch(x, hy, S, C, L, sY, sZ, sO)
        assert np.array_equal(hy, want)
