"""DSPLIB_fltoq15 / DSPLIB_q15tofl: the Q.15 conversions around the integer FIR path.

CPU: the C restatement against the reference's own natural-C kernels
(oracle/_ref) on the reference test distribution (test/DSPLIB_fltoq15/
DSPLIB_fltoq15_idat.c: RANDOM, uniform in [-1, 1) from test/common/
TI_memory.c:2517-2540, at the sizes of its 38 cases) and on every rounding edge;
the reference coverage cases 1000-1007 (DSPLIB_fltoq15_d.c:342-430,
DSPLIB_q15tofl_d.c coverage_test_main) on the C ABI.
GPU: the CUDA kernels through the C ABI, bit-exact against the oracle, for both
function styles, both float types, device / pageable / page-locked host buffers,
unaligned pointers and ragged lengths.
"""
import ctypes

import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle

# dataSize of the reference's fltoq15 / q15tofl test cases (DSPLIB_fltoq15_idat.c)
REF_SIZES = [1, 16, 64, 129, 287, 512, 1021, 1152, 2046, 4096, 8190, 16384, 32768, 51200, 51201, 1024, 2048,
             5, 10, 15, 25, 31, 3, 7, 11]


def _edges(ftype):
    """Scaled values on every rounding boundary of the conversion, divided by 32768."""
    f = np.dtype(ftype).type
    half_below = np.nextafter(f(0.5), f(0))  # 0.5 - 2^-25 (float) / 0.5 - 2^-54 (double)
    m = [0.0, -0.0, 0.5, -0.5, 1.5, -1.5, 2.5, -2.5, 3.5, -3.5, half_below, -half_below,
         np.nextafter(f(1.5), f(2)), np.nextafter(f(2.5), f(2)), 100.49, -100.51, 32766.5, 32767.5, -32767.5,
         -32768.5, 32767.49, 40000.0, -40000.0, 65535.9, -65535.9, 1e6, -1e6, 2.0000152587890 * 32768]
    return (np.array(m, dtype=ftype) / f(32768)).astype(ftype)


def _random(rng, n, ftype):
    return ((rng.random(n) * 2.0 - 1.0)).astype(ftype)


# ------------------------------------------------------------------ CPU: oracle pinning


@pytest.mark.parametrize("ftype", [np.float32, np.float64])
def test_oracle_fltoq15_matches_reference_cn(ftype):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(15)
    for n in REF_SIZES:
        x = _random(rng, n, ftype)
        assert np.array_equal(oracle.fltoq15(x), oracle.fltoq15(x, impl="ref")), n
    e = _edges(ftype)
    assert np.array_equal(oracle.fltoq15(e), oracle.fltoq15(e, impl="ref"))


def test_oracle_fltoq15_styles_differ_only_at_the_half_ulp_input():
    """The natural-C code adds 0.5 in the input precision: for the largest value below
    0.5 (scaled) that sum rounds up to 1.0, so NATC gives +-1 where round-half-even gives 0."""
    for ftype in (np.float32, np.float64):
        e = _edges(ftype)
        a, b = oracle.fltoq15(e, style="natc"), oracle.fltoq15(e, style="opt")
        diff = np.flatnonzero(a != b)
        assert list(diff) == [10, 11], (ftype, diff)
        assert list(a[diff]) == [1, -1] and list(b[diff]) == [0, 0]
        # ties to even, saturation
        assert list(b[2:10]) == [0, 0, 2, -2, 2, -2, 4, -4]
        assert b[17] == 32767 and b[19] == -32768 and b[-1] == 32767


def test_oracle_q15tofl_matches_reference_cn():
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    q = np.arange(-32768, 32768, dtype=np.int32).astype(np.int16)
    for ftype in (np.float32, np.float64):
        got = oracle.q15tofl(q, ftype)
        assert np.array_equal(got, oracle.q15tofl(q, ftype, impl="ref"))
        assert np.array_equal(got, (q.astype(np.float64) / 32768.0).astype(ftype))


# ------------------------------------------------------------------ CPU: API semantics


INT128 = 4  # DSPLIB_INT128


def _buf1d(t, n=16):
    return D.BufParams1D(t, n)


@pytest.mark.parametrize("H", [D.Fltoq15Handle, D.Q15toflHandle])
def test_coverage_cases(H):
    """Coverage cases 1000-1006 of both reference drivers."""
    L = D.lib()
    pre = H.prefix
    h = H()
    a = D.ConvertInitArgs(funcStyle=D.NATC, dataSize=16)
    check = getattr(L, pre + "_init_checkParams")
    init = getattr(L, pre + "_init")
    ref = ctypes.byref
    for style in (D.NATC, D.OPTIMIZED):
        a.funcStyle = style
        assert check(None, ref(_buf1d(D.INT32)), ref(_buf1d(D.INT32)), ref(a)) == D.ERR_NULL_POINTER  # 1000
        assert check(h.h, ref(_buf1d(INT128)), ref(_buf1d(D.INT32)), ref(a)) == D.ERR_INVALID_TYPE  # 1001
        assert check(h.h, ref(_buf1d(D.INT32)), ref(_buf1d(D.INT16)), ref(a)) == D.ERR_INVALID_TYPE  # 1002
        assert init(h.h, ref(_buf1d(INT128)), ref(_buf1d(D.INT32)), ref(a)) == D.ERR_INVALID_TYPE  # 1005
    execc = getattr(L, pre + "_exec_checkParams")
    buf = (ctypes.c_char * 64)()
    assert execc(h.h, None, buf) == D.ERR_NULL_POINTER  # 1003
    assert execc(h.h, buf, None) == D.ERR_NULL_POINTER  # 1004
    assert execc(h.h, buf, buf) == D.SUCCESS
    if H is D.Fltoq15Handle:  # 1006: float in, INT32 out
        assert check(h.h, ref(_buf1d(D.FLOAT32)), ref(_buf1d(D.INT32)), ref(a)) == D.ERR_INVALID_TYPE
        assert check(h.h, ref(_buf1d(D.FLOAT64)), ref(_buf1d(D.INT16)), ref(a)) == D.SUCCESS
    else:  # 1006: INT16 in, INT32 out
        assert check(h.h, ref(_buf1d(D.INT16)), ref(_buf1d(D.INT32)), ref(a)) == D.ERR_INVALID_TYPE
        assert check(h.h, ref(_buf1d(D.INT16)), ref(_buf1d(D.FLOAT64)), ref(a)) == D.SUCCESS


def test_exec_without_init_fails():
    h = D.Fltoq15Handle()
    x = np.zeros(8, np.float32)
    y = np.zeros(8, np.int16)
    assert h.exec(x, y) == D.ERR_FAILURE


# ------------------------------------------------------------------ GPU


def _torch():
    return pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.parametrize("ftype", [np.float32, np.float64])
@pytest.mark.parametrize("style", [D.NATC, D.OPTIMIZED])
def test_fltoq15_device_bitexact(ftype, style):
    torch = _torch()
    rng = np.random.default_rng(7)
    want_style = "natc" if style == D.NATC else "opt"
    for n in REF_SIZES + [1 << 20, (1 << 20) + 5]:
        x = _random(rng, n, ftype)
        got = D.fltoq15(torch.from_numpy(x).cuda(), func_style=style).cpu().numpy()
        assert np.array_equal(got, oracle.fltoq15(x, style=want_style)), n
    # rounding edges, saturation, infinities and NaN (the oracle saturates by sign, NaN -> 0)
    e = np.concatenate([_edges(ftype), np.array([np.inf, -np.inf, np.nan, 3e9, -3e9], ftype)])
    got = D.fltoq15(torch.from_numpy(e).cuda(), func_style=style).cpu().numpy()
    assert np.array_equal(got, oracle.fltoq15(e, style=want_style))


@pytest.mark.gpu
@pytest.mark.parametrize("ftype", [np.float32, np.float64])
def test_fltoq15_unaligned_and_host_buffers(ftype):
    torch = _torch()
    rng = np.random.default_rng(8)
    x = _random(rng, 100003, ftype)
    want = oracle.fltoq15(x)
    xd = torch.from_numpy(np.concatenate([np.zeros(3, ftype), x])).cuda()
    yd = torch.zeros(100003 + 1, dtype=torch.int16, device="cuda")
    D.fltoq15(xd[3:], func_style=D.NATC, out=yd[1:])  # neither pointer 16-byte aligned
    assert np.array_equal(yd[1:].cpu().numpy(), want)
    # pageable host memory, small (one staged call) and large (pipelined blocks)
    assert np.array_equal(D.fltoq15(x, func_style=D.NATC), want)
    big = _random(rng, 3_000_001, ftype)
    assert np.array_equal(D.fltoq15(big, func_style=D.NATC), oracle.fltoq15(big))
    # page-locked host memory, read and written by the kernel in place
    xp = torch.from_numpy(big).pin_memory()
    yp = torch.zeros(big.size, dtype=torch.int16).pin_memory()
    D.fltoq15(xp, func_style=D.NATC, out=yp)
    assert np.array_equal(yp.numpy(), oracle.fltoq15(big))


@pytest.mark.gpu
@pytest.mark.parametrize("ftype", [np.float32, np.float64])
def test_q15tofl_all_values(ftype):
    torch = _torch()
    q = np.tile(np.arange(-32768, 32768, dtype=np.int32).astype(np.int16), 3)
    want = oracle.q15tofl(q, ftype)
    for style in (D.NATC, D.OPTIMIZED):
        got = D.q15tofl(torch.from_numpy(q).cuda(), ftype, func_style=style).cpu().numpy()
        assert np.array_equal(got, want)
    # unaligned device pointers, ragged length
    qd = torch.from_numpy(q).cuda()
    out = torch.zeros(q.size, dtype=torch.float32 if ftype == np.float32 else torch.float64, device="cuda")
    D.q15tofl(qd[1:-2], ftype, out=out[3:q.size])
    assert np.array_equal(out[3:q.size].cpu().numpy(), want[1:-2])
    # pageable and page-locked host buffers
    assert np.array_equal(D.q15tofl(q, ftype), want)
    big = np.random.default_rng(9).integers(-32768, 32768, 5_000_000).astype(np.int16)
    assert np.array_equal(D.q15tofl(big, ftype), oracle.q15tofl(big, ftype))
    qp = torch.from_numpy(big).pin_memory()
    op = torch.zeros(big.size, dtype=out.dtype).pin_memory()
    D.q15tofl(qp, ftype, out=op)
    assert np.array_equal(op.numpy(), oracle.q15tofl(big, ftype))


@pytest.mark.gpu
def test_coverage_case_1007_runs():
    """DSPLIB_fltoq15_d.c:402-425: eight values -0.2 i with the last one 2.0000152587890."""
    x = np.array([-0.2 * i for i in range(8)], np.float32)
    x[7] = np.float32(2.0000152587890)
    got = D.fltoq15(x, func_style=D.NATC)
    assert np.array_equal(got, oracle.fltoq15(x))
    assert got[7] == 32767


@pytest.mark.gpu
def test_round_trip_q15():
    """q15tofl then fltoq15 is the identity on every Q.15 value, for both styles."""
    torch = _torch()
    q = torch.arange(-32768, 32768, dtype=torch.int32).to(torch.int16).cuda()
    for ftype in (np.float32, np.float64):
        f = D.q15tofl(q, ftype)
        for style in (D.NATC, D.OPTIMIZED):
            assert torch.equal(D.fltoq15(f, func_style=style), q)
