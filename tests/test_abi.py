"""C-ABI boundary tests that need no GPU: the library loads, exports every
entry point declared in include/*.h, and reproduces the reference's
parameter handling (status codes of the coverage cases in
test/DSPLIB_fir/DSPLIB_fir_d.c:434-602 and
test/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_d.c:504-781, sizes from
getSizes / get_coefficientsBufferDesc, and the host-side coefficient
transforms of get_coefficients)."""
import ctypes
import os
import re

import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
        for m in re.finditer(r"\b(DSPLIB_\w+)\s*\(", text):
            name = m.group(1)
            if name in ("DSPLIB_sizeof", "DSPLIB_min", "DSPLIB_max", "DSPLIB_ceilingDiv", "DSPLIB_ISSIGNED"):
                continue
            names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = D.lib()
    declared = _declared_functions()
    assert declared == sorted(D.SIGNATURES)  # 7 FIR + 8 biquad + the GPU extensions
    for name in declared:
        assert hasattr(L, name), name
        assert name in D.SIGNATURES, name


def test_handle_sizes():
    assert D.lib().DSPLIB_fir_getHandleSize(None) > 0
    assert D.lib().DSPLIB_cascadeBiquad_getHandleSize(None) > 0


def _fir_args(**kw):
    a = D.FirInitArgs(funcStyle=D.NATC, dataSize=16, batchSize=1, filterSize=4, shift=0, enableNchCoefs=0,
                      enableMMA=0, MMA_SIZE=D.MMA_SIZE[4], enableQ=0, Q=0)
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def test_fir_getsizes():
    args = _fir_args(dataSize=100, filterSize=7, batchSize=3, enableNchCoefs=1)
    pin, pf, po = D.bp(D.FLOAT32, 100, 3, 400), D.bp(D.FLOAT32, 7, 3, 28), D.bp(D.FLOAT32, 0, 3, 0)
    assert D.lib().DSPLIB_fir_getSizes(ctypes.byref(args), pin, pf, po) == D.SUCCESS
    assert po.dim_x == 94 and pf.dim_y == 3 and pf.dim_x == 7 and pf.stride_y == 28
    args.enableMMA = 1
    args.enableNchCoefs = 0
    assert D.lib().DSPLIB_fir_getSizes(ctypes.byref(args), pin, pf, po) == D.SUCCESS
    M = D.MMA_SIZE[4]
    assert pf.dim_y == 1 and pf.dim_x == 2 * M + 7 + M - 1 and pf.stride_y == pf.dim_x * 4
    pin.data_type = D.UINT64
    assert D.lib().DSPLIB_fir_getSizes(ctypes.byref(args), pin, pf, po) == D.ERR_NOT_IMPLEMENTED


def test_fir_coverage_cases():
    """Status codes of DSPLIB_fir_d.c coverage cases 1000-1010."""
    L = D.lib()
    h = D.FirHandle()
    args = _fir_args()
    pin, pf, po = D.bp(D.FLOAT32, 16, 1, 64), D.bp(D.FLOAT32, 4, 1, 16), D.bp(D.FLOAT32, 16, 1, 64)
    byref = ctypes.byref
    # 1000: NULL handle
    assert L.DSPLIB_fir_init_checkParams(None, byref(pin), byref(pf), byref(po), byref(args)) == D.ERR_NULL_POINTER
    # 1001: int16 in / int64 out: checkParams INVALID_TYPE, init NATC and OPT succeed, getSizes succeeds
    pin.data_type, po.data_type, pf.data_type = D.INT16, D.INT64, D.INT16
    assert h.init_check(args, pin, pf, po) == D.ERR_INVALID_TYPE
    args.funcStyle = D.NATC
    assert h.init(args, pin, pf, po) == D.SUCCESS
    args.funcStyle = D.OPTIMIZED
    assert h.init(args, pin, pf, po) == D.SUCCESS
    assert L.DSPLIB_fir_getSizes(byref(args), byref(pin), byref(pf), byref(po)) == D.SUCCESS
    # 1002: int32 in/out, int16 filter
    pin.data_type, po.data_type, pf.data_type = D.INT32, D.INT32, D.INT16
    assert h.init_check(args, pin, pf, po) == D.ERR_INVALID_TYPE
    for fs in (D.NATC, D.OPTIMIZED):
        args.funcStyle = fs
        assert h.init(args, pin, pf, po) == D.SUCCESS
    # 1003: int8 input
    pin.data_type = D.INT8
    assert h.init_check(args, pin, pf, po) == D.ERR_INVALID_TYPE
    for fs in (D.NATC, D.OPTIMIZED):
        args.funcStyle = fs
        assert h.init(args, pin, pf, po) == D.SUCCESS
    # 1004: uint64 input
    pin.data_type = D.UINT64
    assert h.init_check(args, pin, pf, po) == D.ERR_INVALID_TYPE
    for fs in (D.NATC, D.OPTIMIZED):
        args.funcStyle = fs
        assert h.init(args, pin, pf, po) == D.ERR_INVALID_TYPE
    assert L.DSPLIB_fir_getSizes(byref(args), byref(pin), byref(pf), byref(po)) == D.ERR_NOT_IMPLEMENTED
    # 1005-1007: exec_checkParams NULL buffers
    buf = np.zeros(16, np.float32)
    assert L.DSPLIB_fir_exec_checkParams(h.h, None, buf.ctypes.data, buf.ctypes.data) == D.ERR_NULL_POINTER
    assert L.DSPLIB_fir_exec_checkParams(h.h, buf.ctypes.data, None, buf.ctypes.data) == D.ERR_NULL_POINTER
    assert L.DSPLIB_fir_exec_checkParams(h.h, buf.ctypes.data, buf.ctypes.data, None) == D.ERR_NULL_POINTER
    assert L.DSPLIB_fir_exec_checkParams(h.h, buf.ctypes.data, buf.ctypes.data, buf.ctypes.data) == D.SUCCESS
    # 1008/1009: OPT float with empty output
    pin.data_type = D.FLOAT32
    args.funcStyle = D.OPTIMIZED
    args.dataSize, args.filterSize, po.dim_x = 0, 4, 0
    assert h.init(args, pin, pf, po) == D.SUCCESS
    args.dataSize, args.filterSize = 260, 2
    assert h.init(args, pin, pf, po) == D.SUCCESS
    # 1010: int16 everywhere: checkParams rejects (float-only), init accepts
    pin.data_type = po.data_type = pf.data_type = D.INT16
    assert h.init_check(args, pin, pf, po) == D.ERR_INVALID_TYPE
    for fs in (D.NATC, D.OPTIMIZED):
        args.funcStyle = fs
        assert h.init(args, pin, pf, po) == D.SUCCESS
    # float passes the check
    pin.data_type = po.data_type = pf.data_type = D.FLOAT32
    assert h.init_check(args, pin, pf, po) == D.SUCCESS


def _bq_setup(C=2, N=32, S=1, form=D.TIF, nch=0):
    args = D.BiquadInitArgs(funcStyle=D.OPTIMIZED, dataSize=N, numStages=S, numChannels=C, enableNChCoeffs=nch,
                            biquadForm=form)
    pin, pout = D.bp(D.FLOAT32, C, N, 16), D.bp(D.FLOAT32, C, N, 16)
    pvar = D.bp(D.FLOAT32, C, S * 2, 16)
    pcn = D.bp(D.FLOAT32, S * 5, C if nch else 1, S * 20)
    popt = D.BufParams2D()
    D.lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(D.FLOAT32, S, C, form, nch, ctypes.byref(popt))
    return args, pin, pout, pvar, pcn, popt


def test_biquad_coverage_cases():
    """Status codes of DSPLIB_cascadeBiquad_d.c coverage cases 1000-1016 (without the exec of 1008)."""
    L = D.lib()
    h = D.BiquadHandle()
    args, pin, pout, pvar, pcn, popt = _bq_setup()
    byref = ctypes.byref
    assert L.DSPLIB_cascadeBiquad_init_checkParams(None, byref(pin), byref(popt), byref(pvar), byref(pout),
                                                   byref(args)) == D.ERR_NULL_POINTER  # 1000
    pin.data_type = pout.data_type = popt.data_type = D.INT64  # 1001
    args.funcStyle = D.NATC
    assert h.init_check(args, pin, pcn, pvar, pout) == D.ERR_INVALID_TYPE
    assert h.init(args, pin, pcn, pvar, pout) == D.ERR_INVALID_TYPE
    args.funcStyle = D.OPTIMIZED
    assert h.init(args, pin, popt, pvar, pout) == D.ERR_INVALID_TYPE
    pin.data_type = D.FLOAT32  # 1002
    assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_INVALID_TYPE
    pout.data_type = D.FLOAT32  # 1003
    assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_INVALID_TYPE
    buf = np.zeros(64, np.float32).ctypes.data
    for i in range(4):  # 1004-1007
        ptrs = [buf] * 4
        ptrs[i] = None
        assert L.DSPLIB_cascadeBiquad_exec_checkParams(h.h, *ptrs) == D.ERR_NULL_POINTER
    popt.data_type = pvar.data_type = D.FLOAT32  # 1008 setup: NATC init succeeds
    args.numStages, args.funcStyle = 1, D.NATC
    assert h.init_check(args, pin, pcn, pvar, pout) == D.SUCCESS
    assert h.init(args, pin, pcn, pvar, pout) == D.SUCCESS
    for dt in (D.INT8, D.INT16, D.INT32):  # 1009-1011
        pin.data_type = pout.data_type = popt.data_type = dt
        assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_INVALID_TYPE
    pin.data_type = pout.data_type = popt.data_type = D.FLOAT32
    args.funcStyle = D.OPTIMIZED
    for S in (7, 3):  # 1012-1013: zero channels
        args.numStages, args.numChannels = S, 0
        assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_INVALID_VALUE
    args.numStages, args.numChannels, args.enableNChCoeffs = 3, 8, 2  # 1014
    assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_INVALID_VALUE
    args.enableNChCoeffs = 0
    pout.stride_y = 2 * pin.stride_y  # 1015, 1016: in/out pitch mismatch
    assert h.init_check(args, pin, popt, pvar, pout) == D.ERR_NOT_IMPLEMENTED
    assert h.init(args, pin, popt, pvar, pout) == D.ERR_NOT_IMPLEMENTED


@pytest.mark.parametrize("form", [D.TIF, D.DF1, D.DF2, D.TDF2])
@pytest.mark.parametrize("nch", [0, 1])
@pytest.mark.parametrize("S", [1, 7, 8, 13])
def test_coefficient_buffer_desc(form, nch, S):
    C = 17
    popt = D.BufParams2D()
    assert D.lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(D.FLOAT32, S, C, form, nch,
                                                                   ctypes.byref(popt)) == D.SUCCESS
    G = 1 if S <= 7 else (S + 6) // 7
    if form == D.TIF:
        want = (4 * S + G, 1) if not nch else (C, 4 * S + G)
    else:
        want = (5 * S, 1) if not nch else (C, 5 * S)
    assert (popt.dim_x, popt.dim_y) == want
    if nch:
        assert popt.stride_y == 24 * 4  # channels padded to a multiple of 8
    else:
        assert popt.stride_y == popt.dim_x * 4
    assert D.lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(D.INT16, S, C, form, nch,
                                                                   ctypes.byref(popt)) == D.ERR_INVALID_TYPE
    assert D.lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(D.FLOAT32, S, C, 4, nch,
                                                                   ctypes.byref(popt)) == D.ERR_INVALID_VALUE


@pytest.mark.parametrize("S", [1, 3, 7, 8, 9, 13])
@pytest.mark.parametrize("nch", [0, 1])
def test_get_coefficients_tif_matches_oracle(S, nch):
    C = 11
    rng = np.random.default_rng(S * 3 + nch)
    nat = rng.uniform(-0.9, 0.9, size=(C if nch else 1, S * 5)).astype(np.float32)
    nat[:, 0::5] = rng.uniform(0.2, 1.5, size=(nat.shape[0], S)).astype(np.float32)
    opt, popt = D.opt_coefficients(nat, D.TIF, nch, C)
    G = oracle.tif_groups(S)
    for row in range(nat.shape[0]):
        tc, gn = oracle.tif_coefficients(nat[row])
        if not nch:
            np.testing.assert_array_equal(opt[: 4 * S], tc)
            np.testing.assert_array_equal(opt[4 * S: 4 * S + G], gn)
        else:
            pitch = popt.stride_y // 4
            m = opt.reshape(-1, pitch)
            got = np.stack([m[k * S + s, row] for s in range(S) for k in range(4)])
            np.testing.assert_array_equal(got, tc)
            np.testing.assert_array_equal(m[4 * S: 4 * S + G, row], gn)


@pytest.mark.parametrize("form", [D.DF1, D.DF2, D.TDF2])
def test_get_coefficients_df_reorder(form):
    C, S = 13, 4
    nat = np.arange(C * S * 5, dtype=np.float32).reshape(C, S * 5)
    opt, popt = D.opt_coefficients(nat, form, 1, C)
    m = opt.reshape(-1, popt.stride_y // 4)
    np.testing.assert_array_equal(m[: S * 5, :C], nat.T)
    # shared DF coefficients need no transform: the reference reports INVALID_VALUE
    pcn = D.bp(D.FLOAT32, S * 5, 1, S * 20)
    p2 = D.BufParams2D()
    D.lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(D.FLOAT32, S, C, form, 0, ctypes.byref(p2))
    out = np.zeros(S * 5, np.float32)
    assert D.lib().DSPLIB_cascadeBiquad_get_coefficients(form, 0, ctypes.byref(pcn), ctypes.byref(p2),
                                                         nat.ctypes.data, out.ctypes.data) == D.ERR_INVALID_VALUE
    bad = D.bp(D.FLOAT32, S * 5 + 1, C, 0)
    assert D.lib().DSPLIB_cascadeBiquad_get_coefficients(D.TIF, 0, ctypes.byref(bad), ctypes.byref(p2),
                                                         nat.ctypes.data, out.ctypes.data) == D.ERR_NOT_ALIGNED_WIDTHS


def test_exec_without_init_fails_cleanly():
    h = D.FirHandle()
    x = np.zeros(8, np.float32)
    assert h.exec(x, x, x) == D.ERR_FAILURE
    b = D.BiquadHandle()
    assert b.exec(x, x, x, x) == D.ERR_FAILURE


def test_release_handle():
    """DSPLIB_gpu_releaseHandle ends a handle's life: later calls on it fail as on an uninitialised handle."""
    args, pin, pf, po = D.fir_setup(D.FLOAT32, 2, 64, 8, nch=0)
    h = D.FirHandle()
    assert h.init(args, pin, pf, po) == D.SUCCESS
    assert D.lib().DSPLIB_gpu_releaseHandle(h.h) == D.SUCCESS
    assert D.lib().DSPLIB_gpu_releaseHandle(h.h) == D.ERR_NULL_POINTER
    assert D.lib().DSPLIB_gpu_setAsync(h.h, 1) == D.ERR_NULL_POINTER
    x = np.zeros(8, np.float32)
    assert h.exec(x, x, x) == D.ERR_FAILURE
    assert D.lib().DSPLIB_gpu_releaseHandle(None) == D.ERR_NULL_POINTER


def test_stream_and_async_settings_apply_after_init_and_persist():
    """DSPLIB_gpu_setStream / setAsync need an initialised handle (NULL_POINTER before the
    first init); every async level is accepted afterwards and a later init keeps it."""
    args, pin, pout, pvar, _, popt = D.biquad_descs(32, 64, 2, D.DF2, 0)
    h = D.BiquadHandle()
    assert h.set_async(2) == D.ERR_NULL_POINTER
    assert h.set_stream(None) == D.ERR_NULL_POINTER
    assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
    for level in (0, 1, 2, True, False):
        assert h.set_async(level) == D.SUCCESS
    assert h.set_stream(None) == D.SUCCESS
    assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS  # re-init keeps the handle's settings
    assert h.set_async(2) == D.SUCCESS
