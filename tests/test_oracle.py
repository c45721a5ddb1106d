"""Pins the CPU oracle before it is trusted as the checker.

(1) Against golden vectors made by the reference's Python models
    (tests/golden/make_golden.py): abs tolerance 2^-10, the reference test
    drivers' own bound (test/DSPLIB_fir/DSPLIB_fir_d.c:315-317,
    test/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_d.c:391-405).
(2) Bit for bit against the reference's natural-C kernels compiled unmodified
    into oracle/_ref (skipped when that library was not built).
"""
import numpy as np
import pytest

import oracle
from conftest import case_keys

TOL = 2.0 ** -10


def _fir_golden_cases():
    d = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "fir_golden.npz"))
    return case_keys(d, "f") + case_keys(d, "i")


@pytest.mark.parametrize("key", _fir_golden_cases())
def test_fir_port_vs_golden(golden_fir, key):
    meta = golden_fir[key + "_meta"]
    x, h, yg = golden_fir[key + "_x"], golden_fir[key + "_h"], golden_fir[key + "_y"]
    T, nch = int(meta[2]), int(meta[4])
    y = oracle.fir(x, h, T, nch=nch)
    if x.dtype == np.float32:
        assert np.max(np.abs(y.astype(np.float64) - yg)) <= TOL
    else:
        assert np.array_equal(y, yg)  # integer wrap mode: exact


def _bq_cases():
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "biquad_golden.npz"))
    return case_keys(d, "b")


def _run_port(g, key):
    meta = g[key + "_meta"]
    form, nch, N, C, S, reps = (int(v) for v in meta[1:7])
    x = g[key + "_x"]
    if form == 0:
        st = np.zeros((2 * S, C), np.float32)
        y = oracle.biquad_tif(x, g[key + "_tif"], g[key + "_gain"], st, nch=nch)
    else:
        st = np.zeros((S * oracle.nvars(form), C), np.float32)
        y = oracle.biquad(form, x, g[key + "_coef"], st, nch=nch)
    return y, st


@pytest.mark.parametrize("key", _bq_cases())
def test_biquad_port_vs_golden(golden_biquad, key):
    y, st = _run_port(golden_biquad, key)
    # against the fp64 sosfilt golden, as the reference driver does
    assert np.max(np.abs(y - golden_biquad[key + "_y64"])) <= TOL
    # against the model's float32 form-exact recursion (tighter)
    assert np.max(np.abs(y - golden_biquad[key + "_y32"])) <= 1e-5


@pytest.mark.parametrize("key", [k for k in _bq_cases()])
def test_biquad_port_states_vs_model(golden_biquad, key):
    """Final filter states (the reference driver never checks these)."""
    meta = golden_biquad[key + "_meta"]
    form, nch, N, C, S = (int(v) for v in meta[1:6])
    y, st = _run_port(golden_biquad, key)
    zf = golden_biquad[key + "_zf32"]  # [S, nv, C] of the fp32 model
    nv = 4 if form == 1 else 2
    ref = zf.reshape(S * nv, C)
    assert np.max(np.abs(st - ref)) <= 1e-5


def test_tif_coefficients_vs_model(golden_biquad):
    for key in _bq_cases():
        meta = golden_biquad[key + "_meta"]
        if int(meta[1]) != 0:
            continue
        nat = golden_biquad[key + "_coef"]
        for row in range(nat.shape[0]):
            tc, gn = oracle.tif_coefficients(nat[row])
            assert np.allclose(tc, golden_biquad[key + "_tif"][row], rtol=1e-6, atol=1e-6)
            assert np.allclose(gn, golden_biquad[key + "_gain"][row], rtol=1e-6, atol=1e-7)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference _cn library not built")


@needs_ref
@pytest.mark.parametrize("dt", [np.int8, np.int16, np.int32, np.float32])
@pytest.mark.parametrize("nch", [0, 1])
def test_fir_port_bitexact_vs_reference_cn(dt, nch):
    rng = np.random.default_rng(7)
    for (B, N, T) in [(1, 17, 1), (3, 300, 37), (2, 1024, 256), (4, 64, 64)]:
        if dt == np.float32:
            x = rng.standard_normal((B, N)).astype(dt)
            h = rng.standard_normal((B if nch else 1, T)).astype(dt)
        else:
            info = np.iinfo(dt)
            x = rng.integers(info.min, info.max, size=(B, N), endpoint=True).astype(dt)
            h = rng.integers(info.min, info.max, size=(B if nch else 1, T), endpoint=True).astype(dt)
        assert np.array_equal(oracle.fir(x, h, T, nch=nch), oracle.fir(x, h, T, nch=nch, impl="ref"))


@needs_ref
@pytest.mark.parametrize("form", [1, 2, 3])
@pytest.mark.parametrize("nch", [0, 1])
def test_biquad_port_bitexact_vs_reference_cn(golden_biquad, form, nch):
    rng = np.random.default_rng(form * 10 + nch)
    for (N, C, S) in [(1, 1, 1), (64, 3, 2), (257, 17, 5)]:
        x = rng.standard_normal((N, C)).astype(np.float32)
        coef = (rng.standard_normal((C if nch else 1, S * 5)) * 0.3).astype(np.float32)
        st0 = rng.standard_normal((S * oracle.nvars(form), C)).astype(np.float32)
        s1, s2 = st0.copy(), st0.copy()
        y1 = oracle.biquad(form, x, coef, s1, nch=nch)
        y2 = oracle.biquad(form, x, coef, s2, nch=nch, impl="ref")
        assert np.array_equal(y1, y2) and np.array_equal(s1, s2)


def test_q_mode_rounding_and_saturation():
    """Q-mode output stage on hand-made accumulators (no reference counterpart)."""
    # x = [a], h = [1] -> acc = a; shift 2: (a + 2) >> 2 ; saturation to int8
    x = np.array([[5, 6, -5, -6, 127]], np.int8)
    h = np.array([[1]], np.int8)
    y = oracle.fir_q(x, h, 1, 2, nch=0)
    assert y.tolist() == [[(5 + 2) >> 2, (6 + 2) >> 2, (-5 + 2) >> 2, (-6 + 2) >> 2, (127 + 2) >> 2]]
    x = np.array([[100, -100]], np.int8)
    h = np.array([[100, 100]], np.int8)  # acc = 100*100 + (-100)*100 = 0 -> 0; single output
    assert oracle.fir_q(x, h, 2, 0, nch=0).tolist() == [[0]]
    x = np.array([[100, 100]], np.int8)
    assert oracle.fir_q(x, h, 2, 0, nch=0).tolist() == [[127]]
    assert oracle.fir_q(-x, h, 2, 0, nch=0).tolist() == [[-128]]


def test_float_q_mode_restatement_rules():
    """Float Q mode (no reference test covers it; restated from the C7x MMA path):
    x 2^Q and h 2^Q rounded to the nearest int32 (ties to even, saturating), exact sum,
    sum rounded half up and shifted by Q, saturated to int32, scaled back by 2^-Q."""
    Q = 2
    # taps [1.0] -> hq = 4; x values at scale 4: 0.125 -> 0.5 -> 0 (tie to even), 0.375 -> 1.5 -> 2,
    # 0.625 -> 2.5 -> 2, -0.375 -> -1.5 -> -2;  y = round_half_up(xq * 4 / 4) / 4 = xq / 4
    x = np.array([[0.125, 0.375, 0.625, -0.375, 1e12]], np.float32)
    h = np.array([[1.0]], np.float32)
    y = oracle.fir_floatq(x, h, 1, Q, nch=0)
    assert y[0, :4].tolist() == [0.0, 0.5, 0.5, -0.5]
    # 1e12 * 4 saturates to 2^31 - 1; times hq = 4, shifted by 2: 2^31 - 1 again; / 4
    assert y[0, 4] == np.float32(2147483647) / 4
    # sums wider than 64 bits stay exact: 4 products of (2^31 - 1)^2 at Q = 0
    x = np.full((1, 4), 3e9, np.float32)
    h = np.full((1, 4), 3e9, np.float32)
    assert oracle.fir_floatq(x, h, 4, 0, nch=0)[0, 0] == np.float32(2147483647)
