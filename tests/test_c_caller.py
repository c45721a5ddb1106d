"""The drop-in from C: tests/c_caller/dsplib_caller.c, compiled with gcc against include/
only and linked to libdsplib_b200.so, replays the reference test drivers' call
sequences (FIR: DSPLIB_fir_d.c:101-305; cascade biquad: DSPLIB_cascadeBiquad_d.c:123-343)
on host buffers.  Its outputs are checked against the reference's own natural-C kernels
(oracle/_ref; the restatement when that library is absent): natural-C calls bit for bit,
optimized calls to the tolerances of the other tests."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_caller", "dsplib_caller.c")
LIBDIR = os.path.join(ROOT, "c7x_dsplib_b200")


def _compile(outdir):
    if not os.path.exists(os.path.join(LIBDIR, "libdsplib_b200.so")):
        pytest.skip("library not built")
    gcc = shutil.which("gcc") or "gcc"
    exe = os.path.join(outdir, "dsplib_caller")
    cmd = [gcc, "-std=c11", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIBDIR, "-ldsplib_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_c_caller_compiles_against_the_public_headers(tmp_path):
    exe = _compile(str(tmp_path))
    assert os.path.exists(exe)


def _load(d, name, dtype, shape):
    return np.fromfile(os.path.join(d, name + ".bin"), dtype=dtype).reshape(shape)


def _impl():
    return "ref" if oracle.ref_available() else "port"


@pytest.mark.gpu
def test_c_caller_results(tmp_path):
    import c7x_dsplib_b200 as D

    d = str(tmp_path)
    exe = _compile(d)
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    impl = _impl()
    # FIR FLOAT32, per-channel taps: natural C bit-exact, optimized within 2e-6 of each channel's peak
    B, N, T = 3, 1000, 37
    x, h = _load(d, "fir_f32_x", np.float32, (B, N)), _load(d, "fir_f32_h", np.float32, (B, T))
    natc, opt = _load(d, "fir_f32_natc", np.float32, (B, N - T + 1)), _load(d, "fir_f32_opt", np.float32,
                                                                           (B, N - T + 1))
    assert np.array_equal(natc, oracle.fir(x, h, T, nch=1, impl=impl))
    w = oracle.fir_f64(x, h, T, nch=1)
    assert np.all(np.abs(opt - w).max(axis=1) <= 2e-6 * np.abs(w).max(axis=1))
    # the MMA filter layout
    B, N, T = 2, 700, 20
    x, h = _load(d, "fir_mma_x", np.float32, (B, N)), _load(d, "fir_mma_h", np.float32, (B, T))
    opt = _load(d, "fir_mma_opt", np.float32, (B, N - T + 1))
    w = oracle.fir_f64(x, h, T, nch=1)
    assert np.all(np.abs(opt - w).max(axis=1) <= 2e-6 * np.abs(w).max(axis=1))
    # INT16 natural C (wraps modulo 2^16)
    B, N, T = 4, 512, 64
    x, h = _load(d, "fir_i16_x", np.int16, (B, N)), _load(d, "fir_i16_h", np.int16, (1, T))
    assert np.array_equal(_load(d, "fir_i16_natc", np.int16, (B, N - T + 1)), oracle.fir(x, h, T, nch=0, impl=impl))
    # cascade biquad: (tag, form, natc, per-channel, C, N per block, S, blocks)
    cases = [("df2_natc", D.DF2, True, 0, 8, 500, 3, 2), ("df1_natc_nch", D.DF1, True, 1, 5, 300, 2, 1),
             ("df2_opt_nch", D.DF2, False, 1, 40, 4000, 4, 2), ("tdf2_opt_nch", D.TDF2, False, 1, 17, 600, 3, 1),
             ("tif_opt", D.TIF, False, 0, 33, 2000, 9, 2)]
    for tag, form, natc, nch, C, N, S, blocks in cases:
        nv = 4 if form == D.DF1 else 2
        x = _load(d, f"bq_{tag}_x", np.float32, (blocks * N, C))
        nat = _load(d, f"bq_{tag}_nat", np.float32, (C if nch else 1, 5 * S))
        y = _load(d, f"bq_{tag}_y", np.float32, (blocks * N, C))
        var = _load(d, f"bq_{tag}_var", np.float32, (S * nv, C))
        if natc:
            st = np.zeros((S * nv, C), np.float32)
            want = oracle.biquad(form, x, nat, st, nch=nch, impl=impl)
            assert np.array_equal(y, want), tag
            assert np.array_equal(var, st), tag
        else:
            s64 = np.zeros((S * 2, C), np.float64)
            y64 = oracle.biquad_f64(D.DF2 if form == D.TIF else form, x, nat, s64, nch=nch)
            rel = np.abs(y.astype(np.float64) - y64).max(axis=0) / np.abs(y64).max(axis=0)
            assert rel.max() <= 1e-4, (tag, rel.max())
