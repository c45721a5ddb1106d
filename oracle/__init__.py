"""CPU oracle for the DSPLIB filtering path.  TEST INFRASTRUCTURE ONLY.

Two checkers live here, both loaded through ctypes:

* ``port``: this project's C restatement (``dsplib_oracle.c``), built into
  ``oracle/_build/liboracle_port.so`` by ``oracle/Makefile``.
* ``ref``: the reference's own natural-C kernels (``DSPLIB_fir_cn.cpp``,
  ``DSPLIB_cascadeBiquad_cn.cpp``, ``DSPLIB_fltoq15_cn.cpp``, ``DSPLIB_q15tofl_cn.cpp``,
  ``DSPLIB_matTrans_cn.cpp``, ``DSPLIB_addNCh_cn.cpp``)
  compiled unmodified, with the stand-in TI
  headers of ``oracle/shim``, into ``oracle/_ref/libdsplib_ref.so``.  Present
  whenever the library was built here (it travels with the repository
  snapshot) — it is optional; tests that need it skip when it is absent.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product library never does.

Parity status: the port is pinned against the reference ``_cn`` library and
against golden vectors generated by the reference's Python models
(``tests/golden/make_golden.py``).  Q-mode FIR has no reference counterpart in
the natural-C path; its restatement follows the MMA output-stage configuration
(``src/common/c7504/DSPLIB_configurations.cpp:94-160``) and is "parity
unpinned" by reference tests.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libdsplib_ref.so")

DT = {np.dtype(np.int8): 0, np.dtype(np.int16): 1, np.dtype(np.int32): 2, np.dtype(np.float32): 12}

_port = None
_ref = None


def build(ref_root: str | None = None) -> None:
    """Compile the checker libraries (port always; reference when its sources exist)."""
    args = ["make", "-s", "-C", HERE]
    if ref_root:
        args.append(f"REF={ref_root}")
    subprocess.run(args, check=True)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            build()
        _port = ctypes.CDLL(PORT_SO)
        for name in ("oracle_fir_cn", "oracle_fir_q", "oracle_fir_floatq", "oracle_fir_f64", "oracle_biquad_df",
                     "oracle_biquad_df_f64", "oracle_biquad_tif", "oracle_tif_coefficients", "oracle_fltoq15",
                     "oracle_q15tofl", "oracle_transpose", "oracle_addnch"):
            getattr(_port, name).restype = None
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        _ref = ctypes.CDLL(REF_SO)
    return _ref


# ------------------------------------------------------------------ FIR


def fir(x, h, T, *, nch, impl="port", threads=1):
    """Natural-C FIR with explicit tap count ``T``; ``h`` rows hold the stored
    taps (pitch = row length)."""
    x = np.ascontiguousarray(x)
    h = np.ascontiguousarray(h)
    batch, in_pitch = x.shape
    out_size = in_pitch - T + 1
    y = np.zeros((batch, out_size), dtype=x.dtype)
    fp = h.shape[1]
    if impl == "port":
        port().oracle_fir_cn(DT[x.dtype], _ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch, out_size,
                             fp if nch else 0)
    else:
        assert fp == T or not nch, "reference _cn derives the Nch tap pitch from T"
        lib = ref()
        if threads > 1:
            rc = lib.ref_fir_cn_mt(DT[x.dtype], _ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch,
                                   out_size, int(nch), 0, 0, int(threads))
        else:
            rc = lib.ref_fir_cn(DT[x.dtype], _ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch, out_size,
                                int(nch), 0, 0)
        assert rc == 0, rc
    return y


def fir_q(x, h, T, shift, *, nch):
    x = np.ascontiguousarray(x)
    h = np.ascontiguousarray(h)
    batch, in_pitch = x.shape
    out_size = in_pitch - T + 1
    y = np.zeros((batch, out_size), dtype=x.dtype)
    port().oracle_fir_q(DT[x.dtype], _ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch, out_size,
                        h.shape[1] if nch else 0, int(shift))
    return y


def fir_floatq(x, h, T, Q, *, nch):
    """FLOAT32 FIR in float Q mode (quantised to int32 at scale 2^Q, exact sums, rounding shift)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    h = np.ascontiguousarray(h, dtype=np.float32)
    batch, in_pitch = x.shape
    out_size = in_pitch - T + 1
    y = np.zeros((batch, out_size), dtype=np.float32)
    port().oracle_fir_floatq(_ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch, out_size,
                             h.shape[1] if nch else 0, int(Q))
    return y


def fir_f64(x, h, T, *, nch):
    x = np.ascontiguousarray(x, dtype=np.float32)
    h = np.ascontiguousarray(h, dtype=np.float32)
    batch, in_pitch = x.shape
    out_size = in_pitch - T + 1
    y = np.zeros((batch, out_size), dtype=np.float64)
    port().oracle_fir_f64(_ptr(x), _ptr(h), _ptr(y), batch, T, out_size, in_pitch, out_size,
                          h.shape[1] if nch else 0)
    return y


# --------------------------------------------------------------- biquad

FORM = {"TIF": 0, "DF1": 1, "DF2": 2, "TDF2": 3}


def nvars(form):
    return 4 if form == FORM["DF1"] else 2


def biquad(form, x, coef, state, *, nch, impl="port", threads=1):
    """Direct-form cascade over time-major ``x`` [N, C] (dense pitch C).
    ``coef`` natural [rows, S*5]; ``state`` [S*nv, C] is updated in place.
    ``impl='ref'`` runs the reference _cn kernel (TIF -> DF2, as NATC does)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    coef = np.ascontiguousarray(coef, dtype=np.float32)
    assert state.flags.c_contiguous and state.dtype == np.float32
    N, C = x.shape
    S = coef.shape[1] // 5
    y = np.zeros((N, C), dtype=np.float32)
    if impl == "port":
        port().oracle_biquad_df(int(form), _ptr(x), _ptr(coef), _ptr(state), _ptr(y), N, S, C, int(nch), C, C,
                                state.shape[1])
    else:
        lib = ref()
        if threads > 1:
            rc = lib.ref_biquad_cn_mt(int(form), _ptr(x), _ptr(coef), _ptr(state), _ptr(y), N, S, C, int(nch),
                                      C, C, state.shape[1], int(threads))
        else:
            rc = lib.ref_biquad_cn(int(form), _ptr(x), _ptr(coef), _ptr(state), _ptr(y), N, S, C, int(nch), C,
                                   C, state.shape[1])
        assert rc == 0, rc
    return y


def biquad_f64(form, x, coef, state64, *, nch):
    x = np.ascontiguousarray(x, dtype=np.float32)
    coef = np.ascontiguousarray(coef, dtype=np.float32)
    assert state64.flags.c_contiguous and state64.dtype == np.float64
    N, C = x.shape
    S = coef.shape[1] // 5
    y = np.zeros((N, C), dtype=np.float64)
    port().oracle_biquad_df_f64(int(form), _ptr(x), _ptr(coef), _ptr(state64), _ptr(y), N, S, C, int(nch), C,
                                C, state64.shape[1])
    return y


def tif_groups(S):
    return 1 if S <= 7 else (S + 6) // 7


def tif_coefficients(natural_row):
    """natural [S*5] -> (tifCoef [S*4], gains [G]) for one channel."""
    nat = np.ascontiguousarray(natural_row, dtype=np.float32)
    S = nat.size // 5
    tc = np.zeros(S * 4, dtype=np.float32)
    g = np.zeros(tif_groups(S), dtype=np.float32)
    port().oracle_tif_coefficients(_ptr(nat), S, _ptr(tc), _ptr(g))
    return tc, g


def biquad_tif(x, tif_coef, gains, state, *, nch):
    """TIF cascade; tif_coef [rows, S*4] storage order {c0,c1,-a2,-a1}, gains [rows, G]."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    tif_coef = np.ascontiguousarray(tif_coef, dtype=np.float32)
    gains = np.ascontiguousarray(gains, dtype=np.float32)
    N, C = x.shape
    S = tif_coef.shape[1] // 4
    y = np.zeros((N, C), dtype=np.float32)
    port().oracle_biquad_tif(_ptr(x), _ptr(tif_coef), _ptr(gains), _ptr(state), _ptr(y), N, S, C, int(nch), C, C,
                             state.shape[1])
    return y


# ------------------------------------------------------------------ Q.15 conversions

_FT = {np.dtype(np.float32): 12, np.dtype(np.float64): 13}


def fltoq15(x, *, style="natc", impl="port"):
    """Float (float32 / float64, 1-D) to Q.15 int16.  ``style``: "natc" (the natural-C
    steps, DSPLIB_fltoq15_cn.cpp:35-62) or "opt" (round half to even, saturate).
    ``impl='ref'`` runs the reference _cn kernel itself (natc only; inputs whose
    scaled value leaves the int32 range are undefined there)."""
    x = np.ascontiguousarray(x)
    out = np.zeros(x.size, np.int16)
    dt = _FT[x.dtype]
    if impl == "ref":
        if style != "natc":
            raise ValueError("the reference natural-C kernel has one style")
        rc = ref().ref_fltoq15_cn(dt, _ptr(x), _ptr(out), ctypes.c_int(x.size))
        if rc != 0:
            raise RuntimeError(f"ref_fltoq15_cn: {rc}")
    else:
        port().oracle_fltoq15(dt, 0 if style == "natc" else 1, _ptr(x), _ptr(out), ctypes.c_longlong(x.size))
    return out


def q15tofl(x, dtype=np.float32, *, impl="port"):
    """Q.15 int16 (1-D) to float32 / float64: x / 32768 (DSPLIB_q15tofl_cn.cpp:33-37)."""
    x = np.ascontiguousarray(x, dtype=np.int16)
    out = np.zeros(x.size, dtype)
    dt = _FT[np.dtype(dtype)]
    if impl == "ref":
        rc = ref().ref_q15tofl_cn(dt, _ptr(x), _ptr(out), ctypes.c_int(x.size))
        if rc != 0:
            raise RuntimeError(f"ref_q15tofl_cn: {rc}")
    else:
        port().oracle_q15tofl(dt, _ptr(x), _ptr(out), ctypes.c_longlong(x.size))
    return out


# ------------------------------------------------------------------ layout kernels

_LAYOUT_DT = {np.dtype(np.int8): 0, np.dtype(np.int16): 1, np.dtype(np.int32): 2, np.dtype(np.int64): 3,
              np.dtype(np.uint8): 5, np.dtype(np.uint16): 6, np.dtype(np.uint32): 8, np.dtype(np.uint64): 9,
              np.dtype(np.float32): 12, np.dtype(np.float64): 13}


def transpose(x, W, H, stride_in, stride_out, out, *, impl="port"):
    """The interleave / deinterleave transpose (DSPLIB_matTrans_cn.cpp:41-45) on flat
    buffers: ``x`` holds H rows of W elements ``stride_in`` bytes apart; ``out`` (updated in
    place, other bytes untouched) receives W rows of H elements at ``(i*stride_out)/size``."""
    x = np.ascontiguousarray(x)
    assert out.dtype == x.dtype and out.flags.c_contiguous
    if impl == "ref":
        rc = ref().ref_transpose_cn(_LAYOUT_DT[x.dtype], _ptr(x), _ptr(out), W, H, stride_in, stride_out)
        if rc != 0:
            raise RuntimeError(f"ref_transpose_cn: {rc}")
    else:
        port().oracle_transpose(x.itemsize, _ptr(x), _ptr(out), ctypes.c_longlong(W), ctypes.c_longlong(H),
                                ctypes.c_longlong(stride_in), ctypes.c_longlong(stride_out))
    return out


def addnch(x, samples, channels, inputs, sY, sZ, sO, out, *, impl="port"):
    """DSPLIB_addNCh on flat buffers (strides in elements); ``out`` updated in place."""
    x = np.ascontiguousarray(x)
    dt = _FT[x.dtype]
    if impl == "ref":
        rc = ref().ref_addnch_cn(dt, _ptr(x), _ptr(out), samples, channels, inputs, sY, sZ, sO)
        if rc != 0:
            raise RuntimeError(f"ref_addnch_cn: {rc}")
    else:
        L = ctypes.c_longlong
        port().oracle_addnch(dt, _ptr(x), _ptr(out), L(samples), L(channels), L(inputs), L(sY), L(sZ), L(sO))
    return out
