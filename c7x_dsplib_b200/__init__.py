"""B200-native DSPLIB filtering path: DSPLIB_fir and DSPLIB_cascadeBiquad.

The product is the C-ABI shared library ``libdsplib_b200.so`` built from
``csrc/`` (``python -m c7x_dsplib_b200.build``); its entry points are declared
in ``include/DSPLIB_fir.h``, ``include/DSPLIB_cascadeBiquad.h`` and
``include/dsplib_gpu.h``.  This module is the Python binding of that C ABI:

* ``lib()`` returns the loaded ``ctypes.CDLL`` with argument types set;
* ``FirHandle`` / ``BiquadHandle`` mirror the reference call sequence
  (getHandleSize -> init_checkParams -> init -> exec_checkParams -> exec);
* ``fir()`` / ``cascade_biquad()`` run one call on numpy arrays (host
  buffers, staged by the library) or torch CUDA tensors (device buffers).

There is no CPU implementation here: if the library is missing or no CUDA
device is present, calls fail with an error.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libdsplib_b200.so")

# DSPLIB_STATUS (include/DSPLIB_types.h)
SUCCESS = 0
ERR_FAILURE = 1
ERR_INVALID_VALUE = 2
ERR_INVALID_TYPE = 3
ERR_INVALID_DIMENSION = 4
ERR_NULL_POINTER = 5
ERR_NOT_IMPLEMENTED = 6
ERR_NOT_ALIGNED_WIDTHS = 9
ERR_BUFFER_TOO_SMALL = 10

# DSPLIB_data_type_e (include/DSPLIB_bufParams.h)
INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64 = 0, 1, 2, 3, 5, 6, 8, 9, 12, 13
NATC, OPTIMIZED = 0, 1
TIF, DF1, DF2, TDF2 = 0, 1, 2, 3
FIR_SIMT, FIR_BF16X3 = 0, 1
MMA_SIZE = {1: 32, 2: 16, 4: 8}  # DSPLIB_MMA_SIZE_{8,16,32}_BIT

_NP2DT = {np.dtype(np.int8): INT8, np.dtype(np.int16): INT16, np.dtype(np.int32): INT32,
          np.dtype(np.float32): FLOAT32}


class BufParams2D(ctypes.Structure):
    _fields_ = [("data_type", ctypes.c_uint32), ("dim_x", ctypes.c_uint32), ("dim_y", ctypes.c_uint32),
                ("stride_y", ctypes.c_int32)]


class FirInitArgs(ctypes.Structure):
    _fields_ = [("funcStyle", ctypes.c_int8), ("dataSize", ctypes.c_int32), ("batchSize", ctypes.c_int32),
                ("filterSize", ctypes.c_int32), ("shift", ctypes.c_uint32), ("enableNchCoefs", ctypes.c_uint32),
                ("enableMMA", ctypes.c_uint32), ("MMA_SIZE", ctypes.c_int32), ("enableQ", ctypes.c_uint32),
                ("Q", ctypes.c_uint32)]


class BiquadInitArgs(ctypes.Structure):
    _fields_ = [("funcStyle", ctypes.c_int8), ("dataSize", ctypes.c_uint32), ("numStages", ctypes.c_uint32),
                ("numChannels", ctypes.c_uint32), ("enableNChCoeffs", ctypes.c_uint32),
                ("biquadForm", ctypes.c_uint32)]


class BufParams1D(ctypes.Structure):
    _fields_ = [("data_type", ctypes.c_uint32), ("dim_x", ctypes.c_uint32)]


class BufParams3D(ctypes.Structure):
    _fields_ = [("data_type", ctypes.c_uint32), ("dim_x", ctypes.c_uint32), ("dim_y", ctypes.c_uint32),
                ("stride_y", ctypes.c_int32), ("dim_z", ctypes.c_uint32), ("stride_z", ctypes.c_int32)]


class StyleInitArgs(ctypes.Structure):
    """DSPLIB_interleaveInitArgs, DSPLIB_deinterleaveInitArgs, DSPLIB_addNCh_InitArgs."""
    _fields_ = [("funcStyle", ctypes.c_int8)]


class ConvertInitArgs(ctypes.Structure):
    """DSPLIB_fltoq15_InitArgs and DSPLIB_q15tofl_InitArgs (same layout)."""
    _fields_ = [("funcStyle", ctypes.c_int8), ("dataSize", ctypes.c_uint32)]


_lib = None
_P = ctypes.POINTER
_VP = ctypes.c_void_p
_BP = _P(BufParams2D)

# name -> (restype, argtypes); every symbol declared in include/*.h
SIGNATURES = {
    "DSPLIB_fir_getHandleSize": (ctypes.c_int32, [_P(FirInitArgs)]),
    "DSPLIB_fir_getSizes": (ctypes.c_int, [_P(FirInitArgs), _BP, _BP, _BP]),
    "DSPLIB_fir_init": (ctypes.c_int, [_VP, _BP, _BP, _BP, _P(FirInitArgs)]),
    "DSPLIB_fir_init_checkParams": (ctypes.c_int, [_VP, _BP, _BP, _BP, _P(FirInitArgs)]),
    "DSPLIB_fir_exec": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "DSPLIB_fir_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "DSPLIB_fir_perfEst": (None, [_VP, _BP, _BP, _BP, _P(ctypes.c_uint64), _P(ctypes.c_uint64)]),
    "DSPLIB_cascadeBiquad_getHandleSize": (ctypes.c_int32, [_P(BiquadInitArgs)]),
    "DSPLIB_cascadeBiquad_get_coefficientsBufferDesc": (
        ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _BP]),
    "DSPLIB_cascadeBiquad_get_coefficients": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, _BP, _BP, _VP, _VP]),
    "DSPLIB_cascadeBiquad_init": (ctypes.c_int, [_VP, _BP, _BP, _BP, _BP, _P(BiquadInitArgs)]),
    "DSPLIB_cascadeBiquad_init_checkParams": (ctypes.c_int, [_VP, _BP, _BP, _BP, _BP, _P(BiquadInitArgs)]),
    "DSPLIB_cascadeBiquad_exec": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "DSPLIB_cascadeBiquad_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "DSPLIB_cascadeBiquad_perfEst": (None, [_VP, _BP, _BP, _BP, _BP, _P(ctypes.c_uint64), _P(ctypes.c_uint64)]),
    "DSPLIB_fltoq15_getHandleSize": (ctypes.c_int32, [_P(ConvertInitArgs)]),
    "DSPLIB_fltoq15_init_checkParams": (ctypes.c_int, [_VP, _P(BufParams1D), _P(BufParams1D), _P(ConvertInitArgs)]),
    "DSPLIB_fltoq15_init": (ctypes.c_int, [_VP, _P(BufParams1D), _P(BufParams1D), _P(ConvertInitArgs)]),
    "DSPLIB_fltoq15_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_fltoq15_exec": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_q15tofl_getHandleSize": (ctypes.c_int32, [_P(ConvertInitArgs)]),
    "DSPLIB_q15tofl_init_checkParams": (ctypes.c_int, [_VP, _P(BufParams1D), _P(BufParams1D), _P(ConvertInitArgs)]),
    "DSPLIB_q15tofl_init": (ctypes.c_int, [_VP, _P(BufParams1D), _P(BufParams1D), _P(ConvertInitArgs)]),
    "DSPLIB_q15tofl_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_q15tofl_exec": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_interleave_getHandleSize": (ctypes.c_int32, [_P(StyleInitArgs)]),
    "DSPLIB_interleave_init_checkParams": (ctypes.c_int, [_VP, _BP, _BP, _P(StyleInitArgs)]),
    "DSPLIB_interleave_init": (ctypes.c_int, [_VP, _BP, _BP, _P(StyleInitArgs)]),
    "DSPLIB_interleave_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_interleave_exec": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_interleave_perfEst": (None, [_VP, _P(ctypes.c_uint64), _P(ctypes.c_uint64)]),
    "DSPLIB_deinterleave_getHandleSize": (ctypes.c_int32, [_P(StyleInitArgs)]),
    "DSPLIB_deinterleave_init_checkParams": (ctypes.c_int, [_VP, _BP, _BP, _P(StyleInitArgs)]),
    "DSPLIB_deinterleave_init": (ctypes.c_int, [_VP, _BP, _BP, _P(StyleInitArgs)]),
    "DSPLIB_deinterleave_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_deinterleave_exec": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_deinterleave_perfEst": (None, [_VP, _P(ctypes.c_uint64), _P(ctypes.c_uint64), ctypes.c_uint64]),
    "DSPLIB_addNCh_getHandleSize": (ctypes.c_int32, [_P(StyleInitArgs)]),
    "DSPLIB_addNCh_init_checkParams": (ctypes.c_int, [_VP, _P(BufParams3D), _BP, _P(StyleInitArgs)]),
    "DSPLIB_addNCh_init": (ctypes.c_int, [_VP, _P(BufParams3D), _BP, _P(StyleInitArgs)]),
    "DSPLIB_addNCh_exec_checkParams": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_addNCh_exec": (ctypes.c_int, [_VP, _VP, _VP]),
    "DSPLIB_addNCh_perfEst": (None, [_VP, _P(ctypes.c_uint64), _P(ctypes.c_uint64), ctypes.c_uint32]),
    "DSPLIB_gpu_setStream": (ctypes.c_int, [_VP, _VP]),
    "DSPLIB_gpu_setAsync": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_lastError": (ctypes.c_char_p, [_VP]),
    "DSPLIB_gpu_firSetPrecision": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_firSetQMode": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_kernelLaunchCount": (ctypes.c_int64, []),
    "DSPLIB_gpu_autotuneSetMode": (ctypes.c_int, [ctypes.c_int32]),
    "DSPLIB_gpu_autotuneGetMode": (ctypes.c_int32, []),
    "DSPLIB_gpu_autotuneSetCachePath": (ctypes.c_int, [ctypes.c_char_p]),
    "DSPLIB_gpu_autotuneSave": (ctypes.c_int, []),
    "DSPLIB_gpu_autotuneClear": (ctypes.c_int, []),
    "DSPLIB_gpu_autotuneLookup": (ctypes.c_int32, [ctypes.c_char_p]),
    "DSPLIB_gpu_autotuneStore": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32]),
    "DSPLIB_gpu_autotuneCount": (ctypes.c_int32, []),
    "DSPLIB_gpu_autotune": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_autotuneHandleKey": (ctypes.c_int32, [_VP, ctypes.c_char_p, ctypes.c_int32]),
    "DSPLIB_gpu_autotuneHandleCandidate": (ctypes.c_int32, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_releaseHandle": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_firStreamCreate": (ctypes.c_int, [_P(_VP), _P(FirInitArgs), _BP, _BP, _BP]),
    "DSPLIB_gpu_firStreamHandle": (_VP, [_VP]),
    "DSPLIB_gpu_firStreamExec": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "DSPLIB_gpu_firStreamReset": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_firStreamDestroy": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_raggedPlanCreate": (ctypes.c_int, [_P(_VP), ctypes.c_int32, _P(ctypes.c_int32),
                                                   _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    "DSPLIB_gpu_raggedPlanSize": (ctypes.c_int64, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_raggedPlanDestroy": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_raggedPlanStatus": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_raggedPlanSetAsync": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_status": (ctypes.c_int, [_VP]),
    "DSPLIB_gpu_injectFault": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "DSPLIB_gpu_firBiquadBatched_fwd": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "DSPLIB_gpu_firBiquadBatched_bwd": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "DSPLIB_gpu_raggedMseGrad": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "DSPLIB_gpu_firBiquadBatched_stepMse": (ctypes.c_int, [_VP] * 14),
    "DSPLIB_gpu_firBiquadBatched_stepMseHost": (ctypes.c_int, [_VP] * 12),
    "DSPLIB_gpu_firBiquadBatched_bwdStaticScratch": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                                                    _VP]),
}


def lib() -> ctypes.CDLL:
    """Load libdsplib_b200.so (build it first: python -m c7x_dsplib_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m c7x_dsplib_b200.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


class DsplibError(RuntimeError):
    def __init__(self, what, status, detail=""):
        super().__init__(f"{what} returned {status}{': ' + detail if detail else ''}")
        self.status = status


def bp(data_type, dim_x, dim_y, stride_y) -> BufParams2D:
    return BufParams2D(int(data_type), int(dim_x), int(dim_y), int(stride_y))


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


def _dtype_code(a):
    if isinstance(a, np.ndarray):
        return _NP2DT[a.dtype]
    import torch

    return {torch.int8: INT8, torch.int16: INT16, torch.int32: INT32, torch.float32: FLOAT32}[a.dtype]


def _elt(code):
    return {INT8: 1, INT16: 2, INT32: 4, FLOAT32: 4}[code]


class _Handle:
    size_fn = ""

    def __init__(self):
        L = lib()
        self.buf = ctypes.create_string_buffer(int(getattr(L, self.size_fn)(None)))
        self.h = ctypes.cast(self.buf, ctypes.c_void_p)

    def status(self) -> int:
        return lib().DSPLIB_gpu_status(self.h)

    def inject_fault(self, operation: int) -> int:
        return lib().DSPLIB_gpu_injectFault(self.h, int(operation))

    def last_error(self) -> str:
        s = lib().DSPLIB_gpu_lastError(self.h)
        return s.decode() if s else ""

    def set_stream(self, stream):
        """stream: torch.cuda.Stream, raw cudaStream_t int, or None (default stream)."""
        raw = getattr(stream, "cuda_stream", stream)
        return lib().DSPLIB_gpu_setStream(self.h, raw or None)

    def set_async(self, level):
        """False / 0: exec returns complete; True / 1: returns once queued (device buffers);
        2: returns once queued also with page-locked host buffers used in place."""
        return lib().DSPLIB_gpu_setAsync(self.h, int(level))

    def tune_key(self):
        """(autotuner key of this handle's configuration, candidate choices)."""
        buf = ctypes.create_string_buffer(256)
        n = lib().DSPLIB_gpu_autotuneHandleKey(self.h, buf, 256)
        return buf.value.decode(), [lib().DSPLIB_gpu_autotuneHandleCandidate(self.h, i) for i in range(n)]

    def autotune(self) -> int:
        """Measure this configuration's candidates now and store the fastest."""
        return lib().DSPLIB_gpu_autotune(self.h)

    def _check(self, what, st):
        if st != SUCCESS:
            raise DsplibError(what, st, self.last_error())
        return st


class FirHandle(_Handle):
    """Reference call sequence of test/DSPLIB_fir/DSPLIB_fir_d.c:101-305."""

    size_fn = "DSPLIB_fir_getHandleSize"

    def init(self, args: FirInitArgs, pin: BufParams2D, pfilt: BufParams2D, pout: BufParams2D) -> int:
        self.args, self.pin, self.pfilt, self.pout = args, pin, pfilt, pout
        return lib().DSPLIB_fir_init(self.h, ctypes.byref(pin), ctypes.byref(pfilt), ctypes.byref(pout),
                                     ctypes.byref(args))

    def init_check(self, args, pin, pfilt, pout) -> int:
        return lib().DSPLIB_fir_init_checkParams(self.h, ctypes.byref(pin), ctypes.byref(pfilt), ctypes.byref(pout),
                                                 ctypes.byref(args))

    def exec(self, x, h, y) -> int:
        return lib().DSPLIB_fir_exec(self.h, _ptr(x), _ptr(h), _ptr(y))

    def set_precision(self, p: int):
        return lib().DSPLIB_gpu_firSetPrecision(self.h, int(p))

    def set_qmode(self, on: bool):
        return lib().DSPLIB_gpu_firSetQMode(self.h, int(bool(on)))


class BiquadHandle(_Handle):
    """Reference call sequence of test/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_d.c:97-363."""

    size_fn = "DSPLIB_cascadeBiquad_getHandleSize"

    def init(self, args: BiquadInitArgs, pin, pcoef, pvar, pout) -> int:
        self.args = args
        return lib().DSPLIB_cascadeBiquad_init(self.h, ctypes.byref(pin), ctypes.byref(pcoef), ctypes.byref(pvar),
                                               ctypes.byref(pout), ctypes.byref(args))

    def init_check(self, args, pin, pcoef, pvar, pout) -> int:
        return lib().DSPLIB_cascadeBiquad_init_checkParams(self.h, ctypes.byref(pin), ctypes.byref(pcoef),
                                                           ctypes.byref(pvar), ctypes.byref(pout), ctypes.byref(args))

    def exec(self, x, coef, state, y) -> int:
        return lib().DSPLIB_cascadeBiquad_exec(self.h, _ptr(x), _ptr(coef), _ptr(state), _ptr(y))


class Fltoq15Handle(_Handle):
    """Reference call sequence of test/DSPLIB_fltoq15/DSPLIB_fltoq15_d.c:100-221."""

    size_fn = "DSPLIB_fltoq15_getHandleSize"
    prefix = "DSPLIB_fltoq15"

    def init(self, args: ConvertInitArgs, pin: BufParams1D, pout: BufParams1D) -> int:
        return getattr(lib(), self.prefix + "_init")(self.h, ctypes.byref(pin), ctypes.byref(pout), ctypes.byref(args))

    def init_check(self, args, pin, pout) -> int:
        return getattr(lib(), self.prefix + "_init_checkParams")(self.h, ctypes.byref(pin), ctypes.byref(pout),
                                                                 ctypes.byref(args))

    def exec(self, x, y) -> int:
        return getattr(lib(), self.prefix + "_exec")(self.h, _ptr(x), _ptr(y))


class Q15toflHandle(Fltoq15Handle):
    """Reference call sequence of test/DSPLIB_q15tofl/DSPLIB_q15tofl_d.c."""

    size_fn = "DSPLIB_q15tofl_getHandleSize"
    prefix = "DSPLIB_q15tofl"


class LayoutHandle(_Handle):
    """DSPLIB_interleave / DSPLIB_deinterleave / DSPLIB_addNCh handle (``prefix`` picks the kernel);
    reference call sequence of test/DSPLIB_interleave/DSPLIB_interleave_d.c."""

    def __init__(self, prefix="DSPLIB_interleave"):
        self.prefix = prefix
        self.size_fn = prefix + "_getHandleSize"
        super().__init__()

    def init(self, args, pin, pout) -> int:
        return getattr(lib(), self.prefix + "_init")(self.h, ctypes.byref(pin), ctypes.byref(pout), ctypes.byref(args))

    def init_check(self, args, pin, pout) -> int:
        return getattr(lib(), self.prefix + "_init_checkParams")(self.h, ctypes.byref(pin), ctypes.byref(pout),
                                                                 ctypes.byref(args))

    def exec(self, x, y) -> int:
        return getattr(lib(), self.prefix + "_exec")(self.h, _ptr(x), _ptr(y))


_LAYOUT_CODES = {"int8": INT8, "uint8": UINT8, "int16": INT16, "uint16": UINT16, "int32": INT32, "uint32": UINT32,
                 "int64": INT64, "uint64": UINT64, "float32": FLOAT32, "float64": FLOAT64}


def _type_code(a):
    return _LAYOUT_CODES[str(a.dtype).replace("torch.", "")]


def transpose(x, out, W, H, stride_in, stride_out, *, kind="interleave", func_style=OPTIMIZED, handle=None):
    """DSPLIB_interleave / DSPLIB_deinterleave on flat buffers (numpy or torch, host or device):
    ``x`` holds H rows of W elements ``stride_in`` bytes apart, ``out`` receives W rows of H
    elements ``stride_out`` bytes apart.  ``kind`` picks the entry points (same transpose)."""
    prefix = "DSPLIB_" + kind
    hd = handle or LayoutHandle(prefix)
    code = _type_code(x)
    args = StyleInitArgs(funcStyle=func_style)
    pin, pout = bp(code, W, H, stride_in), bp(code, H, W, stride_out)
    hd._check(prefix + "_init", hd.init(args, pin, pout))
    hd._check(prefix + "_exec", hd.exec(x, out))
    return out


def add_nch(x, out, samples, channels, inputs, sY, sZ, sO, *, func_style=OPTIMIZED, handle=None):
    """DSPLIB_addNCh on flat float32 / float64 buffers; strides in elements."""
    hd = handle or LayoutHandle("DSPLIB_addNCh")
    code = _type_code(x)
    e = 4 if code == FLOAT32 else 8
    args = StyleInitArgs(funcStyle=func_style)
    pin = BufParams3D(code, samples, channels, sY * e, inputs, sZ * e)
    pout = bp(code, samples, channels, sO * e)
    hd._check("DSPLIB_addNCh_init_checkParams", hd.init_check(args, pin, pout))
    hd._check("DSPLIB_addNCh_init", hd.init(args, pin, pout))
    hd._check("DSPLIB_addNCh_exec", hd.exec(x, out))
    return out


def _queue_on(hd, stream):
    """After init (which sets the handle up): launch on ``stream`` and return once queued."""
    if stream is not None:
        hd._check("DSPLIB_gpu_setStream", hd.set_stream(stream))
        hd._check("DSPLIB_gpu_setAsync", hd.set_async(True))


def _float_code(a):
    dt = a.dtype if isinstance(a, np.ndarray) else str(a.dtype).replace("torch.", "")
    return {"float32": FLOAT32, "float64": FLOAT64}[str(dt)]


def fltoq15(x, *, func_style=OPTIMIZED, out=None, handle=None, stream=None):
    """Float32 / float64 array (numpy or torch, host or device) to Q.15 int16."""
    n = int(x.size if isinstance(x, np.ndarray) else x.numel())
    if out is None:
        if isinstance(x, np.ndarray):
            out = np.zeros(n, np.int16)
        else:
            import torch

            out = torch.zeros(n, dtype=torch.int16, device=x.device)
    hd = handle or Fltoq15Handle()
    args = ConvertInitArgs(funcStyle=func_style, dataSize=n)
    pin, pout = BufParams1D(_float_code(x), n), BufParams1D(INT16, n)
    hd._check("DSPLIB_fltoq15_init_checkParams", hd.init_check(args, pin, pout))
    hd._check("DSPLIB_fltoq15_init", hd.init(args, pin, pout))
    _queue_on(hd, stream)
    hd._check("DSPLIB_fltoq15_exec", hd.exec(x, out))
    return out


def q15tofl(x, dtype=np.float32, *, func_style=OPTIMIZED, out=None, handle=None, stream=None):
    """Q.15 int16 array (numpy or torch, host or device) to float32 / float64."""
    n = int(x.size if isinstance(x, np.ndarray) else x.numel())
    code = {np.dtype(np.float32): FLOAT32, np.dtype(np.float64): FLOAT64}[np.dtype(dtype)]
    if out is None:
        if isinstance(x, np.ndarray):
            out = np.zeros(n, dtype)
        else:
            import torch

            out = torch.zeros(n, dtype=torch.float32 if code == FLOAT32 else torch.float64, device=x.device)
    hd = handle or Q15toflHandle()
    args = ConvertInitArgs(funcStyle=func_style, dataSize=n)
    pin, pout = BufParams1D(INT16, n), BufParams1D(code, n)
    hd._check("DSPLIB_q15tofl_init_checkParams", hd.init_check(args, pin, pout))
    hd._check("DSPLIB_q15tofl_init", hd.init(args, pin, pout))
    _queue_on(hd, stream)
    hd._check("DSPLIB_q15tofl_exec", hd.exec(x, out))
    return out


# ------------------------------------------------------------------ helpers


def fir_setup(dtype_code, batch, N, T, *, nch, func_style=OPTIMIZED, mma=False, shift=0, in_pitch=None,
              out_pitch=None, filter_pitch=None, float_q=None):
    """Descriptors + InitArgs for a FIR call, as the reference driver builds them.
    ``float_q``: FLOAT32 filters in float Q mode (InitArgs.enableQ = 1, Q = float_q)."""
    elt = _elt(dtype_code)
    args = FirInitArgs(funcStyle=func_style, dataSize=N, batchSize=batch, filterSize=T, shift=shift,
                       enableNchCoefs=int(nch), enableMMA=int(mma), MMA_SIZE=MMA_SIZE[elt],
                       enableQ=int(float_q is not None), Q=int(float_q or 0))
    out_size = N - T + 1
    pin = bp(dtype_code, N, batch, (in_pitch or N) * elt)
    pout = bp(dtype_code, (out_pitch or out_size), batch, (out_pitch or out_size) * elt)
    pfilt = bp(dtype_code, T, batch if nch else 1, (filter_pitch or T) * elt)
    st = lib().DSPLIB_fir_getSizes(ctypes.byref(args), ctypes.byref(pin), ctypes.byref(pfilt), ctypes.byref(pout))
    if st != SUCCESS:
        raise DsplibError("DSPLIB_fir_getSizes", st)
    return args, pin, pfilt, pout


def fir(x, h, T=None, *, nch=None, func_style=OPTIMIZED, precision=FIR_SIMT, qmode=False, shift=0, out=None,
        handle=None, stream=None, float_q=None):
    """y = FIR(x, h) over channel-major rows of ``x`` [batch, N] with stored
    taps ``h`` [1 or batch, T] (reference tap order).  numpy in -> numpy out
    (host staging inside the library); torch CUDA in -> torch CUDA out.
    ``stream``: queue the work on that CUDA stream and return without waiting."""
    batch, N = x.shape
    T = T or h.shape[1]
    if nch is None:
        nch = h.shape[0] > 1
    code = _dtype_code(x)
    args, pin, pfilt, pout = fir_setup(code, batch, N, T, nch=nch, func_style=func_style, shift=shift,
                                       float_q=float_q)
    out_size = N - T + 1
    if out is None:
        if isinstance(x, np.ndarray):
            out = np.zeros((batch, out_size), dtype=x.dtype)
        else:
            import torch

            out = torch.zeros((batch, out_size), dtype=x.dtype, device=x.device)
    hd = handle or FirHandle()
    hd._check("DSPLIB_fir_init", hd.init(args, pin, pfilt, pout))
    hd.set_precision(precision)
    hd.set_qmode(qmode)
    _queue_on(hd, stream)
    hd._check("DSPLIB_fir_exec", hd.exec(x, h, out))
    return out


class FirStream:
    """Streaming (overlap-save) FIR: each ``exec`` takes ``block`` new samples per
    channel (rows of ``x``) and returns ``block`` outputs per channel; the last
    ``T - 1`` samples of every channel are kept on the device for the next call
    (``DSPLIB_gpu_firStream*``)."""

    def __init__(self, dtype_code, channels, block, T, *, nch, func_style=OPTIMIZED, shift=0, precision=FIR_SIMT,
                 qmode=False):
        elt = _elt(dtype_code)
        self.channels, self.block, self.T = channels, block, T
        args = FirInitArgs(funcStyle=func_style, dataSize=block, batchSize=channels, filterSize=T, shift=shift,
                           enableNchCoefs=int(nch), enableMMA=0, MMA_SIZE=MMA_SIZE[elt], enableQ=0, Q=0)
        pin = bp(dtype_code, block, channels, block * elt)
        pout = bp(dtype_code, block, channels, block * elt)
        pfilt = bp(dtype_code, T, channels if nch else 1, T * elt)
        self.s = ctypes.c_void_p()
        st = lib().DSPLIB_gpu_firStreamCreate(ctypes.byref(self.s), ctypes.byref(args), ctypes.byref(pin),
                                              ctypes.byref(pfilt), ctypes.byref(pout))
        if st != SUCCESS:
            raise DsplibError("DSPLIB_gpu_firStreamCreate", st)
        h = lib().DSPLIB_gpu_firStreamHandle(self.s)
        lib().DSPLIB_gpu_firSetPrecision(h, precision)
        lib().DSPLIB_gpu_firSetQMode(h, int(bool(qmode)))
        self.h = h

    def exec(self, x, h, out):
        st = lib().DSPLIB_gpu_firStreamExec(self.s, _ptr(x), _ptr(h), _ptr(out))
        if st != SUCCESS:
            msg = lib().DSPLIB_gpu_lastError(self.h)
            raise DsplibError("DSPLIB_gpu_firStreamExec", st, msg.decode() if msg else "")
        return out

    def reset(self):
        return lib().DSPLIB_gpu_firStreamReset(self.s)

    def __del__(self):
        if getattr(self, "s", None) is not None and self.s.value:
            try:
                lib().DSPLIB_gpu_firStreamDestroy(self.s)
            except Exception:
                pass
            self.s = None


def biquad_descs(C, N, S, form, nch, *, pitch=None, var_pitch=None, func_style=OPTIMIZED):
    nv = 4 if form == DF1 else 2
    pin = bp(FLOAT32, C, N, (pitch or C) * 4)
    pout = bp(FLOAT32, C, N, (pitch or C) * 4)
    pvar = bp(FLOAT32, C, S * nv, (var_pitch or C) * 4)
    pcn = bp(FLOAT32, S * 5, C if nch else 1, S * 5 * 4)
    popt = BufParams2D()
    st = lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(FLOAT32, S, C, form, int(nch), ctypes.byref(popt))
    if st != SUCCESS:
        raise DsplibError("get_coefficientsBufferDesc", st)
    args = BiquadInitArgs(funcStyle=func_style, dataSize=N, numStages=S, numChannels=C, enableNChCoeffs=int(nch),
                          biquadForm=form)
    return args, pin, pout, pvar, pcn, popt


def opt_coefficients(natural, form, nch, C):
    """Natural [rows, S*5] float32 -> the optimized buffer get_coefficients makes (numpy)."""
    natural = np.ascontiguousarray(natural, dtype=np.float32)
    S = natural.shape[1] // 5
    pcn = bp(FLOAT32, S * 5, C if nch else 1, S * 5 * 4)
    popt = BufParams2D()
    lib().DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(FLOAT32, S, C, form, int(nch), ctypes.byref(popt))
    if form != TIF and not nch:
        return natural.copy(), popt
    opt = np.zeros(popt.dim_y * popt.stride_y // 4, dtype=np.float32)
    st = lib().DSPLIB_cascadeBiquad_get_coefficients(form, int(nch), ctypes.byref(pcn), ctypes.byref(popt),
                                                     natural.ctypes.data, opt.ctypes.data)
    if st != SUCCESS:
        raise DsplibError("get_coefficients", st)
    return opt, popt


def cascade_biquad(x, coef, state, *, form, nch, func_style=OPTIMIZED, out=None, handle=None, stream=None):
    """One exec over time-major ``x`` [N, C].  ``coef`` is the natural buffer
    for NATC and the optimized buffer (``opt_coefficients``) for OPTIMIZED;
    ``state`` [S*nv, C] is updated in place."""
    N, C = x.shape
    nv = 4 if form == DF1 else 2
    S = state.shape[0] // nv
    args, pin, pout, pvar, pcn, popt = biquad_descs(C, N, S, form, nch, pitch=x.shape[1],
                                                    var_pitch=state.shape[1], func_style=func_style)
    if out is None:
        if isinstance(x, np.ndarray):
            out = np.zeros_like(x)
        else:
            import torch

            out = torch.zeros_like(x)
    hd = handle or BiquadHandle()
    hd._check("DSPLIB_cascadeBiquad_init", hd.init(args, pin, pcn if func_style == NATC else popt, pvar, pout))
    _queue_on(hd, stream)
    hd._check("DSPLIB_cascadeBiquad_exec", hd.exec(x, coef, state, out))
    return out


def kernel_launch_count() -> int:
    return int(lib().DSPLIB_gpu_kernelLaunchCount())
