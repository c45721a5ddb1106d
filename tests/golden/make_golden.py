"""Generate the golden fixtures in tests/golden/ from the reference's own Python
test models.  Run in a checkout that has the reference project available:

    python tests/golden/make_golden.py --ref <reference checkout>

Outputs (committed; the GPU box never needs the reference tree):
  fir_golden.npz     FIR cases drawn from test/DSPLIB_idat_gen/DSPLIB_fir/test_cases_list.csv
  biquad_golden.npz  cascade-biquad cases drawn from
                     test/DSPLIB_idat_gen/DSPLIB_cascadeBiquad/test_cases_list.csv
  layout_golden.npz  interleave / deinterleave / addNCh cases drawn from
                     test/DSPLIB_idat_gen/DSPLIB_{interleave,deinterleave,addNCh}/test_cases_list.csv
                     (``--what layout`` writes only this file)

FIR goldens follow the reference generator step for step
(test/DSPLIB_idat_gen/DSPLIB_fir/gen_data.py:218-311): uniform data, taps
reversed before storage, golden = numpy.convolve(x, stored_taps, "valid")
computed on the unrounded float64 draws (float inputs) or in the integer dtype
itself (integer inputs, where numpy wraps exactly like the natural-C kernel).
That generator writes into the reference tree at import time, so its few
lines of arithmetic are followed here instead of imported.

Biquad goldens import the reference model class
(test/DSPLIB_idat_gen/DSPLIB_cascadeBiquad/cascadeBiquad.py) and call it the
way gen_data.py:230-300 does: Butterworth designs split into second-order
sections, uniform input, fp64 ``scipy.signal.sosfilt`` output and final state,
and the model's float32 form-exact recursions (precision="fp32").

The reference generator uses the unseeded global numpy RNG; here each case
seeds it (np.random.seed(case_id)) so the fixtures are reproducible.
"""
from __future__ import annotations

import argparse
import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

FIR_IDS = [1, 3, 6, 9, 14, 20, 33, 47, 58, 71, 96, 120, 137, 150, 171, 188, 199, 200]
BIQUAD_STAGES = [1, 3, 4, 8, 9, 12]
BIQUAD_REPS4_IDS = [675, 676, 677, 678]


def fir_cases(ref):
    path = os.path.join(ref, "test/DSPLIB_idat_gen/DSPLIB_fir/test_cases_list.csv")
    rows = {int(r["ID"]): r for r in csv.DictReader(open(path, encoding="utf-8-sig"))}
    out = {}
    for cid in FIR_IDS:
        r = rows[cid]
        N, T, B = int(r["dataSize"]), int(r["filterSize"]), int(r["batchSize"])
        nch, mma = int(r["enableNChCoefs"]), int(r["enableMMA"])
        np.random.seed(cid)
        x = np.random.uniform(low=-1, high=1, size=(B, N)).astype("float")
        f = np.random.uniform(low=-1, high=1, size=(B if nch else 1, T)).astype("float")
        f = f[:, ::-1]
        y = np.stack([np.convolve(x[ch], f[ch if nch else 0], mode="valid") for ch in range(B)])
        key = f"f{cid}"
        out[key + "_meta"] = np.array([cid, N, T, B, nch, mma], dtype=np.int64)
        out[key + "_x"] = x.astype(np.float32)
        out[key + "_h"] = np.ascontiguousarray(f).astype(np.float32)
        out[key + "_y"] = y.astype(np.float32)
    # Integer wrap-mode cases: same generator path with integer dtypes
    # (gen_data.py:218-250), numpy convolve keeps the input dtype and wraps.
    for i, (dt, bits, N, T, B, nch) in enumerate(
        [("int8", 8, 96, 16, 3, 1), ("int16", 16, 128, 32, 4, 0), ("int16", 16, 200, 64, 2, 1),
         ("int32", 32, 80, 8, 2, 1)]
    ):
        np.random.seed(1000 + i)
        lo, hi = -(2 ** (bits - 1)), 2 ** (bits - 1)
        x = np.random.uniform(low=lo, high=hi, size=(B, N)).astype(dt)
        f = np.random.uniform(low=lo, high=hi, size=(B if nch else 1, T)).astype(dt)[:, ::-1]
        y = np.stack([np.convolve(x[ch], f[ch if nch else 0], mode="valid") for ch in range(B)])
        assert y.dtype == np.dtype(dt)
        key = f"i{i}"
        out[key + "_meta"] = np.array([1000 + i, N, T, B, nch, bits], dtype=np.int64)
        out[key + "_x"] = x
        out[key + "_h"] = np.ascontiguousarray(f)
        out[key + "_y"] = y
    return out


def biquad_cases(ref):
    model_dir = os.path.join(ref, "test/DSPLIB_idat_gen/DSPLIB_cascadeBiquad")
    sys.path.insert(0, model_dir)
    from cascadeBiquad import DSPLIB_cascadeBiquad  # reference model

    path = os.path.join(model_dir, "test_cases_list.csv")
    rows = list(csv.DictReader(open(path, encoding="utf-8-sig")))
    chosen = []
    seen = set()
    for r in rows:
        key = (r["biquadForm"], r["enableNChCoeffs"], int(r["numStages"]))
        if (int(r["numStages"]) in BIQUAD_STAGES and r["enableCalcCoeffs"] == "False" and r["numExecReps"] == "1"
                and key not in seen):
            seen.add(key)
            chosen.append(r)
    chosen += [r for r in rows if int(r["ID"]) in BIQUAD_REPS4_IDS]
    out = {}
    forms = {"DSPLIB_BIQUAD_TIF": 0, "DSPLIB_BIQUAD_DF1": 1, "DSPLIB_BIQUAD_DF2": 2, "DSPLIB_BIQUAD_TDF2": 3}
    for r in chosen:
        cid = int(r["ID"])
        N, C, S = int(r["dataSize"]), int(r["numChannels"]), int(r["numStages"])
        reps = int(r["numExecReps"])
        nch = r["enableNChCoeffs"] == "True"
        form = r["biquadForm"]
        np.random.seed(cid)
        m64 = DSPLIB_cascadeBiquad(dataType="float", numStages=S, numChannels=C, biquadForm=form,
                                   enableNChCoeffs=nch, numSamples=N)
        x = np.random.uniform(low=-1.0, high=1.0, size=(reps * N, C)).astype("float")
        y64 = m64.exec(x)
        zf64 = m64.zi.copy()
        m32 = DSPLIB_cascadeBiquad(dataType="float", numStages=S, numChannels=C, biquadForm=form,
                                   enableNChCoeffs=nch, numSamples=N, precision="fp32")
        m32.set_filter_coefficients(m64.sosCoefs)
        y32 = m32.exec(x)
        zf32 = m32.zi.copy()
        rows_c = C if nch else 1
        natural = np.stack([m64.sosCoefs[:, [0, 1, 2, 4, 5], ch].reshape(-1) for ch in range(rows_c)])
        key = f"b{cid}"
        out[key + "_meta"] = np.array([cid, forms[form], int(nch), N, C, S, reps, int(r["dataPitch"]),
                                       int(r["filterVarPitch"])], dtype=np.int64)
        out[key + "_x"] = x.astype(np.float32)
        out[key + "_coef"] = natural.astype(np.float32)
        out[key + "_y64"] = y64.astype(np.float32)  # headers store the golden as float
        out[key + "_y32"] = y32.astype(np.float32)
        out[key + "_zf64"] = zf64.astype(np.float32)
        out[key + "_zf32"] = zf32.astype(np.float32)
        if form == "DSPLIB_BIQUAD_TIF":
            tc = m64.tifBiquadCascadeCoefs  # [S, 4, rows] in model order {c0, c1, -a1, -a2}
            g = m64.tifBiquadCascadeGains  # [G, rows]
            # storage order of the reference buffers: {c0, c1, -a2, -a1} (file_io.py:170-176)
            stor = np.stack([tc[:, [0, 1, 3, 2], ch].reshape(-1) for ch in range(rows_c)])
            out[key + "_tif"] = stor.astype(np.float32)
            out[key + "_gain"] = np.ascontiguousarray(g.T).astype(np.float32)
    return out


LAYOUT_DT = {"int8_t": np.int8, "uint8_t": np.uint8, "int16_t": np.int16, "uint16_t": np.uint16,
             "int32_t": np.int32, "uint32_t": np.uint32, "int64_t": np.int64, "uint64_t": np.uint64,
             "float": np.float32, "double": np.float64}


def calc_stride(nbytes):
    """DSPLIB_CALC_STRIDE(bytes, DSPLIB_ALIGN_SHIFT_64BYTES) (src/common/DSPLIB_types.h:316)."""
    return ((nbytes - 1) >> 6) + 1 << 6


def _layout_input(rng, dt, count):
    if np.dtype(dt).kind == "f":
        return rng.uniform(-1, 1, count).astype(dt)
    info = np.iinfo(dt)
    return rng.integers(info.min, info.max, count, dtype=dt, endpoint=True)


def layout_cases(ref, max_elems=4096, max_sum_elems=16000):
    """Transposes (interleave, deinterleave) and channel sums (addNCh) at the shapes of the
    reference's test tables, outputs from the reference natural-C kernels (oracle/_ref).
    Strides are the drivers' DSPLIB_CALC_STRIDE(stride * size, 64-byte) bytes
    (DSPLIB_interleave_d.c:98-106, DSPLIB_deinterleave_d.c:99-107); addNCh follows
    DSPLIB_addNCh_d.c:93-103 and its generator (DSPLIB_idat_gen/DSPLIB_addNCh/gen_data.py:
    uniform(-10, 10) inputs, golden = float64 sum over the inputs)."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import oracle

    out = {}
    for kind in ("interleave", "deinterleave"):
        path = os.path.join(ref, f"test/DSPLIB_idat_gen/DSPLIB_{kind}/test_cases_list.csv")
        for r in csv.DictReader(open(path, encoding="utf-8-sig")):
            cid, dt = int(r["ID"]), LAYOUT_DT[r["dType"]]
            W, H = int(r["widthIn"]), int(r["heightIn"])
            if W * H > max_elems:
                continue
            e = np.dtype(dt).itemsize
            s_in, s_out = calc_stride(int(r["strideIn"]) * e), calc_stride(int(r["strideOut"]) * e)
            s_in, s_out = max(s_in, calc_stride(W * e)), max(s_out, calc_stride(H * e))
            if H * s_in > (16 << 10) or W * s_out > (16 << 10):
                continue
            rng = np.random.default_rng(cid + (0 if kind == "interleave" else 1000))
            x = _layout_input(rng, dt, H * s_in // e)
            y = np.zeros(((W - 1) * s_out) // e + H, dt)
            oracle.transpose(x, W, H, s_in, s_out, y, impl="ref")
            key = f"{kind[0]}{cid}"
            out[key + "_meta"] = np.array([cid, W, H, s_in, s_out], dtype=np.int64)
            out[key + "_x"] = x
            out[key + "_y"] = y
    path = os.path.join(ref, "test/DSPLIB_idat_gen/DSPLIB_addNCh/test_cases_list.csv")
    for r in csv.DictReader(open(path, encoding="utf-8-sig")):
        cid, dt = int(r["ID"]), LAYOUT_DT[r["dType"]]
        L, C, S = int(r["inInputs"]), int(r["inChannels"]), int(r["inSamples"])
        e = np.dtype(dt).itemsize
        sY = calc_stride(int(r["strideInElements"]) * e) // e
        sZ = sY * C
        if L * sZ > max_sum_elems:
            continue
        np.random.seed(cid)
        x64 = np.random.uniform(low=-10, high=10, size=(L, C, S))
        x = np.zeros((L, C, sY), dt)
        x[:, :, :S] = x64.astype(dt)
        golden = np.sum(x64, axis=0).astype(dt)  # the generator's static reference
        y = np.zeros(C * sY, dt)
        oracle.addnch(x.reshape(-1), S, C, L, sY, sZ, sY, y, impl="ref")
        key = f"a{cid}"
        out[key + "_meta"] = np.array([cid, S, C, L, sY, sZ, sY], dtype=np.int64)
        out[key + "_x"] = x.reshape(-1)
        out[key + "_y"] = y
        out[key + "_golden"] = golden
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference checkout")
    ap.add_argument("--what", default="all", choices=["all", "layout"])
    a = ap.parse_args()
    if a.what == "all":
        np.savez_compressed(os.path.join(HERE, "fir_golden.npz"), **fir_cases(a.ref))
        np.savez_compressed(os.path.join(HERE, "biquad_golden.npz"), **biquad_cases(a.ref))
    np.savez_compressed(os.path.join(HERE, "layout_golden.npz"), **layout_cases(a.ref))


if __name__ == "__main__":
    main()
