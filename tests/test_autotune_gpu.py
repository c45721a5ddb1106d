"""Autotuner on the GPU: every candidate choice a key may hold runs the kernel to the
same oracle checks as the built-in rule (tensor-core FIR: the same output bit for bit;
integer FIR bit-exact to the oracle; cascade scan within the scan's FP64 bound; filter
bank: the forward bit for bit), and MEASURE mode times and stores a choice at init."""
import json

import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def table():
    L = D.lib()
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    L.DSPLIB_gpu_autotuneSetMode(1)
    yield L
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    L.DSPLIB_gpu_autotuneSetMode(1)


def test_fir_bf16x3_every_candidate(table):
    rng = np.random.default_rng(31)
    x = rng.standard_normal((6, 40000)).astype(np.float32)
    h = (rng.standard_normal((6, 256)) / 16).astype(np.float32)
    hd = D.FirHandle()
    y0 = D.fir(x, h, 256, nch=True, precision=D.FIR_BF16X3, handle=hd)
    w = oracle.fir_f64(x, h, 256, nch=1)
    assert np.all(np.abs(y0 - w).max(axis=1) <= 1e-5 * np.abs(w).max(axis=1))
    key, cands = hd.tune_key()
    assert key.startswith("fir_bf16x3|T=256|") and len(cands) >= 3, (key, cands)
    for c in cands:
        assert table.DSPLIB_gpu_autotuneStore(key.encode(), c) == 0
        y = D.fir(x, h, 256, nch=True, precision=D.FIR_BF16X3, handle=hd)
        assert np.array_equal(y, y0), c


@pytest.mark.parametrize("dtype,qmode,shift", [(np.int8, True, 7), (np.int8, False, 0), (np.int16, True, 15),
                                               (np.int16, False, 0)])
def test_fir_int_every_candidate(table, dtype, qmode, shift):
    rng = np.random.default_rng(32)
    info = np.iinfo(dtype)
    x = rng.integers(info.min, info.max, size=(10, 9000), endpoint=True).astype(dtype)
    h = rng.integers(info.min, info.max, size=(1, 128), endpoint=True).astype(dtype)
    want = oracle.fir_q(x, h, 128, shift, nch=0) if qmode else oracle.fir(x, h, 128, nch=0)
    hd = D.FirHandle()
    y0 = D.fir(x, h, 128, nch=False, qmode=qmode, shift=shift, handle=hd)
    assert np.array_equal(y0, want)
    key, cands = hd.tune_key()
    assert key.startswith("fir_int|") and len(cands) >= 4, (key, cands)
    for c in cands:
        assert table.DSPLIB_gpu_autotuneStore(key.encode(), c) == 0
        y = D.fir(x, h, 128, nch=False, qmode=qmode, shift=shift, handle=hd)
        assert np.array_equal(y, want), c


@pytest.mark.parametrize("form", [D.DF1, D.DF2, D.TDF2, D.TIF])
def test_biquad_scan_every_candidate(table, form):
    from test_biquad_gpu import check_accuracy, nv, oracle_run, stable_sections

    rng = np.random.default_rng(40 + form)
    N, C, S, nch = 12000, 64, 4, 1
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = stable_sections(rng, C, S)
    opt, _ = D.opt_coefficients(nat, form, nch, C)
    y32, st32, y64, s64 = oracle_run(form, x, nat, np.zeros((S * nv(form), C), np.float32), nch)
    hd = D.BiquadHandle()
    st = np.zeros((S * nv(form), C), np.float32)
    D.cascade_biquad(x, opt, st, form=form, nch=nch, handle=hd)
    key, cands = hd.tune_key()
    assert key.startswith(f"bq_scan|form={form}|S={S}|") and len(cands) >= 6, (key, cands)
    for c in cands:
        assert table.DSPLIB_gpu_autotuneStore(key.encode(), c) == 0
        st = np.zeros((S * nv(form), C), np.float32)
        y = D.cascade_biquad(x, opt, st, form=form, nch=nch, handle=hd)
        check_accuracy(y, y32, y64, f"form {form} choice {c}")
        if form != D.TIF:  # TIF's state is in transformed coordinates; its output is checked
            check_accuracy(st, st32, s64, f"final state, form {form} choice {c}")


def test_bank_run_length_every_candidate(table):
    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    rng = np.random.default_rng(50)
    lengths = [int(v) for v in rng.integers(1000, 90000, size=24)]
    taps = [int(v) for v in rng.integers(1, 400, size=24)]
    stages = [int(v) for v in rng.integers(0, 5, size=24)]
    x = torch.randn(sum(lengths), device="cuda")
    h = torch.randn(sum(taps), device="cuda") / 8
    c = torch.zeros(5 * sum(stages), device="cuda")
    c[0::5] = 1.0  # pass-through sections: the output is the FIR output

    def forward():
        bank = RaggedFilterBank(lengths, taps, stages)
        y = torch.empty(bank.sizes[0], device="cuda")
        bank.forward_raw(x, h, c, y, torch.empty(bank.sizes[3], device="cuda"))
        torch.cuda.synchronize()
        return y.cpu()

    y0 = forward()
    total = sum(lengths)
    key = f"bank_runs|ch=2^{int(np.ceil(np.log2(24)))}|samples=2^{int(np.ceil(np.log2(total)))}|Tmax={max(taps)}|sms="
    key += str(torch.cuda.get_device_properties(0).multi_processor_count)
    for rt in (1, 2, 8, 16):
        assert table.DSPLIB_gpu_autotuneStore(key.encode(), rt) == 0
        assert torch.equal(forward(), y0), rt


def test_measure_mode_stores_and_saves(table, tmp_path):
    path = tmp_path / "tune.json"
    table.DSPLIB_gpu_autotuneSetCachePath(str(path).encode())
    assert table.DSPLIB_gpu_autotuneSetMode(2) == 0
    rng = np.random.default_rng(60)
    x = rng.standard_normal((4, 30000)).astype(np.float32)
    h = (rng.standard_normal((1, 64)) / 8).astype(np.float32)
    hd = D.FirHandle()
    D.fir(x, h, 64, nch=False, precision=D.FIR_BF16X3, handle=hd)  # precision set after the first init
    key, cands = hd.tune_key()
    assert hd.autotune() == 0
    choice = table.DSPLIB_gpu_autotuneLookup(key.encode())
    assert choice in cands
    assert json.loads(path.read_text())["entries"][key] == choice
    # a second init of the same class measures nothing new; results still match the oracle
    y = D.fir(x, h, 64, nch=False, precision=D.FIR_BF16X3, handle=hd)
    w = oracle.fir_f64(x, h, 64, nch=0)
    assert np.all(np.abs(y - w).max(axis=1) <= 1e-5 * np.abs(w).max(axis=1))
    # the cascade scan is measured at init in MEASURE mode
    from test_biquad_gpu import stable_sections

    C, N, S = 40, 6000, 3
    xb = rng.standard_normal((N, C)).astype(np.float32)
    opt, _ = D.opt_coefficients(stable_sections(rng, 1, S), D.DF2, 0, C)
    hb = D.BiquadHandle()
    D.cascade_biquad(xb, opt, np.zeros((2 * S, C), np.float32), form=D.DF2, nch=0, handle=hb)
    kb, cb = hb.tune_key()
    assert table.DSPLIB_gpu_autotuneLookup(kb.encode()) in cb
