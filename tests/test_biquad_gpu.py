"""Cascade-biquad parity on the GPU, through the C ABI, against the CPU oracle.

NATC is bit-exact to the reference natural-C kernels (outputs and final
states).  OPTIMIZED (chunked parallel-in-time scan) is checked against the
FP64 oracle: max |y - y64| / max |y64| <= 1e-4 per channel, and against the
reference test criterion abs 2^-10 (test/DSPLIB_cascadeBiquad/
DSPLIB_cascadeBiquad_d.c:391-405); final states to the same bounds.
"""
import numpy as np
import pytest

import c7x_dsplib_b200 as D
import oracle
from conftest import case_keys

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL_REF = 2.0 ** -10
REL = 1e-4
FORMS = [D.DF1, D.DF2, D.TDF2, D.TIF]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def stable_sections(rng, rows, S, rmax=0.95):
    """Natural [rows, S*5]: conjugate poles r in [0.5, rmax] at angle theta, zeros on the
    unit circle, each section scaled so |H(e^{j theta})| = 1 (the rule of the benchmark
    workload), which keeps outputs O(1) like the reference's normalised test filters."""
    out = np.zeros((rows, S, 5))
    for r_ in range(rows):
        for s in range(S):
            r, th, ph = rng.uniform(0.5, rmax), rng.uniform(0, np.pi), rng.uniform(0, np.pi)
            b = np.array([1.0, -2 * np.cos(ph), 1.0])
            a = np.array([1.0, -2 * r * np.cos(th), r * r])
            z = np.exp(-1j * th * np.arange(3))
            g = 1.0 / max(abs(np.dot(b, z) / np.dot(a, z)), 1e-12)
            out[r_, s] = [g * b[0], g * b[1], g * b[2], a[1], a[2]]
    return out.reshape(rows, S * 5).astype(np.float32)


def nv(form):
    return 4 if form == D.DF1 else 2


def oracle_run(form, x, nat, state, nch):
    """fp32 form-exact port (TIF through its own transform) and the FP64 ground truth."""
    st32 = state.copy()
    if form == D.TIF:
        rows = nat.shape[0]
        tcs, gns = zip(*[oracle.tif_coefficients(nat[r]) for r in range(rows)])
        y32 = oracle.biquad_tif(x, np.stack(tcs), np.stack(gns), st32, nch=nch)
    else:
        y32 = oracle.biquad(form, x, nat, st32, nch=nch)
    # FP64 truth on the direct form with the same natural coefficients (TIF: DF2 equivalent, zero state)
    s64 = np.zeros((state.shape[0] * (2 if form == D.DF1 else 1), state.shape[1]), np.float64)
    if form == D.TIF:
        s64 = np.zeros((nat.shape[1] // 5 * 2, x.shape[1]), np.float64)
        y64 = oracle.biquad_f64(D.DF2, x, nat, s64, nch=nch)
    else:
        s64 = state.astype(np.float64).copy()
        y64 = oracle.biquad_f64(form, x, nat, s64, nch=nch)
    return y32, st32, y64, s64


def rel_per_channel(y, y64):
    return np.max(np.abs(y.astype(np.float64) - y64), axis=0) / np.maximum(np.max(np.abs(y64), axis=0), 1e-6)


def check_accuracy(y, y32, y64, what):
    """The scan against FP64: max |y - y64| / max |y64| <= 1e-4 per channel, or at most
    4x the error of the reference's own sequential FP32 recursion when that is larger
    (high-gain cascades); and the reference criterion abs 2^-10, scaled by the signal
    peak when the output exceeds 1."""
    seq = rel_per_channel(y32, y64)
    got = rel_per_channel(y, y64)
    assert np.all(got <= np.maximum(REL, 4 * seq + 1e-6)), (what, float(np.max(got)), float(np.max(seq)))
    scale = max(1.0, float(np.max(np.abs(y64))))
    assert np.max(np.abs(y - y32)) <= TOL_REF * scale, what


@pytest.mark.parametrize("form", [D.DF1, D.DF2, D.TDF2])
@pytest.mark.parametrize("nch", [0, 1])
@pytest.mark.parametrize("on_device", [False, True])
def test_natc_bitexact(form, nch, on_device):
    rng = np.random.default_rng(form * 7 + nch)
    for (N, C, S) in [(1, 1, 1), (64, 2, 3), (513, 17, 5), (2000, 40, 12)]:
        x = rng.uniform(-1, 1, size=(N, C)).astype(np.float32)
        nat = stable_sections(rng, C if nch else 1, S)
        st = rng.standard_normal((S * nv(form), C)).astype(np.float32) * 0.1
        s_ref = st.copy()
        want = oracle.biquad(form, x, nat, s_ref, nch=nch)
        if on_device:
            sd = dev(st)
            got = host(D.cascade_biquad(dev(x), dev(nat), sd, form=form, nch=nch, func_style=D.NATC))
            st_got = host(sd)
        else:
            st_got = st.copy()
            got = D.cascade_biquad(x, nat, st_got, form=form, nch=nch, func_style=D.NATC)
        assert np.array_equal(got, want), (N, C, S)
        assert np.array_equal(st_got, s_ref), (N, C, S)


def test_natc_tif_runs_df2():
    """NATC with biquadForm = TIF runs DF2 on natural coefficients (DSPLIB_cascadeBiquad.cpp:468-471)."""
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, size=(300, 8)).astype(np.float32)
    nat = stable_sections(rng, 1, 3)
    st = np.zeros((6, 8), np.float32)
    s_ref = st.copy()
    got = D.cascade_biquad(x, nat, st, form=D.TIF, nch=0, func_style=D.NATC)
    assert np.array_equal(got, oracle.biquad(D.DF2, x, nat, s_ref, nch=0))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference _cn library not built")
def test_natc_bitexact_vs_reference_cn():
    rng = np.random.default_rng(8)
    x = rng.standard_normal((8192, 32)).astype(np.float32)
    nat = stable_sections(rng, 1, 4)
    for form in (D.DF1, D.DF2, D.TDF2):
        st = np.zeros((4 * nv(form), 32), np.float32)
        s2 = st.copy()
        got = D.cascade_biquad(dev(x), dev(nat), dev(st), form=form, nch=0, func_style=D.NATC)
        assert np.array_equal(host(got), oracle.biquad(form, x, nat, s2, nch=0, impl="ref"))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("nch", [0, 1])
def test_opt_scan_accuracy(form, nch):
    rng = np.random.default_rng(100 + form * 3 + nch)
    # C <= 148: one CTA per channel along time; C > 148: lane = channel with clusters
    for (N, C, S) in [(1, 1, 1), (31, 3, 2), (8192, 32, 4), (40000, 40, 3), (3001, 65, 8), (700, 5, 13),
                      (2000, 200, 3), (17000, 149, 2)]:
        x = rng.standard_normal((N, C)).astype(np.float32)
        nat = stable_sections(rng, C if nch else 1, S)
        st = np.zeros((S * nv(form), C), np.float32)
        opt, _ = D.opt_coefficients(nat, form, nch, C)
        sd = dev(st)
        y = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=nch))
        y32, st32, y64, _ = oracle_run(form, x, nat, st, nch)
        check_accuracy(y, y32, y64, (N, C, S))
        sc = max(1.0, float(np.max(np.abs(st32))))
        assert np.max(np.abs(host(sd) - st32)) <= 1e-3 * sc, (N, C, S)


@pytest.mark.parametrize("form", FORMS)
def test_opt_streaming_state_carry(form):
    """numExecReps-style streaming (DSPLIB_cascadeBiquad_d.c:260-273): four exec calls
    on consecutive blocks equal one call on the whole signal."""
    rng = np.random.default_rng(form)
    N, C, S = 5000, 12, 4
    x = rng.standard_normal((4 * N, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, form, 0, C)
    st = dev(np.zeros((S * nv(form), C), np.float32))
    h = D.BiquadHandle()
    parts = []
    for k in range(4):
        parts.append(host(D.cascade_biquad(dev(x[k * N:(k + 1) * N]), dev(opt), st, form=form, nch=0, handle=h)))
    y = np.concatenate(parts)
    y32, st32, y64, _ = oracle_run(form, x, nat, np.zeros((S * nv(form), C), np.float32), 0)
    check_accuracy(y, y32, y64, form)
    assert np.max(np.abs(host(st) - st32)) <= 1e-3 * max(1.0, float(np.max(np.abs(st32))))


def test_opt_nonzero_initial_state():
    rng = np.random.default_rng(77)
    for form in (D.DF1, D.DF2, D.TDF2):
        N, C, S = 3000, 33, 3
        x = rng.standard_normal((N, C)).astype(np.float32)
        nat = stable_sections(rng, C, S)
        st = (rng.standard_normal((S * nv(form), C)) * 0.5).astype(np.float32)
        opt, _ = D.opt_coefficients(nat, form, 1, C)
        sd = dev(st)
        y = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=1))
        s_ref = st.copy()
        want = oracle.biquad(form, x, nat, s_ref, nch=1)
        s64 = st.astype(np.float64)
        y64 = oracle.biquad_f64(form, x, nat, s64, nch=1)
        check_accuracy(y, want, y64, form)
        assert np.max(np.abs(host(sd) - s64)) <= 1e-3 * max(1.0, float(np.max(np.abs(s64))))


@pytest.mark.parametrize("C", [5, 160])
def test_opt_single_sample_multi_stage(C):
    """N = 1 with several stages and a nonzero state: every stage's old state shifts
    (DF1: xd1/yd1 move into xd2/yd2 of the same stage)."""
    rng = np.random.default_rng(C)
    for form in (D.DF1, D.DF2, D.TDF2):
        N, S = 1, 3
        x = rng.standard_normal((N, C)).astype(np.float32)
        nat = stable_sections(rng, C, S)
        st = (rng.standard_normal((S * nv(form), C)) * 0.5).astype(np.float32)
        opt, _ = D.opt_coefficients(nat, form, 1, C)
        sd = dev(st)
        y = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=1))
        s_ref = st.copy()
        want = oracle.biquad(form, x, nat, s_ref, nch=1)
        assert np.max(np.abs(y - want)) <= 1e-5 * max(1.0, float(np.max(np.abs(want)))), form
        assert np.max(np.abs(host(sd) - s_ref)) <= 1e-5 * max(1.0, float(np.max(np.abs(s_ref)))), form


def test_opt_in_place():
    rng = np.random.default_rng(3)
    N, C, S = 10000, 32, 4
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, D.DF2, 0, C)
    xd = dev(x)
    D.cascade_biquad(xd, dev(opt), dev(np.zeros((2 * S, C), np.float32)), form=D.DF2, nch=0, out=xd)
    _, _, y64, _ = oracle_run(D.DF2, x, nat, np.zeros((2 * S, C), np.float32), 0)
    assert np.max(rel_per_channel(host(xd), y64)) <= REL


@pytest.mark.parametrize("form", FORMS)
def test_opt_deep_cascade_lane_scan(form):
    """Cascades of 26 - 160 stages stay on the lane-per-channel scan kernel with the matrix
    powers formed per stage (no per-stage table): across a cluster of CTAs (5000 samples)
    and within one CTA (600 samples), shared and per-channel coefficients."""
    rng = np.random.default_rng(80 + form)
    for (N, C, S, nch) in [(5000, 48, 40, 0), (600, 200, 33, 1), (2000, 40, 120, 1)]:
        x = rng.standard_normal((N, C)).astype(np.float32)
        nat = stable_sections(rng, C if nch else 1, S, rmax=0.8)
        st = np.zeros((S * nv(form), C), np.float32)
        opt, _ = D.opt_coefficients(nat, form, nch, C)
        sd = dev(st)
        y = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=nch))
        y32, st32, y64, s64 = oracle_run(form, x, nat, st, nch)
        # against FP64 only (per channel, within 1e-4 or 4x the error of the sequential FP32
        # recursion): over a deep high-gain cascade the FP32 restatement itself drifts beyond
        # the reference's absolute 2^-10 criterion, in its own direction
        seq = rel_per_channel(y32, y64)
        assert np.all(rel_per_channel(y, y64) <= np.maximum(REL, 4 * seq + 1e-6)), (form, N, C, S)
        got = host(sd).astype(np.float64)
        if form != D.TIF:
            # final states against FP64: within 1e-3 of their scale, or 4x the error of the
            # sequential FP32 recursion when that is larger (deep cascades with large inner gain)
            seq = float(np.max(np.abs(st32 - s64)))
            tol = max(1e-3 * max(1.0, float(np.max(np.abs(s64)))), 4 * seq + 1e-6)
            assert np.max(np.abs(got - s64)) <= tol, (form, N, C, S)
        else:
            # TIF keeps its own state form (no FP64 restatement): check it by what it does,
            # continuing the signal for a second block from the returned state
            x2 = rng.standard_normal((N, C)).astype(np.float32)
            y2 = host(D.cascade_biquad(dev(x2), dev(opt), sd, form=form, nch=nch))
            xx = np.concatenate([x, x2])
            yy32, _, yy64, _ = oracle_run(form, xx, nat, st, nch)
            seq = rel_per_channel(yy32, yy64)
            got2 = rel_per_channel(np.concatenate([y, y2]), yy64)
            assert np.all(got2 <= np.maximum(REL, 4 * seq + 1e-6)), (form, N, C, S, float(np.max(got2)))


def test_opt_deep_cascade_uses_sequential_kernel():
    rng = np.random.default_rng(6)
    N, C, S = 300, 9, 170  # DF1 beyond the scan kernel's stage limit (160)
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S, rmax=0.6)
    st = np.zeros((4 * S, C), np.float32)
    y = host(D.cascade_biquad(dev(x), dev(nat), dev(st), form=D.DF1, nch=0))
    s_ref = st.copy()
    assert np.array_equal(y, oracle.biquad(D.DF1, x, nat, s_ref, nch=0))


def _golden_cases():
    import os

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "biquad_golden.npz"))
    return case_keys(d, "b")


@pytest.mark.parametrize("key", _golden_cases())
@pytest.mark.parametrize("style", [D.NATC, D.OPTIMIZED])
def test_reference_flow_golden(golden_biquad, key, style):
    """Reference driver flow (DSPLIB_cascadeBiquad_d.c:97-405): pitched buffers,
    get_coefficients for OPTIMIZED, numExecReps consecutive exec calls carrying
    the state; outputs against the reference golden at abs 2^-10."""
    meta = golden_biquad[key + "_meta"]
    cid, form, nch, N, C, S, reps, pitch_b, var_b = (int(v) for v in meta)
    pitch, var_pitch = pitch_b // 4, var_b // 4
    x = golden_biquad[key + "_x"]
    nat = golden_biquad[key + "_coef"]
    args, pin, pout, pvar, pcn, popt = D.biquad_descs(C, N, S, form, nch, pitch=pitch, var_pitch=var_pitch,
                                                      func_style=style)
    coef = nat if style == D.NATC else D.opt_coefficients(nat, form, nch, C)[0]
    xin = np.zeros((reps * N, pitch), np.float32)
    xin[:, :C] = x
    out = np.zeros_like(xin)
    state = np.zeros((S * nv(form if style == D.OPTIMIZED else (D.DF2 if form == D.TIF else form)), var_pitch),
                     np.float32)
    h = D.BiquadHandle()
    assert h.init_check(args, pin, pcn if style == D.NATC else popt, pvar, pout) == D.SUCCESS
    assert h.init(args, pin, pcn if style == D.NATC else popt, pvar, pout) == D.SUCCESS
    xd, od, sd, cd = dev(xin), dev(out), dev(state), dev(coef)
    for r in range(reps):
        st = D.lib().DSPLIB_cascadeBiquad_exec(h.h, xd.data_ptr() + r * N * pitch * 4, cd.data_ptr(),
                                                sd.data_ptr(), od.data_ptr() + r * N * pitch * 4)
        assert st == D.SUCCESS, h.last_error()
    y = host(od)[:, :C]
    assert np.max(np.abs(y - golden_biquad[key + "_y64"])) <= TOL_REF
    if style == D.NATC:
        f = D.DF2 if form == D.TIF else form
        s_ref = np.zeros((S * nv(f), C), np.float32)
        assert np.array_equal(y, oracle.biquad(f, x, nat, s_ref, nch=nch))
        assert np.array_equal(host(sd)[:, :C], s_ref)
    elif form == D.TDF2:  # TDF2 states coincide with scipy's sosfilt zf
        zf = golden_biquad[key + "_zf64"].reshape(S * 2, C)
        assert np.max(np.abs(host(sd)[:, :C] - zf)) <= TOL_REF


@pytest.mark.parametrize("C", [8, 64])
def test_opt_blocks_replayed_from_cuda_graph(C):
    """Block-by-block processing (the numExecReps pattern) captured once in a CUDA
    graph: asynchronous exec calls on device buffers queue kernels only, so a
    sequence of blocks replays as one graph and equals one call on the whole signal."""
    rng = np.random.default_rng(40 + C)
    N, blocks, S = 2048, 4, 4
    x = rng.standard_normal((N * blocks, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, D.DF2, 0, C)
    xd, cd = dev(x), dev(opt)
    yd = torch.zeros_like(xd)
    sd = torch.zeros((2 * S, C), device="cuda")
    args, pin, pout, pvar, pcn, popt = D.biquad_descs(C, N, S, D.DF2, 0)
    h = D.BiquadHandle()
    assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
    h.set_async(True)
    cs = torch.cuda.Stream()
    h.set_stream(cs)
    with torch.cuda.stream(cs):  # one eager pass sets up the launch attributes
        for b in range(blocks):
            assert h.exec(xd[b * N:(b + 1) * N], cd, sd, yd[b * N:(b + 1) * N]) == D.SUCCESS
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=cs):
        for b in range(blocks):
            assert h.exec(xd[b * N:(b + 1) * N], cd, sd, yd[b * N:(b + 1) * N]) == D.SUCCESS
    sd.zero_()
    yd.zero_()
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    st_whole = dev(np.zeros((2 * S, C), np.float32))
    want = host(D.cascade_biquad(xd, cd, st_whole, form=D.DF2, nch=0))
    scale = max(1.0, float(np.abs(want).max()))
    assert np.max(np.abs(host(yd) - want)) <= 1e-4 * scale
    assert np.max(np.abs(host(sd) - host(st_whole))) <= 1e-4 * max(1.0, float(np.abs(host(st_whole)).max()))


@pytest.mark.parametrize("form", FORMS)
def test_opt_pinned_host_buffers_read_in_place(form):
    """Page-locked signal buffers of 32+ channels are read and written by the scan kernel in
    place (no staging copy): identical results to device buffers, state included, and the
    call returns complete even in asynchronous mode."""
    rng = np.random.default_rng(50 + form)
    N, C, S = 5000, 64, 3
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, form, 0, C)
    st0 = (rng.standard_normal((S * nv(form), C)) * 0.1).astype(np.float32)
    sd = dev(st0)
    want = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=0))
    hx, hy = torch.from_numpy(x).pin_memory(), torch.zeros(N, C).pin_memory()
    hs, hc = torch.from_numpy(st0.copy()).pin_memory(), torch.from_numpy(opt).pin_memory()
    args, pin, pout, pvar, _, popt = D.biquad_descs(C, N, S, form, 0)
    h = D.BiquadHandle()
    assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
    assert h.set_async(True) == D.SUCCESS  # settings apply after the first init
    D.cascade_biquad(hx, hc, hs, form=form, nch=0, out=hy, handle=h)
    assert np.array_equal(hy.numpy(), want)
    assert np.array_equal(hs.numpy(), host(sd))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("C,pinned,in_place", [(40, True, False), (16, True, False), (40, True, True),
                                               (40, False, False)])
def test_opt_large_host_signals(form, C, pinned, in_place):
    """Page-locked host signals of 4 MB or more are copied in, filtered and copied out in
    blocks of rows on three streams, each block starting from the state the previous one
    left (lane kernel, per-channel kernel, in place); pageable ones are staged whole.
    Outputs and final state equal the FP64 oracle to the scan's accuracy, and the call
    returns complete in asynchronous mode."""
    rng = np.random.default_rng(60 + form + C)
    N, S = (30001 if C == 40 else 70001), 3  # 4.5 - 4.8 MB of input, the last block ragged
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, form, 0, C)
    st0 = (rng.standard_normal((S * nv(form), C)) * 0.1).astype(np.float32)
    hx, hs, hc = torch.from_numpy(x.copy()), torch.from_numpy(st0.copy()), torch.from_numpy(opt)
    if pinned:
        hx, hs, hc = hx.pin_memory(), hs.pin_memory(), hc.pin_memory()
    hy = hx if in_place else (torch.zeros(N, C).pin_memory() if pinned else torch.zeros(N, C))
    args, pin, pout, pvar, _, popt = D.biquad_descs(C, N, S, form, 0)
    h = D.BiquadHandle()
    assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
    assert h.set_async(True) == D.SUCCESS
    D.cascade_biquad(hx, hc, hs, form=form, nch=0, out=hy, handle=h)
    y32, st32, y64, _ = oracle_run(form, x, nat, st0, 0)
    if form != D.TIF:
        check_accuracy(hy.numpy(), y32, y64, (form, C))
    else:  # the FP64 truth of TIF runs from a zero state: compare with the FP32 restatement
        assert np.max(np.abs(hy.numpy() - y32)) <= TOL_REF * max(1.0, float(np.max(np.abs(y32))))
    assert np.max(np.abs(hs.numpy() - st32)) <= 1e-3 * max(1.0, float(np.max(np.abs(st32))))


@pytest.mark.parametrize("form", [D.DF1, D.DF2, D.TDF2])
def test_natc_host_signals_pipelined_bitexact(form):
    """NATC on page-locked host signals through the block pipeline (sequential kernel per
    block, state chained) stays bit-exact to the natural-C restatement, outputs and final
    state."""
    rng = np.random.default_rng(70 + form)
    N, C, S = 22001, 48, 4  # 4.2 MB of input: two blocks
    x = rng.uniform(-1, 1, size=(N, C)).astype(np.float32)
    nat = stable_sections(rng, C, S)
    st = (rng.standard_normal((S * nv(form), C)) * 0.1).astype(np.float32)
    s_ref = st.copy()
    want = oracle.biquad(form, x, nat, s_ref, nch=1)
    hx, hn = torch.from_numpy(x).pin_memory(), torch.from_numpy(nat).pin_memory()
    hs, hy = torch.from_numpy(st.copy()).pin_memory(), torch.zeros(N, C).pin_memory()
    D.cascade_biquad(hx, hn, hs, form=form, nch=1, func_style=D.NATC, out=hy)
    assert np.array_equal(hy.numpy(), want)
    assert np.array_equal(hs.numpy(), s_ref)


def test_opt_async_level2_pinned_calls_overlap():
    """DSPLIB_gpu_setAsync(h, 2): calls on page-locked host buffers read and written in place
    return once queued.  Three handles on three streams filter independent signals
    concurrently; once each stream is synchronized, every output and final state equals the
    synchronous call's."""
    rng = np.random.default_rng(71)
    N, C, S = 8192, 32, 4
    nat = stable_sections(rng, 1, S)
    opt, _ = D.opt_coefficients(nat, D.DF2, 0, C)
    hc = torch.from_numpy(opt).pin_memory()
    runs = []
    for k in range(3):
        x = rng.standard_normal((N, C)).astype(np.float32)
        st0 = (rng.standard_normal((2 * S, C)) * 0.1).astype(np.float32)
        sd = dev(st0)
        want = host(D.cascade_biquad(dev(x), dev(opt), sd, form=D.DF2, nch=0))
        args, pin, pout, pvar, _, popt = D.biquad_descs(C, N, S, D.DF2, 0)
        h, stream = D.BiquadHandle(), torch.cuda.Stream()
        assert h.init(args, pin, popt, pvar, pout) == D.SUCCESS
        assert h.set_stream(stream) == D.SUCCESS and h.set_async(2) == D.SUCCESS
        hx, hy = torch.from_numpy(x).pin_memory(), torch.zeros(N, C).pin_memory()
        hs = torch.from_numpy(st0.copy()).pin_memory()
        runs.append((h, stream, hx, hy, hs, want, host(sd)))
    for h, stream, hx, hy, hs, _, _ in runs:
        assert h.exec(hx, hc, hs, hy) == D.SUCCESS
    for h, stream, hx, hy, hs, want, st_want in runs:
        stream.synchronize()
        assert np.array_equal(hy.numpy(), want)
        assert np.array_equal(hs.numpy(), st_want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("nch", [0, 1])
def test_get_coefficients_on_device_buffers_matches_host(form, nch):
    """get_coefficients with device buffers runs the transform on the GPU: bit for bit the
    host function's result (TIF transform with its 7-stage group gains, per-channel
    reorder), the padding between channel columns left untouched."""
    import ctypes

    from c7x_dsplib_b200 import BufParams2D, bp, lib

    if form != D.TIF and not nch:
        pytest.skip("DF forms with shared coefficients have no optimized layout (INVALID_VALUE)")
    rng = np.random.default_rng(70 + form * 2 + nch)
    for S, C in [(1, 1), (4, 33), (7, 5), (8, 17), (15, 3), (22, 40)]:
        nat = stable_sections(rng, C if nch else 1, S)
        nat[0, 0] = 0.0  # b0 = 0: the reciprocal is taken as 0
        want, popt = D.opt_coefficients(nat, form, nch, C)
        pcn = bp(D.FLOAT32, S * 5, C if nch else 1, S * 5 * 4)
        opt_d = torch.full((popt.dim_y * popt.stride_y // 4,), 3.0, device="cuda")
        st = lib().DSPLIB_cascadeBiquad_get_coefficients(form, int(nch), ctypes.byref(pcn), ctypes.byref(popt),
                                                         dev(nat).data_ptr(), opt_d.data_ptr())
        assert st == D.SUCCESS
        got = host(opt_d)
        if nch:  # columns beyond C keep what the caller had there
            got2 = got.reshape(popt.dim_y, popt.stride_y // 4)
            assert np.all(got2[:, C:] == 3.0)
            got2[:, C:] = want.reshape(popt.dim_y, -1)[:, C:]
        assert np.array_equal(got, want), (S, C)


def sections_at_radius(rng, rows, S, r):
    """Natural [rows, S*5]: every pole pair at radius r (angle U[0.05, pi - 0.05]), zeros on
    the unit circle, each section scaled to unit gain at its pole angle."""
    out = np.zeros((rows, S, 5))
    for r_ in range(rows):
        for s in range(S):
            th, ph = rng.uniform(0.05, np.pi - 0.05), rng.uniform(0, np.pi)
            b = np.array([1.0, -2 * np.cos(ph), 1.0])
            a = np.array([1.0, -2 * r * np.cos(th), r * r])
            z = np.exp(-1j * th * np.arange(3))
            g = 1.0 / max(abs(np.dot(b, z) / np.dot(a, z)), 1e-12)
            out[r_, s] = [g * b[0], g * b[1], g * b[2], a[1], a[2]]
    return out.reshape(rows, S * 5).astype(np.float32)


@pytest.mark.parametrize("radius", [0.99, 0.995, 0.999])
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("C", [4, 64])
def test_opt_scan_poles_near_unit_circle(radius, form, C):
    """Poles at radius 0.99 / 0.995 / 0.999, where the transition powers are formed in FP64:
    the per-channel scan (4 channels) and the lane scan (64 channels, clustered CTAs) over
    signals of several windows, outputs and final states against FP64.  Bound: the one of
    check_accuracy (1e-4, or 4x the sequential FP32 recursion's own error, which grows like
    1 / (1 - r) here)."""
    rng = np.random.default_rng(int(radius * 1e4) + form * 10 + C)
    N, S = 20000, 3
    x = rng.standard_normal((N, C)).astype(np.float32)
    nat = sections_at_radius(rng, 1, S, radius)
    st = np.zeros((S * nv(form), C), np.float32)
    opt, _ = D.opt_coefficients(nat, form, 0, C)
    sd = dev(st)
    y = host(D.cascade_biquad(dev(x), dev(opt), sd, form=form, nch=0))
    y32, st32, y64, s64 = oracle_run(form, x, nat, st, 0)
    check_accuracy(y, y32, y64, (radius, form, C))
    if form != D.TIF:  # TIF keeps its own state variables (no FP64 counterpart)
        sgot = host(sd).astype(np.float64)
        seq = np.abs(st32 - s64).max() / max(np.abs(s64).max(), 1e-30)
        err = np.abs(sgot - s64).max() / max(np.abs(s64).max(), 1e-30)
        assert err <= max(1e-4, 4 * seq), (err, seq)
