"""DSPLIB_gpu_firBiquadBatched_bwdStaticScratch (the filter-bank adjoint with
its scratch in a fixed array inside the library) against
DSPLIB_gpu_firBiquadBatched_bwd with a caller scratch buffer.

Kept in a file of its own, collected last, and written to pass both alone and
after the other GPU tests: it builds every input itself and relies on no state
a previous test may have left (the static array carries nothing from one call
to the next that the adjoint reads)."""
import ctypes

import numpy as np
import pytest


def _case(seed):
    rng = np.random.default_rng(seed)
    lengths = [3000, 17, 9000, 512, 4100, 64]
    taps = [31, 17, 200, 1, 64, 8]
    stages = [3, 1, 5, 0, 2, 4]
    x = rng.standard_normal(sum(lengths)).astype(np.float32)
    h = np.concatenate([rng.standard_normal(T) / np.sqrt(T) for T in taps]).astype(np.float32)
    c = []
    for S in stages:
        for _ in range(S):
            r, th = rng.uniform(0.3, 0.9), rng.uniform(0.1, 3.0)
            c += [0.5, 0.2, 0.1, -2 * r * np.cos(th), r * r]
    return lengths, taps, stages, x, h, np.asarray(c, np.float32)


@pytest.mark.gpu
def test_static_scratch_adjoint_matches_buffer_adjoint_twice():
    import torch

    from c7x_dsplib_b200 import SUCCESS, lib
    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    lengths, taps, stages, x, h, c = _case(21)
    bank = RaggedFilterBank(lengths, taps, stages)
    dev = "cuda"
    xt, ht, ct = (torch.from_numpy(a).to(dev) for a in (x, h, c))
    y = torch.empty(bank.sizes[0], device=dev)
    work = torch.empty(bank.sizes[3], device=dev)
    bank.forward_raw(xt, ht, ct, y, work)
    gy = torch.randn(bank.sizes[0], device=dev, generator=torch.Generator(dev).manual_seed(5))
    want = [torch.empty_like(xt), torch.empty_like(ht), torch.empty_like(ct)]
    scratch = torch.empty(bank.sizes[4], device=dev)
    bank.backward_raw(xt, ht, ct, work, gy, *want, scratch)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):  # two calls in a row reuse the same static array
        got = [torch.full_like(xt, 7.0), torch.full_like(ht, 7.0), torch.full_like(ct, 7.0)]
        st = lib().DSPLIB_gpu_firBiquadBatched_bwdStaticScratch(
            bank._plan, xt.data_ptr(), ht.data_ptr(), ct.data_ptr(), work.data_ptr(), gy.data_ptr(),
            got[0].data_ptr(), got[1].data_ptr(), got[2].data_ptr(), stream)
        assert st == SUCCESS
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            assert torch.equal(g, w)  # the adjoint is bitwise repeatable: same inputs, same bits


@pytest.mark.gpu
def test_static_scratch_rejects_plans_beyond_its_size():
    import torch

    from c7x_dsplib_b200 import ERR_BUFFER_TOO_SMALL, lib
    from c7x_dsplib_b200.filterbank import RaggedFilterBank

    # 4 channels of 1M samples: the adjoint needs > 4M floats of scratch (the gradient
    # w.r.t. the FIR output alone is 4M), the array holds 4M
    bank = RaggedFilterBank([1 << 20] * 4, [8] * 4, [1] * 4)
    assert bank.sizes[4] > (4 << 20)
    d = torch.zeros(16, device="cuda")
    p = d.data_ptr()
    st = lib().DSPLIB_gpu_firBiquadBatched_bwdStaticScratch(bank._plan, p, p, p, p, p, p, p, p, None)
    assert st == ERR_BUFFER_TOO_SMALL
    torch.cuda.synchronize()
    assert torch.count_nonzero(d).item() == 0  # nothing was queued
