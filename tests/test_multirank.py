"""Multi-rank host logic on CPU (gloo, world size 2): each rank filters its own
block of channels with no data-path collective; gathering the blocks gives the
single-process result; timing agrees on the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from c7x_dsplib_b200.shard import balance_ragged, channel_block, max_over_ranks


def test_channel_block_partitions():
    for C in (1, 7, 32, 4096):
        for world in (1, 2, 3, 8):
            blocks = [channel_block(r, world, C) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == C
            for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
                assert a1 == b0
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


def test_balance_ragged():
    rng = np.random.default_rng(0)
    lengths = np.exp(rng.uniform(np.log(256), np.log(262144), 2048)).astype(int)
    parts = balance_ragged(lengths, 8)
    assert sorted(i for p in parts for i in p) == list(range(2048))
    loads = [int(lengths[p].sum()) for p in parts]
    assert max(loads) <= min(loads) + int(lengths.max())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, result_dir):
    import torch
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(123)  # same inputs on every rank
    C, N, T = 10, 300, 17
    x = rng.standard_normal((C, N)).astype(np.float32)
    h = rng.standard_normal((C, T)).astype(np.float32)
    c0, c1 = channel_block(rank, world, C)
    y_local = oracle.fir(np.ascontiguousarray(x[c0:c1]), np.ascontiguousarray(h[c0:c1]), T, nch=1)
    # gather the blocks (verification only: the filtering itself needed no exchange);
    # C = 10 over 2 ranks gives equal blocks, so all_gather applies directly
    buf = [torch.zeros((c1 - c0, N - T + 1)) for _ in range(world)]
    dist.all_gather(buf, torch.from_numpy(np.ascontiguousarray(y_local)))
    y = torch.cat(buf).numpy()
    elapsed = max_over_ranks(0.001 * (rank + 1), dist)
    if rank == 0:
        np.save(os.path.join(result_dir, "y.npy"), y)
        np.save(os.path.join(result_dir, "t.npy"), np.array([elapsed]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_gloo_two_ranks_match_single_process(tmp_path):
    import oracle

    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    rng = np.random.default_rng(123)
    C, N, T = 10, 300, 17
    x = rng.standard_normal((C, N)).astype(np.float32)
    h = rng.standard_normal((C, T)).astype(np.float32)
    assert np.array_equal(np.load(tmp_path / "y.npy"), oracle.fir(x, h, T, nch=1))
    assert float(np.load(tmp_path / "t.npy")[0]) == pytest.approx(0.002)
