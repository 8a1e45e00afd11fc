"""Multi-rank path on CPU: two gloo ranks shard a batch of problems, each
convolves its slice through the library's C ABI (host replay build), and the
gathered result equals the single-rank one; the timing reduction is the max
over ranks."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

from conftest import ROOT

R = importlib.import_module("c-permutation-avoiding-convolution_b200.replicas")


def test_shard_covers_batch():
    for batch in (1, 2, 5, 1024, 4160):
        for world in (1, 2, 3, 8):
            parts = [R.shard(batch, world, r) for r in range(world)]
            covered = [i for s in parts for i in range(s.start, s.stop)]
            assert covered == list(range(batch))
            sizes = [s.stop - s.start for s in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        R.shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import torch

    import parity as P
    pac = importlib.import_module("c-permutation-avoiding-convolution_b200")
    L = pac.load(emulate=True)
    g = np.random.default_rng(123)
    batch, dims = 5, (256,)
    x = g.standard_normal((batch,) + dims) + 1j * g.standard_normal((batch,) + dims)
    h = g.standard_normal(dims) + 1j * g.standard_normal(dims)
    sl = R.shard(batch, world, rank)
    mine = P.native_conv(L, dims, sl.stop - sl.start, 2, 0, x[sl], h)
    # gather for the check only (the product path never gathers)
    buf = torch.zeros((batch,) + dims, dtype=torch.complex128)
    buf[sl] = torch.from_numpy(mine)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    full = sum(parts).numpy()
    t = R.max_over_ranks(1.0 + rank, dist)
    dist.barrier()
    if rank == 0:
        np.save(os.path.join(out_dir, "full.npy"), full)
        np.save(os.path.join(out_dir, "t.npy"), np.array([t]))
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    tmp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                        start_method="spawn", join=True)
    full = np.load(tmp_path / "full.npy")
    t = np.load(tmp_path / "t.npy")[0]
    assert t == 2.0
    import parity as P
    import importlib as il
    pac = il.import_module("c-permutation-avoiding-convolution_b200")
    L = pac.load(emulate=True)
    g = np.random.default_rng(123)
    x = g.standard_normal((5, 256)) + 1j * g.standard_normal((5, 256))
    h = g.standard_normal(256) + 1j * g.standard_normal(256)
    ref = P.native_conv(L, (256,), 5, 2, 0, x, h)
    assert np.array_equal(full, ref)
    assert P.crel(full, P.fftconv(x, h[None], (1,))) < P.TOL
