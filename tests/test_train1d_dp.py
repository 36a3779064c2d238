"""CPU: data-parallel closure training's exchange step (gradient all-reduce over trajectories), gloo, 2 ranks."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from weno_sr_publishing_b200 import train1d as T


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        m = T.ClosureMLP(seed=83, dtype=torch.float32)
        for k, p in enumerate(m.parameters()):
            p.grad = torch.full_like(p, float(rank + 1) * (k + 1))
        T.allreduce_gradients(m)
        grads = torch.cat([p.grad.reshape(-1) for p in m.parameters()]).numpy()
        mean = T._allreduce_mean(float(rank + 1), "cpu")
        out[rank] = (grads, mean, T._world())
    finally:
        dist.destroy_process_group()


def test_gradient_allreduce_two_ranks():
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    g0, m0, w0 = out[0]
    g1, m1, w1 = out[1]
    assert w0 == (2, 0) and w1 == (2, 1)
    assert np.array_equal(g0, g1)
    sizes = [p.numel() for p in T.ClosureMLP(seed=83).parameters()]
    expect = np.concatenate([np.full(n, 1.5 * (k + 1)) for k, n in enumerate(sizes)])
    assert np.allclose(g0, expect)
    assert m0 == m1 == 1.5


def test_single_process_is_a_no_op():
    m = T.ClosureMLP(seed=1)
    for p in m.parameters():
        p.grad = torch.ones_like(p)
    T.allreduce_gradients(m)
    assert all(float(p.grad.sum()) == p.numel() for p in m.parameters())
    assert T._world() == (1, 0)


def test_batch_must_split_evenly_over_ranks(tmp_path):
    cfg = T.TrainConfig(out_dir=tmp_path, steps=1, batch=6, device="cpu")
    # one process: a batch of 6 trajectories is fine for the split check, the CUDA step is not reached here
    with pytest.raises(ValueError):
        T.train(T.TrainConfig(out_dir=tmp_path, steps=1, batch=5, device="cpu"))
    del cfg
