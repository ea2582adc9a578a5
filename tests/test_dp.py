"""Data-parallel training over patches (two ranks on the gloo backend, CPU): each rank
differentiates the loss of its shard (normalised by the global batch) and the table
gradients are summed with one all-reduce. The sum equals the full-batch gradient; pixel
gradients stay on their rank. The binary64 restatement stands in for the GPU kernels,
whose gradients the GPU tests compare with it."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from neo_fft_b200.autograd import allreduce_grad, shard
from neo_fft_b200.plan import DFTConfig

N, S = 5, 48
CFG = dict(block=16, overlap=8, ftype=0, sigma=4.0)


def _data():
    from tests.synth import noisy_patches
    noisy, clean = noisy_patches(N, S, 91)
    return torch.from_numpy(noisy).double(), torch.from_numpy(clean).double()


def _grads(o, table, noisy, clean, idx):
    x = noisy[list(idx)].clone().requires_grad_()
    t = table.clone().requires_grad_()
    loss = ((o.forward(x, t) - clean[list(idx)]) ** 2).sum() / clean.numel()
    loss.backward()
    return x.grad, t.grad


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.dft_fp64 import DFTTestFP64
        o = DFTTestFP64(S, S, DFTConfig(**CFG))
        noisy, clean = _data()
        table = torch.from_numpy(o.uniform_table()).double()
        idx = shard(N, rank, world)
        gx, gt = _grads(o, table, noisy, clean, idx)
        allreduce_grad(gt)
        out[rank] = (list(idx), gx.numpy(), gt.numpy())
    finally:
        dist.destroy_process_group()


def test_shards_cover_the_batch():
    for n in range(1, 12):
        for world in range(1, 5):
            got = [i for r in range(world) for i in shard(n, r, world)]
            assert got == list(range(n))


def test_table_gradient_allreduce_equals_full_batch(ref):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)

    from oracle.dft_fp64 import DFTTestFP64
    o = DFTTestFP64(S, S, DFTConfig(**CFG))
    noisy, clean = _data()
    table = torch.from_numpy(o.uniform_table()).double()
    gx, gt = _grads(o, table, noisy, clean, range(N))
    for r in range(world):
        idx, rgx, rgt = out[r]
        np.testing.assert_allclose(rgt, gt.numpy(), rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(rgx, gx.numpy()[idx], rtol=1e-12, atol=1e-15)
