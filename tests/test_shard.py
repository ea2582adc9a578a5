"""Single-clip sharding by output-frame ranges (neo_fft_b200/shard.py), on the CPU with
two gloo ranks: every output frame is produced by exactly one rank, and the window each
rank uses for it is the host layer's selection over the whole clip (filter.hpp:266-305,
433-452); the union of a rank's windows is what it loads. tests/test_gpu_shard.py runs
the ranges through the GPU path."""
import os

import pytest
import torch.multiprocessing as mp

from neo_fft_b200.shard import frame_ranges, rank_sources, window
from neo_fft_b200.temporal import centred_slots, fft3d_slots, temporal_blocks

KINDS = [("fft3d", 3, 0), ("fft3d", 2, 0), ("fft3d", 5, 0), ("dft0", 5, 0), ("dft1", 5, 0), ("dft1", 5, 2),
         ("dft1", 3, 1), ("single", 1, 0)]


def test_frame_ranges_cover_each_frame_once():
    for n in (0, 1, 7, 60, 121):
        for world in (1, 2, 3, 8):
            r = frame_ranges(n, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("kind,size,overlap", KINDS)
def test_windows_are_the_host_layers(kind, size, overlap):
    N = 23
    for n in range(N):
        w = window(kind, n, N, size, overlap)
        if kind == "fft3d":
            assert list(w.sources) == fft3d_slots(n, N, size)
        elif kind == "dft0":
            assert list(w.sources) == centred_slots(n, N, size)
        elif kind == "dft1":
            blocks = temporal_blocks(n, N, size, overlap)
            assert list(w.sources) == [s for b in blocks for s in b["slots"]]
            assert list(w.targets) == [b["target"] for b in blocks]
        else:
            assert w.sources == (n,)


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        N = 37
        res = {}
        for kind, size, overlap in KINDS:
            rng = frame_ranges(N, world)[rank]
            produced = torch.zeros(N, dtype=torch.int64)
            produced[rng[0]:rng[1]] = 1
            dist.all_reduce(produced)  # how many ranks produce each frame
            srcs = rank_sources(kind, rng, N, size, overlap)
            need = set()
            for n in range(*rng):
                need.update(window(kind, n, N, size, overlap).sources)
            res[(kind, size, overlap)] = (produced.tolist(), srcs == sorted(need), rng, srcs)
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_two_ranks_produce_every_frame_once():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for key in res[0]:
        produced, ok, rng0, srcs0 = res[0][key]
        assert produced == [1] * 37, key
        assert ok and res[1][key][1]
        # the ranks' loads overlap only in the halo their windows reach
        rng1, srcs1 = res[1][key][2], res[1][key][3]
        assert rng0[1] == rng1[0]
        kind, size, _ = key
        if kind == "single":
            assert not set(srcs0) & set(srcs1)
        if kind == "fft3d":
            assert max(srcs0) == rng0[1] - 1 + (size - 1) // 2 and min(srcs1) == rng1[0] - size // 2
