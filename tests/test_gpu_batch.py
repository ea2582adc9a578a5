"""Batched/persistent form: one persistent launch per block shape over many planes of
different sizes and plans (luma+chroma, mixed resolutions) equals per-plane
processing bit for bit, with and without CUDA-graph replay."""
import numpy as np
import pytest

from neo_fft_b200.plan import Batch, DFTConfig, FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu


def test_batch_mixed_planes_equal_per_plane(cuda):
    dft = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])
    f16 = SampleFormat(16)
    sizes = [(192, 108), (96, 54), (96, 54), (320, 180), (160, 90), (160, 90), (128, 72)]
    plans = {s: Plan(s[0], s[1], f16, dft) for s in set(sizes)}
    f8 = SampleFormat(8)
    fplan = Plan(200, 120, f8, FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0))
    items, refs = [], []
    for i, (w, h) in enumerate(sizes):
        src = cuda.from_numpy(plane(h, w, 16, False, seed=(7, 0, i))).cuda()
        items.append((plans[(w, h)], src, cuda.empty_like(src)))
    for i in range(3):
        src = cuda.from_numpy(plane(120, 200, 8, False, seed=(7, 1, i))).cuda()
        items.append((fplan, src, cuda.empty_like(src)))
    for p, s, d in items:
        r = cuda.empty_like(s)
        p.process_at([s], r)
        refs.append(r)
    b = Batch(items)
    b.launch()
    b.sync_status()
    for (p, s, d), r in zip(items, refs):
        assert cuda.equal(d, r)
    for (p, s, d) in items:
        d.zero_()
    b.launch(graph=True)
    b.launch(graph=True)
    cuda.cuda.synchronize()
    for (p, s, d), r in zip(items, refs):
        assert cuda.equal(d, r)


def test_batch_rejects_multi_frame_plans(cuda):
    p = Plan(64, 48, SampleFormat(8), DFTConfig(tbsize=3))
    s = cuda.zeros((48, 64), dtype=cuda.uint8, device="cuda")
    with pytest.raises(ValueError, match="batch items must be single-frame plans"):
        Batch([(p, s, cuda.empty_like(s))])


@pytest.mark.parametrize("fmt,cfg,size", [
    (SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0), (256, 256)),
    (SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8]), (320, 180)),
    (SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0, sharpen=0.3), (200, 120)),
    (SampleFormat(10), DFTConfig(block=12, overlap=9, ftype=1, sigma=6.0), (150, 98)),
], ids=["f32-dft16", "u16-dft16", "u8-fft3d32", "u10-dft12"])
def test_multi_plane_launch_equals_per_plane(cuda, fmt, cfg, size):
    """nf_plan_process_planes_device over 35 planes (two launches: 32 + 3), some of them
    strided views, equals one nf_plan_process_device call per plane bit for bit."""
    w, h = size
    p = Plan(w, h, fmt, cfg)
    srcs = []
    for i in range(35):
        a = cuda.from_numpy(plane(h, w, fmt.bits, fmt.floating, seed=(9, 0, i))).cuda()
        if i % 4 == 1:  # padded rows: stride larger than the width
            big = cuda.zeros((h, w + 24), dtype=a.dtype, device=a.device)
            big[:, :w] = a
            a = big[:, :w]
        srcs.append(a)
    outs = [cuda.empty((h, w), dtype=s.dtype, device=s.device) for s in srcs]
    p.process_planes(srcs, outs)
    for s, o in zip(srcs, outs):
        r = cuda.empty_like(o)
        p.process_at([s], r)
        assert cuda.equal(o, r)
    p.sync_status()


def test_multi_plane_launch_rejects_temporal_plans(cuda):
    p = Plan(64, 48, SampleFormat(8), FFT3DConfig(bw=16, bh=16, bt=3))
    a = cuda.zeros((48, 64), dtype=cuda.uint8, device="cuda")
    with pytest.raises(ValueError, match="single-frame plans"):
        p.process_planes([a], [cuda.empty_like(a)])


def test_batch_every_geometry_equals_per_plane(cuda):
    """Each candidate strip geometry of a batch (the first launch times them all) writes
    the per-plane outputs bit for bit; the tuned choice is one of them."""
    dft = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0)
    f16 = SampleFormat(16)
    sizes = [(640, 360), (320, 180), (320, 180)]
    plans = {s: Plan(s[0], s[1], f16, dft) for s in set(sizes)}
    items, refs = [], []
    for i, (w, h) in enumerate(sizes * 2):
        src = cuda.from_numpy(plane(h, w, 16, False, seed=(8, 0, i))).cuda()
        items.append((plans[(w, h)], src, cuda.empty_like(src)))
        r = cuda.empty_like(src)
        plans[(w, h)].process_at([src], r)
        refs.append(r)
    b = Batch(items)
    assert b.geometry == -1 and 1 <= b.geometry_count <= 3
    b.launch()
    cuda.cuda.synchronize()
    assert 0 <= b.geometry < b.geometry_count
    for (p, s, d), r in zip(items, refs):
        assert cuda.equal(d, r)
    for g in range(b.geometry_count):
        b.select_geometry(g)
        for graph in (False, True):
            for (_, _, d) in items:
                d.zero_()
            b.launch(graph=graph)
            cuda.cuda.synchronize()
            for (p, s, d), r in zip(items, refs):
                assert cuda.equal(d, r), (g, graph)
    with pytest.raises(ValueError, match="geometry index"):
        b.select_geometry(b.geometry_count)


@pytest.mark.parametrize("fmt,cfg", [
    (SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0)),
    (SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])),
    (SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0)),
    (SampleFormat(10), DFTConfig(block=12, overlap=9, ftype=1, sigma=6.0)),
    (SampleFormat(32, True), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, sigma=3.0, sharpen=0.3)),
])
def test_batch_bulk_tensor_staging(cuda, fmt, cfg):
    """Batched planes stage the interior block rows of their strips through bulk-tensor
    copies prefetched one block row ahead; a plane whose base address and row stride are
    not multiples of 16 bytes is staged by direct loads in the same batch. Every output
    equals the per-plane call bit for bit, directly and from the graph, with no error."""
    w, h = 640, 360
    plan = Plan(w, h, fmt, cfg)
    items = []
    for i in range(3):
        src = cuda.from_numpy(plane(h, w, fmt.bits, fmt.floating, seed=(9, i))).cuda()
        items.append((plan, src, cuda.empty_like(src)))
    wide = cuda.from_numpy(plane(h, w + 1, fmt.bits, fmt.floating, seed=(9, 7))).cuda()
    view = wide[:, 1:]  # one sample into each row of a w + 1 sample buffer
    items.append((plan, view, cuda.empty((h, w), dtype=view.dtype, device=view.device)))
    refs = []
    for p, s, d in items:
        r = cuda.empty((h, w), dtype=s.dtype, device=s.device)
        p.process_at([s], r)
        refs.append(r)
    b = Batch(items)
    assert b.mapped_planes == 3
    b.launch()
    b.sync_status()
    assert b.mapped_planes == 3  # every candidate geometry maps the aligned planes
    for (p, s, d), r in zip(items, refs):
        assert cuda.equal(d, r)
    for (_, _, d) in items:
        d.zero_()
    b.launch(graph=True)
    b.launch(graph=True)
    cuda.cuda.synchronize()
    b.sync_status()
    for (p, s, d), r in zip(items, refs):
        assert cuda.equal(d, r)
