"""Temporal clips in batched form (nf_clip_batch): every output frame equals one
nf_plan_process_device call with the host layer's frame selection bit for bit — FFT3D
bt 2..5 with temporal.fft3d_slots (frames n-bt/2 .. n+(bt-1)/2, single frame at the clip
edges), DFTTest tmode 1 with temporal.temporal_blocks — and the reference core."""
import numpy as np
import pytest

from neo_fft_b200.plan import ClipBatch, DFTConfig, FFT3DConfig, Plan, SampleFormat
from neo_fft_b200.temporal import fft3d_slots, temporal_blocks
from tests.synth import plane

pytestmark = pytest.mark.gpu


def _clip(cuda, n, h, w, fmt, seed):
    return [cuda.from_numpy(plane(h, w, fmt.bits, fmt.floating, seed=(seed, 0, f))).cuda() for f in range(n)]


def _per_frame(cuda, plan, frames):
    outs = []
    for t in range(len(frames)):
        o = cuda.empty_like(frames[t])
        plan.process_at([frames[j] for j in fft3d_slots(t, len(frames), plan.temporal_size)], o)
        outs.append(o)
    return outs


@pytest.mark.parametrize("bt", [2, 3, 4, 5])
def test_clip_batch_equals_per_frame(cuda, bt):
    fmt = SampleFormat(8)
    plan = Plan(200, 120, fmt, FFT3DConfig(bw=32, bh=32, ow=16, oh=16, bt=bt, sigma=3.0))
    frames = _clip(cuda, 9, 120, 200, fmt, 60 + bt)
    dsts = [cuda.empty_like(f) for f in frames]
    ClipBatch([(plan, frames, dsts)]).launch()
    for got, exp in zip(dsts, _per_frame(cuda, plan, frames)):
        assert cuda.equal(got, exp)
    plan.sync_status()


def test_clip_batch_mixed_clips_enhancement_and_graph(cuda):
    """Luma and chroma plans of several resolutions (10-bit, 48x48 blocks, sharpen and
    dehalo), clips of different lengths including one shorter than bt; graph replay."""
    cfg = FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3, dehalo=0.5)
    y10, c10 = SampleFormat(10), SampleFormat(10, chroma=True)
    sizes = [(256, 144, 7), (192, 108, 5), (160, 96, 2)]
    clips = []
    for i, (w, h, n) in enumerate(sizes):
        for fmt, (pw, ph) in ((y10, (w, h)), (c10, (w // 2, h // 2))):
            p = Plan(pw, ph, fmt, cfg)
            fr = _clip(cuda, n, ph, pw, fmt, 70 + i)
            clips.append((p, fr, [cuda.empty_like(f) for f in fr]))
    batch = ClipBatch(clips)
    for graph in (False, True, True):
        for _, _, d in clips:
            for t in d:
                t.fill_(0)
        batch.launch(graph=graph)
        for p, fr, d in clips:
            for got, exp in zip(d, _per_frame(cuda, p, fr)):
                assert cuda.equal(got, exp)
    for p, _, _ in clips:
        p.sync_status()


def test_clip_batch_matches_reference(cuda, ref):
    fmt = SampleFormat(16)
    cfg = FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=3, sigma=600.0)
    w, h, n = 96, 64, 5
    plan = Plan(w, h, fmt, cfg)
    host = [plane(h, w, 16, False, seed=(80, 0, f)) for f in range(n)]
    frames = [cuda.from_numpy(x).cuda() for x in host]
    dsts = [cuda.empty_like(f) for f in frames]
    ClipBatch([(plan, frames, dsts)]).launch()
    rp = ref.RefPlan(w, h, fmt, cfg)
    for t in range(n):
        exp = rp.process([host[j] for j in fft3d_slots(t, n, 3)])
        assert np.array_equal(dsts[t].cpu().numpy(), exp)


def _per_frame_dft(cuda, plan, frames):
    outs = []
    for t in range(len(frames)):
        blocks = temporal_blocks(t, len(frames), plan.temporal_size, 0)
        o = cuda.empty_like(frames[t])
        plan.process_at([frames[j] for b in blocks for j in b["slots"]], o, targets=[b["target"] for b in blocks])
        outs.append(o)
    return outs


@pytest.mark.parametrize("fmt,cfg,n", [
    (SampleFormat(32, True), DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1, sigma=8.0), 12),
    (SampleFormat(16), DFTConfig(block=16, overlap=8, tbsize=3, temporal_mode=1, ftype=0, sigma=6.0,
                                 slocation=[0, 4, 0.5, 8, 1, 12]), 7),
    (SampleFormat(8), DFTConfig(block=8, overlap=4, tbsize=2, temporal_mode=1, ftype=2, sigma=0.7, zmean=0), 5),
    (SampleFormat(10), DFTConfig(block=10, overlap=5, tbsize=4, temporal_mode=1, ftype=0, sigma=5.0), 6),
], ids=["f32-t5-b12", "u16-t3-b16-curve", "u8-t2-b8", "u10-t4-b10"])
def test_dfttest_clip_batch_equals_per_frame(cuda, fmt, cfg, n):
    w, h = 150, 98
    plan = Plan(w, h, fmt, cfg)
    frames = _clip(cuda, n, h, w, fmt, 95)
    dsts = [cuda.empty_like(f) for f in frames]
    batch = ClipBatch([(plan, frames, dsts)])
    for graph in (False, True):
        for d in dsts:
            d.fill_(0)
        batch.launch(graph=graph)
        for got, exp in zip(dsts, _per_frame_dft(cuda, plan, frames)):
            assert cuda.equal(got, exp)
    plan.sync_status()


def test_dfttest_clip_batch_matches_reference(cuda, ref):
    fmt = SampleFormat(32, True)
    cfg = DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1, sigma=8.0)
    w, h, n = 64, 48, 7
    plan = Plan(w, h, fmt, cfg)
    host = [plane(h, w, 32, True, seed=(96, 0, f)) for f in range(n)]
    frames = [cuda.from_numpy(x).cuda() for x in host]
    dsts = [cuda.empty_like(f) for f in frames]
    ClipBatch([(plan, frames, dsts)]).launch()
    rp = ref.RefPlan(w, h, fmt, cfg)
    for t in range(n):
        blocks = temporal_blocks(t, n, 5, 0)
        exp = rp.process([host[j] for b in blocks for j in b["slots"]], targets=[b["target"] for b in blocks])
        assert np.array_equal(dsts[t].cpu().numpy(), exp)


def test_clip_batch_rejects_invalid_items(cuda):
    fmt = SampleFormat(8)
    fr = _clip(cuda, 4, 64, 96, fmt, 90)
    d = [cuda.empty_like(f) for f in fr]
    with pytest.raises(ValueError, match="bt 2..5"):
        ClipBatch([(Plan(96, 64, fmt, FFT3DConfig(bw=16, bh=16, bt=1)), fr, d)])
    with pytest.raises(ValueError, match="at least tbsize"):
        ClipBatch([(Plan(96, 64, fmt, DFTConfig(tbsize=5, temporal_mode=1)), fr, d)])
    p16 = Plan(96, 64, fmt, FFT3DConfig(bw=16, bh=16, bt=3))
    p32 = Plan(96, 64, fmt, FFT3DConfig(bw=32, bh=32, bt=3))
    with pytest.raises(ValueError, match="share algorithm, block shape"):
        ClipBatch([(p16, fr, d), (p32, fr, [cuda.empty_like(f) for f in fr])])
    with pytest.raises(ValueError):
        ClipBatch([(p16, fr, [fr[1], d[1], d[2], d[3]])])  # an output overlaps a frame of the clip


def _per_frame_window(cuda, plan, frames, tmode, overlap=0):
    """One process_at per output frame with the host layer's selection: tmode 0 the clamped
    centred window (filter.hpp:289-296), tmode 1 the covering temporal blocks."""
    n, T = len(frames), plan.temporal_size
    outs = []
    for t in range(n):
        o = cuda.empty_like(frames[t])
        if tmode == 0:
            plan.process_at([frames[min(max(t - T // 2 + j, 0), n - 1)] for j in range(T)], o)
        else:
            blocks = temporal_blocks(t, n, T, overlap)
            plan.process_at([frames[j] for b in blocks for j in b["slots"]], o, targets=[b["target"] for b in blocks])
        outs.append(o)
    return outs


def test_clip_batch_per_frame_dfttest_modes(cuda):
    """DFTTest tmode 0, tmode 1 with tosize > 0 and smode 0 clips in one clip batch beside a
    grouped tmode 1 clip: every output equals its per-frame call, plain and from the graph."""
    fmt = SampleFormat(16)
    w, h, n = 120, 90, 7
    cases = [
        (DFTConfig(block=16, overlap=8, tbsize=3, ftype=0, sigma=6.0), 0, 0),  # tmode 0
        (DFTConfig(block=16, overlap=8, tbsize=5, ftype=1, sigma=8.0), 0, 0),  # tmode 0, T=5
        (DFTConfig(block=12, overlap=6, tbsize=4, temporal_mode=1, temporal_overlap=2, ftype=0, sigma=5.0), 1, 2),
        (DFTConfig(block=9, mode=0, tbsize=3, ftype=0, sigma=4.0), 0, 0),  # smode 0 (centre)
        (DFTConfig(block=16, overlap=8, tbsize=3, temporal_mode=1, ftype=0, sigma=6.0), 1, 0),  # grouped
    ]
    clips, expect = [], []
    for i, (cfg, tmode, overlap) in enumerate(cases):
        plan = Plan(w, h, fmt, cfg)
        frames = _clip(cuda, n, h, w, fmt, 120 + i)
        dsts = [cuda.empty_like(f) for f in frames]
        clips.append((plan, frames, dsts))
        expect.append(_per_frame_window(cuda, plan, frames, tmode, overlap))
    batch = ClipBatch(clips)
    for graph in (False, True):
        for _, _, dsts in clips:
            for d in dsts:
                d.fill_(0)
        batch.launch(graph=graph)
        for (plan, _, dsts), exp in zip(clips, expect):
            for t, (got, e) in enumerate(zip(dsts, exp)):
                assert cuda.equal(got, e), (plan, t, graph)
            plan.sync_status()
