"""Single-clip sharding through the GPU path: the ranges of 2 and 3 ranks, run one after
another on this GPU (no rank waits on another: the ranges need no exchange), together
give every output frame of the whole clip, bit for bit equal to the single-GPU clip."""
import numpy as np
import pytest

from neo_fft_b200.plan import ClipBatch, DFTConfig, FFT3DConfig, Plan, SampleFormat
from neo_fft_b200.shard import ClipShard, frame_ranges, window
from tests.synth import plane

pytestmark = pytest.mark.gpu

CASES = [
    ("fft3d bt3 u10", SampleFormat(10), FFT3DConfig(bw=16, bh=16, bt=3, sigma=3.0, sharpen=0.3), 11),
    ("fft3d bt4 f32", SampleFormat(32, True), FFT3DConfig(bw=8, bh=8, ow=4, oh=4, bt=4, sigma=2.0), 9),
    ("dft tmode1 T5", SampleFormat(32, True), DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1,
                                                        sigma=8.0), 13),
    ("dft tmode1 T5 tosize2", SampleFormat(16), DFTConfig(block=8, overlap=4, tbsize=5, temporal_mode=1,
                                                          temporal_overlap=2, sigma=6.0), 12),
    ("dft tmode0 T3", SampleFormat(8), DFTConfig(tbsize=3, sigma=8.0), 7),
    ("single dft", SampleFormat(16), DFTConfig(sigma=8.0), 5),
]


@pytest.mark.parametrize("name,fmt,cfg,n", CASES, ids=[c[0] for c in CASES])
def test_ranges_equal_whole_clip(cuda, name, fmt, cfg, n):
    w, h = 96, 72
    clip = [plane(h, w, fmt.bits, fmt.floating, seed=(150, f)) for f in range(n)]
    plan = Plan(w, h, fmt, cfg)
    dev = [cuda.from_numpy(f).cuda() for f in clip]
    # the whole clip on one GPU: the clip form where it applies, else one call per frame
    whole = []
    if isinstance(cfg, FFT3DConfig) or (cfg.temporal_mode == 1 and cfg.temporal_overlap == 0):
        outs = [cuda.empty_like(d) for d in dev]
        ClipBatch([(plan, dev, outs)]).launch()
        whole = [o.cpu().numpy() for o in outs]
    else:
        from neo_fft_b200.shard import plan_kind
        kind, size, ov = plan_kind(plan)
        for f in range(n):
            wd = window(kind, f, n, size, ov)
            o = cuda.empty_like(dev[f])
            plan.process_at([dev[s] for s in wd.sources], o, frame=f, targets=wd.targets)
            whole.append(o.cpu().numpy())
    plan.sync_status()
    for world in (2, 3):
        got = {}
        for rank, rng in enumerate(frame_ranges(n, world)):
            shard = ClipShard(plan, lambda f: clip[f], n, rng)
            part = shard.run()
            assert set(part) == set(range(*rng))
            got.update({k: v.cpu().numpy() for k, v in part.items()})
        assert sorted(got) == list(range(n))
        for f in range(n):
            assert np.array_equal(got[f], whole[f]), (world, f)
