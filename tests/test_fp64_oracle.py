"""The binary64 re-evaluation (oracle/fp64_pipeline.py) against the reference core compiled
from its own sources (oracle/_ref), on the CPU: FFT3D bt=1 (uniform and varying sigma,
sharpen, dehalo, beta floor, chroma base), bt=2..5, Kalman (bt=0) over a sequence, and
DFTTest tbsize 1 (ftype 0..4, curves) and 3-D (tmode 0 and tmode 1).

Where the reference keeps binary32 arithmetic and the re-evaluation binary64, the two may
differ by the reference's own rounding only: float outputs within 2e-6 of full scale, and
integer outputs by at most one step (in the few pixels whose exact value lies within the
reference's rounding error of a rounding boundary), with the reference's value within
0.52 of a step of the exact one. Filters whose gain exceeds 1 (DFTTest ftype 2/3/4 multiply
by sigma) scale the reference's error with it, and the bars with them (`check`). This pins
the re-evaluation before the GPU tests use it as the independent check of the sm_100a
path; tests/test_fp64_oracle_fuzz.py extends it to seeded random configurations."""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, SampleFormat
from neo_fft_b200.temporal import temporal_blocks
from tests.synth import plane

R = pytest.importorskip("oracle.ref")
if not R.available():
    pytest.skip("reference oracle not built", allow_module_level=True)
from oracle.fp64_pipeline import FP64Kalman, FP64Plan  # noqa: E402


def check(ref_out, value, fp64, fmt, threshold=False, gain=1.0):
    """threshold: a gain that switches at a threshold (DFTTest ftype 1's hard threshold,
    ftype 3's pmin/pmax range), where a bin whose power lies within binary32 rounding of
    the threshold switches in one of the two evaluations; a few pixels then differ by that
    bin's share of the block times the step of the gain. gain: the largest gain the filter
    applies when it exceeds 1 (DFTTest ftype 2/3/4 multiply by sigma), which bounds that
    step and scales the binary32 error in output steps, and so the share of integer pixels
    that round to the neighbouring step. Float full scale is 1, or the output's largest
    magnitude where such a gain carries the output beyond it."""
    gain = max(1.0, gain)
    if fmt.floating:
        scale = max(1.0, float(np.abs(ref_out).max()))
        e = np.abs(ref_out.astype(np.float64) - value) / scale
        if threshold:
            assert e.max() <= 1e-3 * gain and np.mean(e > 2e-6) <= 0.02
        else:
            assert e.max() <= 2e-6
        return
    q = fp64.quantize(value)
    d = np.abs(ref_out.astype(np.int64) - q.astype(np.int64))
    assert d.max() <= 1 and np.mean(d > 0) <= 0.01 * gain
    inside = (value > 0) & (value < fp64.peak)  # where no clamp applies
    far = np.abs(ref_out.astype(np.float64) - value)[inside] > 0.5 + 0.02 * gain
    if threshold:
        assert np.mean(far) <= 0.01
    else:
        assert not far.any()


CASES = [
    ("fft3d u8 32/16", 200, 150, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0), 1),
    ("fft3d f32 32 default overlap", 200, 150, SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, sigma=2.0), 1),
    ("fft3d u10 48/24 bt3 sharpen", 200, 150, SampleFormat(10),
     FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3), 3),
    ("fft3d f32 16 bt2 dehalo varying", 130, 100, SampleFormat(32, True),
     FFT3DConfig(bw=16, bh=16, bt=2, sigma=2, sigma2=4, sigma3=1, sigma4=3, dehalo=0.4), 2),
    ("fft3d f32 16 bt5 beta", 96, 80, SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, bt=5, sigma=2, beta=1.3), 5),
    ("fft3d f32 16 varying sharpen", 130, 100, SampleFormat(32, True),
     FFT3DConfig(bw=16, bh=16, sigma=2, sigma2=4, sigma3=1, sigma4=3, sharpen=0.4), 1),
    ("fft3d u16 chroma beta", 130, 100, SampleFormat(16, chroma=True), FFT3DConfig(bw=16, bh=16, sigma=2, beta=1.5), 1),
    ("fft3d f32 bt-1 sharpen only", 96, 80, SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, bt=-1, sharpen=0.5), 1),
    ("dft u16 16/12 flat curve", 200, 150, SampleFormat(16),
     DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8]), 1),
    ("dft f32 16/12 ftype0", 200, 150, SampleFormat(32, True), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0), 1),
    ("dft f32 16/8 f0beta 0.5", 120, 100, SampleFormat(32, True), DFTConfig(block=16, overlap=8, sigma=8.0,
                                                                            f0beta=0.5), 1),
    ("dft f32 ftype1", 120, 100, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=1, sigma=8.0), 1),
    ("dft f32 ftype2", 120, 100, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=2, sigma=0.8), 1),
    ("dft f32 ftype3", 120, 100, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=3, sigma=0.8,
                                                                   sigma2=1.2, pmin=3, pmax=250), 1),
    ("dft f32 ftype4", 120, 100, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=4, sigma=1.2,
                                                                   pmin=3, pmax=250), 1),
    ("dft u8 12/9 T5 tmode0", 96, 80, SampleFormat(8), DFTConfig(block=12, overlap=9, tbsize=5, sigma=8.0), 5),
    ("dft f32 16/12 T3 curves", 96, 80, SampleFormat(32, True),
     DFTConfig(block=16, overlap=12, tbsize=3, sigma=8.0, slocation=[0, 4, 0.5, 8, 1, 12]), 3),
    ("dft f32 9 smode0", 40, 32, SampleFormat(32, True), DFTConfig(block=9, mode=0, sigma=8.0), 1),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg,nsrc", CASES, ids=[c[0] for c in CASES])
def test_fp64_reevaluation_matches_reference(name, w, h, fmt, cfg, nsrc):
    srcs = [plane(h, w, fmt.bits, fmt.floating, seed=(61, f)) for f in range(nsrc)]
    ref_out = R.RefPlan(w, h, fmt, cfg).process(srcs)
    fp = FP64Plan(w, h, fmt, cfg)
    check(ref_out, fp.process(srcs), fp, fmt)


@pytest.mark.parametrize("ftype,tbsize,tosize", [(0, 5, 0), (1, 5, 0), (0, 4, 2), (0, 5, 2)])
def test_fp64_temporal_overlap_add_matches_reference(ftype, tbsize, tosize):
    """tmode 1, with and without overlapping temporal blocks (tosize > 0: an output adds the
    slices of every temporal block that covers it)."""
    w, h, n = 96, 80, 9
    fmt = SampleFormat(32, True)
    cfg = DFTConfig(block=12, overlap=9, tbsize=tbsize, temporal_mode=1, temporal_overlap=tosize, ftype=ftype,
                    sigma=8.0)
    clip = [plane(h, w, 32, True, seed=(62, f)) for f in range(n)]
    rp, fp = R.RefPlan(w, h, fmt, cfg), FP64Plan(w, h, fmt, cfg)
    for t in (0, 2, 4, 8):
        blocks = temporal_blocks(t, n, tbsize, tosize)
        srcs = [clip[s] for b in blocks for s in b["slots"]]
        tg = [b["target"] for b in blocks]
        check(rp.process(srcs, targets=tg), fp.process(srcs, targets=tg), fp, fmt, threshold=ftype == 1)


@pytest.mark.parametrize("bw,sharpen", [(32, 0.0), (16, 0.3)])
def test_fp64_kalman_sequence_matches_reference(bw, sharpen):
    w, h = 200, 150
    fmt = SampleFormat(32, True)
    cfg = FFT3DConfig(bw=bw, bh=bw, bt=0, sigma=2.5, kratio=2.0, sharpen=sharpen)
    rp, fp = R.RefPlan(w, h, fmt, cfg), FP64Plan(w, h, fmt, cfg)
    st, k = rp.kalman_state(), FP64Kalman(fp)
    rng = np.random.default_rng(63)
    base = plane(h, w, 32, True, seed=(63, 0)) * 0.8
    for _ in range(24):
        src = (base + rng.standard_normal((h, w)) * 0.02).astype(np.float32)
        rp.advance_kalman(src, st)
        k.advance(src)
        check(rp.render_kalman(src, st), k.render(), fp, fmt)
