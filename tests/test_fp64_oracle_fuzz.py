"""Seeded random configurations: the binary64 re-evaluation (oracle/fp64_pipeline.py)
against the reference core compiled from its own sources, on the CPU. Draws cover both
algorithms, every sample format, odd and non-square blocks, overlaps, windows, filter
types, temporal sizes and modes, enhancement, degrid and sigma curves. A draw the reference
rejects is rejected by the re-evaluation too (it takes its validation and geometry from the
reference's plan); otherwise the bar is the one
of tests/test_fp64_oracle.py (the reference's own binary32 rounding only), with the
threshold allowance wherever a gain switches at a threshold (DFTTest ftype 1, and ftype 3,
whose gain switches at pmin/pmax) and the error scaled by the gain where it exceeds 1."""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, SampleFormat
from neo_fft_b200.temporal import temporal_blocks
from tests.synth import plane
from tests.test_fp64_oracle import check

R = pytest.importorskip("oracle.ref")
if not R.available():
    pytest.skip("reference oracle not built", allow_module_level=True)
from oracle.fp64_pipeline import FP64Plan  # noqa: E402

FORMATS = [SampleFormat(8), SampleFormat(10), SampleFormat(16), SampleFormat(32, True),
           SampleFormat(8, chroma=True), SampleFormat(12, chroma=True), SampleFormat(32, True, chroma=True)]


def _dft(rng):
    block = int(rng.choice([4, 5, 6, 8, 9, 10, 12, 15, 16, 20]))
    tb = int(rng.choice([1, 1, 2, 3, 4, 5]))
    tmode = int(rng.integers(0, 2)) if tb > 1 else 0
    if tmode == 0 and tb % 2 == 0:
        tb += 1
    mode = 0 if block % 2 == 1 and rng.random() < 0.4 else 1  # centre mode needs an odd block
    cfg = DFTConfig(block=block, overlap=int(rng.integers(0, block)), mode=mode,
                    swin=int(rng.integers(0, 12)), twin=int(rng.integers(0, 12)), ftype=int(rng.integers(0, 5)),
                    tbsize=tb, sbeta=float(rng.uniform(1.0, 4.0)), tbeta=float(rng.uniform(1.0, 4.0)),
                    sigma=float(rng.uniform(0.5, 16.0)), sigma2=float(rng.uniform(0.5, 16.0)),
                    pmin=float(rng.uniform(0.0, 4.0)), pmax=float(rng.uniform(50.0, 800.0)),
                    f0beta=float(rng.choice([1.0, 0.5])), zmean=bool(rng.integers(0, 2)), temporal_mode=tmode,
                    temporal_overlap=int(rng.integers(0, max(1, tb // 2 + 1))) if tmode == 1 else 0)
    if rng.random() < 0.4:
        cfg.slocation = [0.0, float(rng.uniform(1, 12)), 0.5, float(rng.uniform(1, 12)),
                         1.0, float(rng.uniform(1, 12))]
    return cfg


def _fft3d(rng):
    bw = int(rng.choice([4, 6, 8, 12, 16, 20, 24, 32]))
    bh = bw if rng.random() < 0.6 else int(rng.choice([4, 8, 12, 16, 24, 32]))
    cfg = FFT3DConfig(bw=bw, bh=bh, ow=int(rng.integers(0, bw // 2 + 1)), oh=int(rng.integers(0, bh // 2 + 1)),
                      wintype=int(rng.integers(0, 3)), bt=int(rng.choice([-1, 1, 1, 2, 3, 4, 5])),
                      sigma=float(rng.uniform(0.5, 6.0)), beta=float(rng.uniform(1.0, 3.0)),
                      degrid=float(rng.choice([0.0, 1.0, 0.6])),
                      sharpen=float(rng.choice([0.0, 0.0, 0.4])), dehalo=float(rng.choice([0.0, 0.0, 0.5])))
    if rng.random() < 0.3:
        cfg.sigma2, cfg.sigma3, cfg.sigma4 = (float(rng.uniform(0.5, 6.0)) for _ in range(3))
    return cfg


@pytest.mark.parametrize("seed", range(160))
def test_random_configuration_fp64_matches_reference(seed):
    rng = np.random.default_rng([700, seed])
    fmt = FORMATS[int(rng.integers(0, len(FORMATS)))]
    cfg = _dft(rng) if rng.random() < 0.55 else _fft3d(rng)
    w, h = int(rng.integers(24, 120)), int(rng.integers(24, 96))
    try:
        rp = R.RefPlan(w, h, fmt, cfg)
    except ValueError as e:
        with pytest.raises(ValueError) as mine:
            FP64Plan(w, h, fmt, cfg)
        assert str(mine.value) == str(e)
        return
    fp = FP64Plan(w, h, fmt, cfg)
    is_dft = isinstance(cfg, DFTConfig)
    T = cfg.tbsize if is_dft else max(cfg.bt, 1)
    frames = [plane(h, w, fmt.bits, fmt.floating, seed=(701, seed, t)) for t in range(T + 2)]
    targets = ()
    if is_dft and cfg.temporal_mode == 1:
        blocks = temporal_blocks(2, len(frames), T, cfg.temporal_overlap)
        srcs = [frames[s] for b in blocks for s in b["slots"]]
        targets = [b["target"] for b in blocks]
    else:
        srcs = frames[:T]
    ref_out = rp.process(srcs, targets=targets)
    threshold = is_dft and cfg.ftype in (1, 3)
    # DFTTest ftype 2/3/4 multiply by the sigma table (or sigma2): the largest of them bounds
    # the gain; the other filters' gains stay within 1
    gain = max([cfg.sigma, cfg.sigma2] + list(cfg.slocation[1::2])) if is_dft and cfg.ftype >= 2 else 1.0
    check(ref_out, fp.process(srcs, targets=targets), fp, fmt, threshold=threshold, gain=gain)


@pytest.mark.parametrize("seed", range(24))
def test_random_kalman_sequence_fp64_matches_reference(seed):
    """FFT3D bt=0 (Kalman) over 8 frames of a slowly varying clip, random block shape,
    overlap, sigma, kratio, enhancement and format: every rendered frame within the bar.
    A motion-test decision within binary32 rounding of its threshold (counted by the
    re-evaluation) may go the other way in the reference; such frames take the
    threshold allowance."""
    from oracle.fp64_pipeline import FP64Kalman
    rng = np.random.default_rng([702, seed])
    fmt = FORMATS[int(rng.integers(0, len(FORMATS)))]
    bw = int(rng.choice([8, 12, 16, 20, 32]))
    bh = bw if rng.random() < 0.7 else int(rng.choice([8, 16, 32]))
    cfg = FFT3DConfig(bw=bw, bh=bh, ow=int(rng.integers(0, bw // 2 + 1)), oh=int(rng.integers(0, bh // 2 + 1)),
                      bt=0, sigma=float(rng.uniform(1.0, 4.0)), kratio=float(rng.uniform(1.5, 3.0)),
                      sharpen=float(rng.choice([0.0, 0.0, 0.3])), dehalo=float(rng.choice([0.0, 0.0, 0.4])))
    w, h = int(rng.integers(40, 120)), int(rng.integers(32, 96))
    try:
        rp = R.RefPlan(w, h, fmt, cfg)
    except ValueError as e:
        with pytest.raises(ValueError) as mine:
            FP64Plan(w, h, fmt, cfg)
        assert str(mine.value) == str(e)
        return
    fp = FP64Plan(w, h, fmt, cfg)
    st, k = rp.kalman_state(), FP64Kalman(fp)
    base = plane(h, w, fmt.bits, fmt.floating, seed=(703, seed, 0)).astype(np.float64)
    sd = 0.02 if fmt.floating else 0.02 * fp.peak
    dtype = np.float32 if fmt.floating else np.uint8 if fmt.bits == 8 else np.uint16
    for _ in range(8):
        v = base + rng.standard_normal((h, w)) * sd
        src = (v if fmt.floating else np.clip(np.round(v), 0, fp.peak)).astype(dtype)
        rp.advance_kalman(src, st)
        k.advance(src)
        check(rp.render_kalman(src, st), k.render(), fp, fmt, threshold=k.ambiguous > 0)
