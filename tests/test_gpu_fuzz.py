"""Seeded random configurations against the reference core: for every draw the GPU plan
and the reference either both reject the configuration (same exception type) or both
build, and then filter the same random planes to bit-identical output. Draws cover
both algorithms, every sample format, odd and non-square blocks, overlaps, windows,
filter types, temporal sizes and modes, enhancement and sigma curves."""
import numpy as np
import pytest

from neo_fft_b200 import DeviceError, NonFiniteError
from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
from neo_fft_b200.temporal import temporal_blocks
from tests.synth import plane

pytestmark = pytest.mark.gpu

FORMATS = [SampleFormat(8), SampleFormat(10), SampleFormat(16), SampleFormat(32, True),
           SampleFormat(8, chroma=True), SampleFormat(12, chroma=True), SampleFormat(32, True, chroma=True)]


def _dft(rng):
    block = int(rng.choice([4, 5, 6, 8, 9, 10, 12, 15, 16, 20, 24, 32]))
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
    bw = int(rng.choice([4, 6, 8, 12, 16, 20, 24, 32, 48]))
    bh = bw if rng.random() < 0.6 else int(rng.choice([4, 8, 12, 16, 24, 32]))
    return FFT3DConfig(bw=bw, bh=bh, ow=int(rng.integers(0, bw // 2 + 1)), oh=int(rng.integers(0, bh // 2 + 1)),
                       wintype=int(rng.integers(0, 3)), bt=int(rng.choice([-1, 1, 1, 2, 3, 4, 5])),
                       sigma=float(rng.uniform(0.5, 6.0)), beta=float(rng.uniform(1.0, 3.0)),
                       degrid=float(rng.choice([0.0, 1.0, 0.6])),
                       sharpen=float(rng.choice([0.0, 0.0, 0.4])), dehalo=float(rng.choice([0.0, 0.0, 0.5])))


def _reference_outcome(fn):
    try:
        return fn(), None
    except (ValueError, RuntimeError) as e:  # the oracle maps the reference's exceptions
        return None, type(e)


@pytest.mark.parametrize("seed", range(64))
def test_random_configuration_matches_reference(ref, cuda, seed):
    rng = np.random.default_rng([500, seed])
    fmt = FORMATS[int(rng.integers(0, len(FORMATS)))]
    cfg = _dft(rng) if rng.random() < 0.6 else _fft3d(rng)
    w, h = int(rng.integers(24, 160)), int(rng.integers(24, 120))
    rp, ref_err = _reference_outcome(lambda: ref.RefPlan(w, h, fmt, cfg))
    try:
        gp, gpu_err = Plan(w, h, fmt, cfg), None
    except ValueError as e:
        gp, gpu_err = None, type(e)
    if ref_err is not None or gpu_err is not None:
        assert ref_err == gpu_err, (cfg, ref_err, gpu_err)
        return
    T = gp.temporal_size
    frames = [plane(h, w, fmt.bits, fmt.floating, seed=(501, seed, t)) for t in range(max(T, 1) + 2)]
    targets = ()
    if isinstance(cfg, DFTConfig) and cfg.temporal_mode == 1:
        blocks = temporal_blocks(2, len(frames), T, cfg.temporal_overlap)
        srcs = [frames[s] for b in blocks for s in b["slots"]]
        targets = [b["target"] for b in blocks]
    else:
        srcs = frames[:T] if T > 1 else frames[:1]
    exp, exp_err = _reference_outcome(lambda: rp.process(srcs, targets=targets))
    try:
        got, got_err = gp.process_at(srcs, np.empty_like(frames[0]), targets=targets), None
    except (ValueError, NonFiniteError, DeviceError) as e:
        got, got_err = None, type(e)
    assert exp_err == got_err, (cfg, exp_err, got_err)
    if exp is not None:
        assert np.array_equal(got, exp), (cfg, fmt, w, h)


def _per_frame(plan, cfg, clip, n):
    """One per-frame call with the host layer's frame selection."""
    from neo_fft_b200.temporal import centred_slots, fft3d_slots
    N = len(clip)
    if isinstance(cfg, FFT3DConfig):
        return plan.process([clip[f] for f in fft3d_slots(n, N, plan.temporal_size)])
    T = plan.temporal_size
    if T == 1:
        return plan.process([clip[n]])
    if cfg.temporal_mode == 1:
        blocks = temporal_blocks(n, N, T, cfg.temporal_overlap)
        return plan.process_at([clip[f] for b in blocks for f in b["slots"]], np.empty_like(clip[n]),
                               targets=[b["target"] for b in blocks])
    return plan.process([clip[f] for f in centred_slots(n, N, T)])


@pytest.mark.parametrize("seed", range(24))
def test_random_configuration_through_frame_server(cuda, seed):
    """The frame server picks the batched, clip or per-frame form from the plan; every
    output frame of a random valid configuration equals the per-frame call."""
    from neo_fft_b200.plan import FrameServer
    rng = np.random.default_rng([502, seed])
    fmt = FORMATS[int(rng.integers(0, len(FORMATS)))]
    for _ in range(20):  # draw until the configuration is valid
        cfg = _dft(rng) if rng.random() < 0.6 else _fft3d(rng)
        w, h = int(rng.integers(40, 160)), int(rng.integers(40, 120))
        try:
            p = Plan(w, h, fmt, cfg)
            break
        except ValueError:
            continue
    else:
        pytest.skip("no valid draw")
    N = 7
    if p.temporal_size > N:
        pytest.skip("temporal size above the clip")
    clip = [plane(h, w, fmt.bits, fmt.floating, seed=(503, seed, f)) for f in range(N)]
    server = FrameServer([p], N, lambda f, _p: clip[f], range_frames=int(rng.integers(1, 5)))
    for n in rng.permutation(N):
        assert np.array_equal(server.get(int(n))[0], _per_frame(p, cfg, clip, int(n))), (cfg, fmt, w, h, n)
