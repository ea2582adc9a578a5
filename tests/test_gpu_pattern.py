"""FFT3D sampled noise model (pfactor) and preview (pshow) on the GPU against the
reference core: the pattern candidate (search, power, scaling) is bit-exact, plans with
the published pattern filter bit-exactly (spatial, temporal and Kalman), and the
preview renders the same block."""
import numpy as np
import pytest

from neo_fft_b200.plan import FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu

W, H = 200, 152
CASES = [
    (SampleFormat(8), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, pfactor=1.0, sigma=2.0)),
    (SampleFormat(10, chroma=True), FFT3DConfig(bw=16, bh=16, ow=4, oh=4, pfactor=0.7, px=3, py=4, degrid=0.0)),
    (SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, pfactor=2.0, pcutoff=0.2, sharpen=0.4)),
    (SampleFormat(16), FFT3DConfig(bw=12, bh=12, ow=6, oh=6, pfactor=1.5, bt=3)),
]
IDS = ["u8-auto", "u10c-px-nodegrid", "f32-sharpen", "u16-b12-bt3"]


def _frames(cuda, fmt, n, seed):
    host = [plane(H, W, fmt.bits, fmt.floating, seed=(seed, 0, f)) for f in range(n)]
    return host, [cuda.from_numpy(x).cuda() for x in host]


@pytest.mark.parametrize("fmt,cfg", CASES, ids=IDS)
def test_pattern_candidate_and_filtering_match_reference(cuda, ref, fmt, cfg):
    host, dev = _frames(cuda, fmt, 5, 110)
    p = Plan(W, H, fmt, cfg)
    rp = ref.RefPlan(W, H, fmt, cfg)
    assert p.needs_pattern_frame and not p.pattern_ready
    T = max(1, cfg.bt)
    srcs = [dev[j] for j in range(T)]
    with pytest.raises(ValueError, match="FFT3D sampled model not initialized"):
        p.process_at(srcs, cuda.empty_like(dev[0]))
    cand = p.pattern_candidate(dev[2])
    exp = rp.pattern_candidate(host[2])
    assert np.array_equal(cand, exp)
    p.publish_pattern(cand)
    rp.publish_pattern(exp)
    assert p.pattern_ready
    out = cuda.empty_like(dev[0])
    p.process_at(srcs, out)
    assert np.array_equal(out.cpu().numpy(), rp.process([host[j] for j in range(T)]))
    p.sync_status()


def test_prepare_pattern_publishes_once(cuda, ref):
    fmt, cfg = CASES[0]
    host, dev = _frames(cuda, fmt, 2, 111)
    p = Plan(W, H, fmt, cfg)
    p.prepare_pattern(dev[0])
    p.prepare_pattern(dev[1])  # already published: unchanged
    rp = ref.RefPlan(W, H, fmt, cfg)
    rp.publish_pattern(rp.pattern_candidate(host[0]))
    out = cuda.empty_like(dev[1])
    p.process_at([dev[1]], out)
    assert np.array_equal(out.cpu().numpy(), rp.process([host[1]]))


def test_kalman_with_sampled_pattern(cuda, ref):
    fmt = SampleFormat(32, True)
    cfg = FFT3DConfig(bw=16, bh=16, bt=0, pfactor=1.0, sigma=2.5, kratio=2.0)
    host, dev = _frames(cuda, fmt, 4, 112)
    p = Plan(W, H, fmt, cfg)
    st = p.initial_kalman()
    with pytest.raises(ValueError, match="Kalman sampled model not initialized"):
        p.advance_kalman(dev[0], st)
    rp = ref.RefPlan(W, H, fmt, cfg)
    cand = p.pattern_candidate(dev[0])
    assert np.array_equal(cand, rp.pattern_candidate(host[0]))  # factor 1 for Kalman
    p.publish_pattern(cand)
    rp.publish_pattern(cand)
    rst = rp.kalman_state()
    for f in range(1, 4):
        p.advance_kalman(dev[f], st)
        rp.advance_kalman(host[f], rst)
    out = cuda.empty_like(dev[3])
    p.render_kalman(dev[3], out, st)
    assert np.array_equal(out.cpu().numpy(), rp.render_kalman(host[3], rst))


@pytest.mark.parametrize("fmt,cfg", [
    (SampleFormat(8), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, pfactor=1.0, pshow=True)),
    (SampleFormat(10, chroma=True), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0, sigma2=4.0, pshow=True)),
    (SampleFormat(32, True), FFT3DConfig(bw=12, bh=12, ow=6, oh=6, pfactor=1.0, px=5, py=2, pshow=True)),
], ids=["u8-sampled", "u10c-varying", "f32-px"])
def test_pshow_preview_matches_reference(cuda, ref, fmt, cfg):
    host, dev = _frames(cuda, fmt, 1, 113)
    p = Plan(W, H, fmt, cfg)
    out = cuda.empty_like(dev[0])
    p.process_at([dev[0]], out)
    assert np.array_equal(out.cpu().numpy(), ref.RefPlan(W, H, fmt, cfg).process([host[0]]))
    p.sync_status()
