"""Kalman seeks over device-resident checkpoints: each rendered frame equals the
reference core's render after advancing its own initial state over the frames the
bounded-warmup rule prescribes (src/plugin/filter.hpp:152-250)."""
import numpy as np
import pytest

from neo_fft_b200.checkpoints import KalmanCheckpoints, KalmanSeek
from neo_fft_b200.plan import FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fp64", [False, True])
def test_seek_matches_reference_replays(cuda, ref, fp64):
    w, h, warmup = 96, 64, 4
    fmt = SampleFormat(32, True)
    cfg = FFT3DConfig(bw=16, bh=16, bt=0, sigma=2.5, kratio=2.0)
    plan = Plan(w, h, fmt, cfg)
    if fp64:
        orig = plan.initial_kalman
        plan.initial_kalman = lambda: orig(fp64_variance=True)
    host = [plane(h, w, 32, True, seed=(97, 0, f)) for f in range(24)]
    dev = [cuda.from_numpy(x).cuda() for x in host]
    seek = KalmanSeek([plan], warmup=warmup, checkpoints=KalmanCheckpoints())
    rp = ref.RefPlan(w, h, fmt, cfg)
    first = {5: 1, 6: 1, 7: 1, 20: 16, 3: 1, 21: 16}
    for n in (5, 6, 7, 20, 3, 21, 0):
        out = cuda.empty_like(dev[n])
        seek.frame(n, lambda f, p: dev[f], [out])
        got = out.cpu().numpy()
        if n == 0:
            assert np.array_equal(got, host[0])
            continue
        st = rp.kalman_state()
        for f in range(first[n], n + 1):
            rp.advance_kalman(host[f], st)
        exp = rp.render_kalman(host[n], st)
        if fp64:  # binary64 variance: within the float tolerance of the binary32 reference
            assert np.abs(got.astype(np.float64) - exp).max() <= 2e-5
        else:
            assert np.array_equal(got, exp)
    assert len(seek.checkpoints.frames()) == 4
    plan.sync_status()


def test_clone_keeps_precision_and_contents(cuda):
    plan = Plan(64, 48, SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, bt=0, sigma=2.0))
    src = cuda.from_numpy(plane(48, 64, 32, True, seed=(98, 0, 0))).cuda()
    for fp64 in (False, True):
        st = plan.initial_kalman(fp64_variance=fp64)
        plan.advance_kalman(src, st)
        c = st.clone()
        assert c.nbytes == st.nbytes == st.count * (8 + 2 * (8 if fp64 else 4))
        plan.advance_kalman(src, st)
        plan.advance_kalman(src, c)
        a, b = cuda.empty_like(src), cuda.empty_like(src)
        plan.render_kalman(src, a, st)
        plan.render_kalman(src, b, c)
        assert cuda.equal(a, b)
