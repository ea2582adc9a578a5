"""Host request layer (nf_frame_server): output frames served in ranges of batched
launches with the host layer's frame selection (src/plugin/filter.hpp:253-528) equal
one per-frame Plan call with the same selection bit for bit — single-frame plans
(batched form), FFT3D bt 2..5 and DFTTest tmode 1 tosize 0 (clip forms, including
range margins and the short tail range), DFTTest tmode 0 and tmode 1 with tosize > 0
(per-frame calls over device-resident sources) — in sequential and random order, with
passed-through planes, the FFT3D sampled model prepared from the pattern frame, and
the reference core."""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, FrameServer, Plan, SampleFormat
from neo_fft_b200.temporal import centred_slots, fft3d_slots, temporal_blocks
from tests.synth import plane

pytestmark = pytest.mark.gpu


def _clip(n, sizes, fmt, seed):
    return [[plane(h, w, fmt.bits, fmt.floating, seed=(seed, f, p)) for p, (w, h) in enumerate(sizes)]
            for f in range(n)]


def _expected(plan, clip, p, n, fmt):
    """One per-frame call with the host layer's frame selection."""
    N = len(clip)
    if isinstance(plan.config, FFT3DConfig):
        return plan.process([clip[f][p] for f in fft3d_slots(n, N, plan.temporal_size)])
    T = plan.temporal_size
    if T == 1:
        return plan.process([clip[n][p]])
    if plan.config.temporal_mode == 1:
        blocks = temporal_blocks(n, N, T, plan.config.temporal_overlap)
        dst = np.empty_like(clip[n][p])
        return plan.process_at([clip[f][p] for b in blocks for f in b["slots"]], dst,
                               targets=[b["target"] for b in blocks])
    return plan.process([clip[f][p] for f in centred_slots(n, N, T)])


def _serve(plans, clip, order, R):
    src = lambda f, p: clip[f][p]  # noqa: E731
    server = FrameServer(plans, len(clip), src, range_frames=R)
    got = {n: server.get(n) for n in order}
    return server, got


CASES = [
    ("dft-single-yuv", SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0), 9, 4),
    ("fft3d-bt3", SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, bt=3, sigma=3.0), 11, 4),
    ("fft3d-bt4", SampleFormat(10), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=4, sigma=2.5, sharpen=0.3), 10, 3),
    ("fft3d-bt2", SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=2, sigma=2.0), 7, 3),
    ("dft-tmode1", SampleFormat(16), DFTConfig(block=12, overlap=9, tbsize=3, temporal_mode=1, ftype=1, sigma=6.0),
     13, 4),
    ("dft-tmode0", SampleFormat(8), DFTConfig(block=8, overlap=4, tbsize=3, ftype=0, sigma=4.0), 8, 3),
    ("dft-tmode1-overlap", SampleFormat(32, True),
     DFTConfig(block=8, overlap=4, tbsize=3, temporal_mode=1, temporal_overlap=1, ftype=0, sigma=3.0), 7, 3),
]


@pytest.mark.parametrize("name,fmt,cfg,N,R", CASES, ids=[c[0] for c in CASES])
def test_server_equals_per_frame_selection(cuda, name, fmt, cfg, N, R):
    sizes = [(160, 96), (80, 48), (80, 48)]
    cfmt = SampleFormat(fmt.bits, fmt.floating, chroma=True)
    luma, chroma = Plan(*sizes[0], fmt, cfg), Plan(*sizes[1], cfmt, cfg)
    clip = _clip(N, sizes, fmt, 300 + N)
    plans = [luma, chroma, None]                            # plane 2 passed through
    rng = np.random.default_rng(N)
    for order in (list(range(N)), list(rng.permutation(N))):
        server, got = _serve(plans, clip, order, R)
        for n in range(N):
            for p, plan in enumerate(plans):
                exp = clip[n][p] if plan is None else _expected(plan, clip, p, n, fmt)
                assert np.array_equal(got[n][p], exp), (name, n, p)
        if order == list(range(N)):
            computed, fetched = server.counters
            assert computed >= N and computed <= N + R  # the prefetched range may run past the clip's use
    for n in range(N):
        req = server.request(n)
        if isinstance(cfg, FFT3DConfig):
            assert req == fft3d_slots(n, N, cfg.bt)
        elif cfg.tbsize == 1:
            assert req == [n]
        elif cfg.temporal_mode == 1:
            assert req == sorted({f for b in temporal_blocks(n, N, cfg.tbsize, cfg.temporal_overlap)
                                  for f in b["slots"]})
        else:
            assert req == sorted(set(centred_slots(n, N, cfg.tbsize)))


def test_server_matches_reference(ref, cuda):
    fmt = SampleFormat(16)
    cfg = FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=3, sigma=600.0)
    w, h, N = 96, 64, 7
    clip = [[plane(h, w, 16, False, seed=(310, f, 0))] for f in range(N)]
    server = FrameServer([Plan(w, h, fmt, cfg)], N, lambda f, p: clip[f][p], range_frames=3)
    rp = ref.RefPlan(w, h, fmt, cfg)
    for n in range(N):
        exp = rp.process([clip[f][0] for f in fft3d_slots(n, N, 3)])
        assert np.array_equal(server.get(n)[0], exp), n


def test_server_prepares_fft3d_pattern(cuda):
    fmt = SampleFormat(8)
    cfg = FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=3, sigma=2.0, pfactor=0.8, pframe=2)
    w, h, N = 128, 96, 6
    clip = [[plane(h, w, 8, False, seed=(320, f, 0))] for f in range(N)]
    sp = Plan(w, h, fmt, cfg)
    server = FrameServer([sp], N, lambda f, p: clip[f][p], range_frames=4)
    assert 2 in server.request(0)                           # the pattern frame is requested too
    got = [server.get(n)[0] for n in range(N)]
    assert sp.model_state == 2
    ep = Plan(w, h, fmt, cfg)
    ep.prepare_pattern(cuda.from_numpy(clip[2][0]).cuda())
    for n in range(N):
        exp = ep.process([clip[f][0] for f in fft3d_slots(n, N, 3)])
        assert np.array_equal(got[n], exp), n


def test_server_errors(cuda):
    fmt = SampleFormat(8)
    clip = [[plane(48, 64, 8, False, seed=(330, f, 0))] for f in range(4)]
    with pytest.raises(ValueError, match="temporal configuration"):
        FrameServer([Plan(64, 48, fmt, FFT3DConfig(bw=16, bh=16, bt=0)),
                     Plan(64, 48, fmt, FFT3DConfig(bw=16, bh=16, bt=1))], 4, lambda f, p: clip[f][p])
    with pytest.raises(ValueError, match="at least one processed plane"):
        FrameServer([None], 4, lambda f, p: clip[f][p])
    with pytest.raises(ValueError, match="tbsize"):
        FrameServer([Plan(64, 48, fmt, DFTConfig(tbsize=5, temporal_mode=1))], 4, lambda f, p: clip[f][p])
    good = Plan(64, 48, fmt, DFTConfig())
    server = FrameServer([good], 4, lambda f, p: clip[f][p])
    with pytest.raises(ValueError, match="outside clip"):
        server.get(4)

    def broken(f, p):
        if f == 2:
            raise KeyError("frame 2 unavailable")
        return clip[f][p]
    server = FrameServer([good], 4, broken, range_frames=2)
    assert np.array_equal(server.get(0)[0], good.process([clip[0][0]]))
    with pytest.raises(KeyError):
        server.get(3)
    wrong = FrameServer([good], 4, lambda f, p: np.zeros((40, 64), np.uint8))
    with pytest.raises(ValueError, match="dimensions"):
        wrong.get(0)


def test_server_kalman_random_access_matches_reference(ref, cuda):
    """FFT3D bt=0 through the frame server: frame 0 passes through, other frames follow
    the host layer's bounded warm-up with four checkpoints, so each output equals the
    reference advanced from the frame its replay starts at (as in the KalmanSeek test)."""
    w, h, warmup = 96, 64, 4
    fmt = SampleFormat(32, True)
    cfg = FFT3DConfig(bw=16, bh=16, bt=0, sigma=2.5, kratio=2.0, kalman_warmup=warmup)
    host = [plane(h, w, 32, True, seed=(97, 0, f)) for f in range(24)]
    chroma = [plane(h // 2, w // 2, 32, True, seed=(97, 1, f)) for f in range(24)]
    server = FrameServer([Plan(w, h, fmt, cfg), None], 24,
                         lambda f, p: host[f] if p == 0 else chroma[f], range_frames=4)
    assert server.request(20) == [16, 17, 18, 19, 20] and server.request(0) == [0]
    rp = ref.RefPlan(w, h, fmt, cfg)
    first = {5: 1, 6: 1, 7: 1, 20: 16, 3: 1, 21: 16}
    for n in (5, 6, 7, 20, 3, 21, 0):
        got, passed = server.get(n)
        assert np.array_equal(passed, chroma[n])
        if n == 0:
            assert np.array_equal(got, host[0])
            continue
        st = rp.kalman_state()
        for f in range(first[n], n + 1):
            rp.advance_kalman(host[f], st)
        assert np.array_equal(got, rp.render_kalman(host[n], st)), n


def test_server_dithered_output_uses_frame_and_plane(cuda):
    """8-bit DFTTest with dither: the server's per-frame path passes each output's frame
    and plane number, so the dither hash matches a direct call with the same coordinates."""
    fmt = SampleFormat(8)
    cfg = DFTConfig(block=16, overlap=8, sigma=4.0, dither=2, dither_seed=7)
    w, h, N = 96, 64, 5
    clip = [[plane(h, w, 8, False, seed=(340, f, p)) for p in range(2)] for f in range(N)]
    plans = [Plan(w, h, fmt, cfg), Plan(w, h, fmt, cfg)]
    server = FrameServer(plans, N, lambda f, p: clip[f][p], range_frames=2)
    for n in (3, 0, 4, 1):
        got = server.get(n)
        for p in range(2):
            exp = np.empty_like(clip[n][p])
            plans[p].process_at([clip[n][p]], exp, frame=n, plane=p)
            assert np.array_equal(got[p], exp), (n, p)
