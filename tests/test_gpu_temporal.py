"""GPU parity of the multi-frame paths against the reference core (oracle/_ref):
FFT3D bt=2..5 (temporal Wiener + enhancement), DFTTest tbsize>1 with tmode 0
(centre slice) and tmode 1 (temporal overlap-add), and the Kalman recursion
(bt=0) including its device-resident state."""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
from tests.synth import plane
from tests.test_gpu_parity import check_parity

pytestmark = pytest.mark.gpu


def frames(n, h, w, fmt, seed):
    return [plane(h, w, fmt.bits, fmt.floating, seed=(*seed, f)) for f in range(n)]


def gpu_process(cuda, plan, srcs, targets=()):
    dev = [cuda.from_numpy(s).cuda() for s in srcs]
    out = cuda.empty_like(dev[len(dev) // 2])
    plan.process_at(dev, out, targets=targets)
    plan.sync_status()
    return out.cpu().numpy()


FFT3D_T = [
    ("C-shape u10 48/24 bt3 sharpen", 200, 150, SampleFormat(10), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3,
                                                                             sigma=3.0, sharpen=0.3)),
    ("u8 16 bt2", 96, 80, SampleFormat(8), FFT3DConfig(bw=16, bh=16, bt=2, sigma=2.0)),
    ("u16 chroma 32 bt4 dehalo", 130, 100, SampleFormat(16, chroma=True),
     FFT3DConfig(bw=32, bh=32, bt=4, sigma=2.5, dehalo=0.4)),
    ("f32 8 bt5 beta", 80, 64, SampleFormat(32, True), FFT3DConfig(bw=8, bh=8, ow=4, oh=4, bt=5, sigma=2, beta=1.3)),
    ("u12 12 bt3 varying", 100, 90, SampleFormat(12),
     FFT3DConfig(bw=12, bh=12, bt=3, sigma=2, sigma2=4, sigma3=1, sigma4=3, sharpen=0.2)),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg", FFT3D_T, ids=[c[0] for c in FFT3D_T])
def test_fft3d_temporal(ref, cuda, name, w, h, fmt, cfg):
    srcs = frames(cfg.bt, h, w, fmt, (3, 0))
    exp = ref.RefPlan(w, h, fmt, cfg).process(srcs)
    gpu = gpu_process(cuda, Plan(w, h, fmt, cfg), srcs)
    check_parity(gpu, exp, fmt)
    # single-frame fallback at clip edges (filter.hpp:266-278)
    exp1 = ref.RefPlan(w, h, fmt, cfg).process([srcs[0]])
    gpu1 = gpu_process(cuda, Plan(w, h, fmt, cfg), [srcs[0]])
    check_parity(gpu1, exp1, fmt)


DFT_T = [
    ("u8 16/12 T3 tmode0", 96, 80, SampleFormat(8), DFTConfig(tbsize=3, sigma=8)),
    ("f32 8/4 T5 tmode0 ftype2", 72, 64, SampleFormat(32, True), DFTConfig(block=8, overlap=4, tbsize=5, ftype=2,
                                                                          sigma=0.7, twin=0)),
    ("u16 32/16 T3 ftype4", 128, 96, SampleFormat(16), DFTConfig(block=32, overlap=16, tbsize=3, ftype=4, sigma=1.2,
                                                                 pmin=3, pmax=250)),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg", DFT_T, ids=[c[0] for c in DFT_T])
def test_dfttest_volume_centre(ref, cuda, name, w, h, fmt, cfg):
    srcs = frames(cfg.tbsize, h, w, fmt, (4, 0))
    exp = ref.RefPlan(w, h, fmt, cfg).process(srcs)
    gpu = gpu_process(cuda, Plan(w, h, fmt, cfg), srcs)
    check_parity(gpu, exp, fmt)


def test_dfttest_temporal_ola_d2_shape(ref, cuda):
    """tbsize=5, tmode=1, sbsize 12, sosize 9, ftype 1 on float frames (the temporal
    overlap-add configuration), for outputs at the clip start, middle and end."""
    from oracle import ref as R  # noqa: F401
    fmt = SampleFormat(32, True)
    w, h, n_frames = 120, 72, 9
    cfg = DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, temporal_overlap=0, ftype=1, sigma=8.0,
                    swin=0, twin=7)
    clip = frames(n_frames, h, w, fmt, (5, 0))
    rp = ref.RefPlan(w, h, fmt, cfg)
    p = Plan(w, h, fmt, cfg)
    from neo_fft_b200.temporal import temporal_blocks
    for n in (0, 4, 8):
        blocks = temporal_blocks(n, n_frames, cfg.tbsize, cfg.temporal_overlap)
        srcs = [clip[s] for b in blocks for s in b["slots"]]
        targets = [b["target"] for b in blocks]
        exp = rp.process(srcs, targets=targets)
        gpu = gpu_process(cuda, p, srcs, targets)
        check_parity(gpu, exp, fmt)


@pytest.mark.parametrize("fmt,cfg", [
    (SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0)),
    (SampleFormat(8), FFT3DConfig(bw=16, bh=16, bt=0, sigma=3.0, kratio=1.5, sharpen=0.4)),
    (SampleFormat(10), FFT3DConfig(bw=12, bh=12, bt=0, sigma=2, sigma2=3, sigma3=1, sigma4=2, kratio=2.0)),
])
def test_kalman_recursion_and_render(ref, cuda, fmt, cfg):
    w, h = 160, 120
    clip = frames(6, h, w, fmt, (6, 0))
    rp = ref.RefPlan(w, h, fmt, cfg)
    rs = rp.kalman_state()
    p = Plan(w, h, fmt, cfg)
    st = p.initial_kalman()
    last0, cov0, proc0 = st.read()
    rl, rc, rq = rs.read()
    assert np.array_equal(last0, rl) and np.array_equal(cov0, rc) and np.array_equal(proc0, rq)
    for f in range(1, len(clip)):
        rp.advance_kalman(clip[f], rs)
        src = cuda.from_numpy(clip[f]).cuda()
        p.advance_kalman(src, st)
        p.sync_status()
        gl, gc, gq = st.read()
        rl, rc, rq = rs.read()
        assert np.array_equal(gl.view(np.uint32), rl.view(np.uint32)), f"L differs at frame {f}"
        assert np.array_equal(gc.view(np.uint32), rc.view(np.uint32)), f"C differs at frame {f}"
        assert np.array_equal(gq.view(np.uint32), rq.view(np.uint32)), f"Q differs at frame {f}"
        exp = rp.render_kalman(clip[f], rs)
        out = cuda.empty_like(src)
        p.render_kalman(src, out, st)
        p.sync_status()
        check_parity(out.cpu().numpy(), exp, fmt)


def test_kalman_fp64_variance_tracks_reference(ref, cuda):
    """The binary64 variance mode stays within the float tolerance of the binary32
    reference on a smooth clip and reports its deviation."""
    fmt = SampleFormat(32, True)
    cfg = FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0)
    w, h = 160, 120
    clip = frames(12, h, w, fmt, (6, 1))
    rp = ref.RefPlan(w, h, fmt, cfg)
    rs = rp.kalman_state()
    p = Plan(w, h, fmt, cfg)
    st = p.initial_kalman(fp64_variance=True)
    worst = 0.0
    for f in range(1, len(clip)):
        rp.advance_kalman(clip[f], rs)
        src = cuda.from_numpy(clip[f]).cuda()
        p.advance_kalman(src, st)
        exp = rp.render_kalman(clip[f], rs)
        out = cuda.empty_like(src)
        p.render_kalman(src, out, st)
        worst = max(worst, float(np.abs(out.cpu().numpy() - exp).max()))
    assert worst <= 2e-5, worst
