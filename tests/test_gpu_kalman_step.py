"""The Kalman step (nf_kalman_step_device: advance then render of one frame in one pass over
the blocks) against the two separate calls, which the reference pins
(tests/test_gpu_temporal.py): every output frame and the whole state equal bit for bit over
a sequence, for codelet and project block shapes, enhancement, both variance modes and a
plane whose last block column lies beyond the visible area; a non-finite frame is reported
the same way."""
import numpy as np
import pytest

from neo_fft_b200.plan import FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu

CASES = [
    ("f32 32/16 (D1 shape)", 200, 136, SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0),
     False),
    ("f32 32/16 binary64 variance", 200, 136, SampleFormat(32, True),
     FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0), True),
    ("u8 16 sharpen", 160, 120, SampleFormat(8), FFT3DConfig(bw=16, bh=16, bt=0, sigma=3.0, kratio=1.5, sharpen=0.4),
     False),
    ("u10 12 sigma curve", 160, 120, SampleFormat(10),
     FFT3DConfig(bw=12, bh=12, bt=0, sigma=2, sigma2=3, sigma3=1, sigma4=2, kratio=2.0), False),
    ("u16 32/8, last column invisible", 95, 71, SampleFormat(16), FFT3DConfig(bw=32, bh=32, ow=8, oh=8, bt=0,
                                                                              sigma=4.0, kratio=2.0), False),
    ("u8 8 dehalo", 96, 64, SampleFormat(8), FFT3DConfig(bw=8, bh=8, bt=0, sigma=2.0, dehalo=1.0), False),
    ("f32 20 project shape", 120, 100, SampleFormat(32, True), FFT3DConfig(bw=20, bh=20, bt=0, sigma=2.0, kratio=2.0),
     True),
    ("u10 48/24 sharpen", 200, 150, SampleFormat(10), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=0, sigma=3.0,
                                                                   kratio=2.0, sharpen=0.3), False),
    # 45 bins per block: runs keep the state in global memory (no 16-byte bulk copies)
    ("u8 9 state unstaged", 90, 66, SampleFormat(8), FFT3DConfig(bw=9, bh=9, bt=0, sigma=2.0, kratio=2.0), True),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg,fp64", CASES, ids=[c[0] for c in CASES])
def test_step_equals_advance_then_render(cuda, name, w, h, fmt, cfg, fp64):
    torch = cuda
    clip = [plane(h, w, fmt.bits, fmt.floating, seed=(7, f)) for f in range(6)]
    sep, stp = Plan(w, h, fmt, cfg), Plan(w, h, fmt, cfg)
    s_sep, s_stp = sep.initial_kalman(fp64_variance=fp64), stp.initial_kalman(fp64_variance=fp64)
    for f, frame in enumerate(clip):
        src = torch.from_numpy(frame).cuda()
        a, b = torch.empty_like(src), torch.empty_like(src)
        sep.advance_kalman(src, s_sep)
        sep.render_kalman(src, a, s_sep)
        stp.step_kalman(src, b, s_stp)
        sep.sync_status()
        stp.sync_status()
        assert torch.equal(a, b), f"{name}: output differs at frame {f}"
        for x, y in zip(s_sep.read(), s_stp.read()):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"{name}: state differs at frame {f}"


def test_step_reports_non_finite_input(cuda):
    torch = cuda
    fmt, cfg = SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0)
    w, h = 128, 96
    frame = plane(h, w, 32, True, seed=(7, 9))
    frame[40, 50] = np.nan
    src = torch.from_numpy(frame).cuda()
    for use_step in (False, True):
        p = Plan(w, h, fmt, cfg)
        st = p.initial_kalman()
        out = torch.empty_like(src)
        if use_step:
            p.step_kalman(src, out, st)
        else:
            p.advance_kalman(src, st)
            p.render_kalman(src, out, st)
        with pytest.raises(Exception, match="non-finite|finite"):
            p.sync_status()
