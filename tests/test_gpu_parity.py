"""GPU parity: the sm_100a path (through the C ABI) against the reference core compiled
from its own sources, on identical seeded inputs.

The parity bar: float output within 2e-5 of full scale, integer output within
±1 LSB on at most 0.01 % of pixels. The GPU path restates the reference's arithmetic
step by step, so these cases are expected to be bit-identical; `exact=False` cases
(binary32 pow for f0beta outside {1, 0.5}) use the tolerance.
"""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu

FLOAT_TOL = 2e-5      # of full scale
INT_FRACTION = 1e-4   # at most 0.01 % of pixels may differ, by at most 1 LSB


def check_parity(gpu: np.ndarray, exp: np.ndarray, fmt: SampleFormat, exact: bool = True):
    assert gpu.shape == exp.shape and gpu.dtype == exp.dtype
    if exact and np.array_equal(gpu, exp):
        return
    if fmt.floating:
        err = np.abs(gpu.astype(np.float64) - exp.astype(np.float64)).max()
        assert err <= FLOAT_TOL, f"max abs error {err:.3g}"
        if exact:
            pytest.fail(f"not bit-exact (max abs error {err:.3g})")
    else:
        d = np.abs(gpu.astype(np.int64) - exp.astype(np.int64))
        frac = float((d > 0).mean())
        assert d.max() <= 1 and frac <= INT_FRACTION, f"max {d.max()} LSB on {frac:.4%} of pixels"
        if exact:
            pytest.fail(f"not bit-exact: {int((d > 0).sum())} pixels differ by 1 LSB")


def run_both(ref, cuda, w, h, fmt, cfg, frames, seed=(1, 0)):
    srcs = [plane(h, w, fmt.bits, fmt.floating, seed=(*seed, f)) for f in range(frames)]
    exp = ref.RefPlan(w, h, fmt, cfg).process(srcs)
    p = Plan(w, h, fmt, cfg)
    dev = [cuda.from_numpy(s).cuda() for s in srcs]
    out = cuda.empty_like(dev[0])
    p.process(dev, out)
    p.sync_status()
    host_out = p.process(srcs)            # host-memory entry point
    gpu = out.cpu().numpy()
    assert np.array_equal(gpu, host_out)
    return gpu, exp


FFT3D_T1 = [
    ("A-shape u8 32/16", 640, 360, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0, beta=1)),
    ("u10 chroma 16 sharpen+dehalo", 200, 120, SampleFormat(10, chroma=True),
     FFT3DConfig(bw=16, bh=16, sigma=3.0, sharpen=0.3, dehalo=0.2)),
    ("f32 8x8 wintype1", 128, 80, SampleFormat(32, True), FFT3DConfig(bw=8, bh=8, ow=4, oh=4, wintype=1, sigma=2.0)),
    ("u16 12x12 varying sigma", 100, 70, SampleFormat(16),
     FFT3DConfig(bw=12, bh=12, sigma=2, sigma2=3, sigma3=1.5, sigma4=4, sharpen=0.5)),
    ("u8 16x8 non-square", 96, 64, SampleFormat(8), FFT3DConfig(bw=16, bh=8, ow=5, oh=2, sigma=2.5)),
    ("u8 bt=-1 sharpen only", 96, 64, SampleFormat(8), FFT3DConfig(bw=16, bh=16, bt=-1, sharpen=0.7)),
    ("u12 wintype2 beta1.5", 150, 90, SampleFormat(12), FFT3DConfig(bw=32, bh=32, wintype=2, beta=1.5, sigma=4)),
    ("u8 degrid0", 96, 96, SampleFormat(8), FFT3DConfig(bw=8, bh=8, degrid=0, sigma=3)),
    ("u14 48x48", 260, 150, SampleFormat(14), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, sigma=3.0, sharpen=0.3)),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg", FFT3D_T1, ids=[c[0] for c in FFT3D_T1])
def test_fft3d_single_frame(ref, cuda, name, w, h, fmt, cfg):
    gpu, exp = run_both(ref, cuda, w, h, fmt, cfg, 1)
    check_parity(gpu, exp, fmt)


DFT_T1 = [
    ("B-shape u16 16/12 ftype0 curve", 480, 270, SampleFormat(16),
     DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8]), True),
    ("u8 ftype1", 130, 90, SampleFormat(8), DFTConfig(ftype=1, sigma=6.0), True),
    ("f32 ftype2 curve", 120, 88, SampleFormat(32, True),
     DFTConfig(ftype=2, sigma=0.8, ssx=[0, 1, 1, 0.5], ssy=[0, 1, 1, 0.7]), True),
    ("u10 ftype3", 110, 70, SampleFormat(10), DFTConfig(ftype=3, sigma=1.2, sigma2=0.4, pmin=2, pmax=200), True),
    ("u16 ftype4", 110, 70, SampleFormat(16), DFTConfig(ftype=4, sigma=1.0, pmin=5, pmax=300), True),
    ("u8 f0beta0.5", 96, 80, SampleFormat(8), DFTConfig(ftype=0, sigma=10, f0beta=0.5), True),
    ("u8 f0beta2 (pow)", 96, 80, SampleFormat(8), DFTConfig(ftype=0, sigma=10, f0beta=2.0), False),
    ("u8 smode0 centre 5", 64, 48, SampleFormat(8), DFTConfig(block=5, mode=0, sigma=4), True),
    ("f32 zmean off", 100, 60, SampleFormat(32, True), DFTConfig(zmean=False, sigma=3), True),
    ("u12 12/9 project", 144, 100, SampleFormat(12), DFTConfig(block=12, overlap=9, sigma=5, swin=2), True),
    ("u8 8/6 heavy overlap", 90, 70, SampleFormat(8), DFTConfig(block=8, overlap=6, sigma=4, swin=4), True),
    ("u16 32/16 radial curve", 200, 150, SampleFormat(16),
     DFTConfig(block=32, overlap=16, sigma=6, slocation=[0, 2, 0.5, 8, 1, 16], ssystem=1), True),
]


@pytest.mark.parametrize("name,w,h,fmt,cfg,exact", DFT_T1, ids=[c[0] for c in DFT_T1])
def test_dfttest_single_frame(ref, cuda, name, w, h, fmt, cfg, exact):
    gpu, exp = run_both(ref, cuda, w, h, fmt, cfg, 1, seed=(2, 0))
    check_parity(gpu, exp, fmt, exact)


def test_dfttest_full_hd_luma_and_chroma(ref, cuda):
    """The benchmark workload's planes at full size (1920x1080 and 960x540 u16)."""
    fmt = SampleFormat(16)
    cfg = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])
    for (w, h) in ((1920, 1080), (960, 540)):
        gpu, exp = run_both(ref, cuda, w, h, fmt, cfg, 1, seed=(2, 1))
        check_parity(gpu, exp, fmt)


def test_non_finite_input_is_reported(cuda):
    fmt = SampleFormat(32, True)
    p = Plan(64, 48, fmt, DFTConfig(sigma=2))
    x = plane(48, 64, 32, True, seed=(9, 9, 9))
    x[10, 20] = np.nan
    from neo_fft_b200 import NonFiniteError
    with pytest.raises(NonFiniteError, match="non-finite sample or intermediate"):
        p.process(x)
    x[10, 20] = 0.5
    p.process(x)  # flag was cleared; a finite frame succeeds


def test_shape_and_alias_errors(cuda):
    p = Plan(64, 48, SampleFormat(8), FFT3DConfig(bw=16, bh=16))
    x = np.zeros((48, 64), np.uint8)
    with pytest.raises(ValueError, match="frame dimensions differ from plan"):
        p.process(np.zeros((40, 64), np.uint8))
    with pytest.raises(ValueError, match="partially overlapping or aliased buffers"):
        p.process_at([x], x)
