"""ROI and interlaced packing on the device (src/plugin/roi.hpp): pack/unpack follow the
row order of ROI::row, and filtering the packed image then unpacking equals the
reference core on the host-packed image written back the same way."""
import numpy as np
import pytest

from neo_fft_b200.plan import ROI, DFTConfig, FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu


def _pack_np(a, r: ROI):
    return np.stack([a[r.top + r.row(y), r.left:r.left + r.width] for y in range(r.height)])


@pytest.mark.parametrize("interlaced", [False, True])
def test_pack_unpack_row_order(cuda, interlaced):
    a = plane(100, 140, 16, False, seed=(130, 0, 0))
    r = ROI.make(140, 100, 0, 0, left=8, top=6, right=4, bottom=10, interlaced=interlaced)
    d = cuda.from_numpy(a).cuda()
    packed = r.pack(d)
    assert np.array_equal(packed.cpu().numpy(), _pack_np(a, r))
    out = cuda.zeros_like(d)
    r.unpack(packed, out)
    exp = np.zeros_like(a)
    exp[r.top:r.top + r.height, r.left:r.left + r.width] = a[r.top:r.top + r.height, r.left:r.left + r.width]
    assert np.array_equal(out.cpu().numpy(), exp)


@pytest.mark.parametrize("fmt,cfg", [
    (SampleFormat(8), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, sigma=3.0)),
    (SampleFormat(32, True), DFTConfig(block=12, overlap=6, sigma=6.0)),
], ids=["fft3d-u8", "dft-f32"])
def test_interlaced_roi_filtering_matches_reference(cuda, ref, fmt, cfg):
    W, H = 160, 120
    a = plane(H, W, fmt.bits, fmt.floating, seed=(131, 0, 0))
    r = ROI.make(W, H, 1, 1, left=8, top=4, right=16, bottom=12, interlaced=True)
    d = cuda.from_numpy(a).cuda()
    p = Plan(r.width, r.height, fmt, cfg)
    filtered = p.process(r.pack(d))
    out = d.clone()
    r.unpack(filtered, out)
    packed_host = _pack_np(a, r)
    ref_filtered = ref.RefPlan(r.width, r.height, fmt, cfg).process(packed_host)
    exp = a.copy()
    for y in range(r.height):
        exp[r.top + r.row(y), r.left:r.left + r.width] = ref_filtered[y]
    assert np.array_equal(out.cpu().numpy(), exp)


def test_reference_roi_code_through_facade(cuda, ref, tmp_path):
    """The reference host layer's ROI code (src/plugin/roi.hpp, compiled unchanged against the
    facade by tests/test_capi.py into tests/native/_bin/roi_facade_check) on an interlaced ROI:
    FFT3D bt=3, Kalman render and the sampled-pattern filter each equal the reference core
    on the host-packed image, written back in the ROI's row order."""
    import subprocess
    from pathlib import Path
    exe = Path(__file__).resolve().parent / "native" / "_bin" / "roi_facade_check"
    if not exe.exists():
        pytest.skip("roi_facade_check not built (needs the reference sources at build time)")
    W, H = 160, 120
    a = plane(H, W, 8, False, seed=(132, 0, 0))
    paths = [tmp_path / n for n in ("in.u8", "fft3d.u8", "kalman.f32", "pattern.u8")]
    a.tofile(paths[0])
    run = subprocess.run([str(exe), *map(str, paths)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    r = ROI.make(W, H, 0, 0, left=8, top=4, right=16, bottom=12, interlaced=True)
    packed = _pack_np(a, r)

    def write_back(base, filtered):
        out = base.copy()
        for y in range(r.height):
            out[r.top + r.row(y), r.left:r.left + r.width] = filtered[y]
        return out
    cfg = FFT3DConfig(bw=16, bh=16, ow=8, oh=8, sigma=3.0, bt=3)
    exp = write_back(a, ref.RefPlan(r.width, r.height, SampleFormat(8), cfg).process([packed] * 3))
    assert np.array_equal(np.fromfile(paths[1], np.uint8).reshape(H, W), exp)
    fa = (a.astype(np.float32) / np.float32(255.0)).astype(np.float32)
    fpk = _pack_np(fa, r)
    kp = ref.RefPlan(r.width, r.height, SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, sigma=3.0,
                                                                           bt=0, kratio=2.0))
    st = kp.kalman_state()
    for _ in range(2):
        kp.advance_kalman(fpk, st)
    exp_k = write_back(fa, kp.render_kalman(fpk, st))
    assert np.array_equal(np.fromfile(paths[2], np.float32).reshape(H, W), exp_k)
    pp = ref.RefPlan(r.width, r.height, SampleFormat(8), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, sigma=3.0,
                                                                     pfactor=1.0))
    pp.publish_pattern(pp.pattern_candidate(packed))
    exp_p = write_back(a, pp.process([packed]))
    assert np.array_equal(np.fromfile(paths[3], np.uint8).reshape(H, W), exp_p)
