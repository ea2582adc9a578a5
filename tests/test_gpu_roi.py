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
