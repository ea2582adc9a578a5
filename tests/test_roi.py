"""ROI validation (make_roi, src/plugin/roi.hpp:13-23) on the host; device packing is
covered by tests/test_gpu_roi.py."""
import pytest

from neo_fft_b200.plan import ROI


def test_roi_validation_messages():
    with pytest.raises(ValueError, match="align to subsampling"):
        ROI.make(100, 80, 1, 1, left=3)
    with pytest.raises(ValueError, match="ROI must be nonempty"):
        ROI.make(100, 80, 0, 0, left=60, right=40)
    with pytest.raises(ValueError, match="interlaced ROI height must be even"):
        ROI.make(100, 81, 0, 0, interlaced=True)


def test_roi_margins_and_field_order():
    r = ROI.make(160, 120, 1, 1, left=8, top=4, right=16, bottom=12, interlaced=True)
    assert (r.left, r.top, r.width, r.height) == (4, 2, 148, 112)  # margins halved for 4:2:0 chroma
    assert [r.row(y) for y in range(r.height)][:3] == [0, 2, 4]
    assert [r.row(y) for y in range(r.height)][-3:] == [5, 3, 1]
