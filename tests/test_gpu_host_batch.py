"""Streamed host form (nf_host_batch): frames in host memory through a ring of device
slots, copies overlapped with the batched launch on separate streams. Every output
plane equals the reference core's Plan::process on the same plane bit for bit —
with partial last chunks, slot reuse across calls, pageable and page-locked host
buffers, strided host rows and in-place calls."""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, HostBatch, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu

DFT = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])


def _frames(n, sizes, fmt, seed):
    return [[plane(h, w, fmt.bits, fmt.floating, seed=(seed, f, p)) for p, (w, h) in enumerate(sizes)]
            for f in range(n)]


def test_host_batch_equals_reference_per_plane(ref, cuda):
    fmt = SampleFormat(16)
    sizes = [(320, 180), (160, 90), (160, 90)]
    luma, chroma = Plan(320, 180, fmt, DFT), Plan(160, 90, fmt, DFT)
    rl, rc = ref.RefPlan(320, 180, fmt, DFT), ref.RefPlan(160, 90, fmt, DFT)
    hb = HostBatch([luma, chroma, chroma], frames_per_chunk=3, depth=2)
    assert hb.device_bytes >= 2 * 2 * 3 * (320 * 180 + 2 * 160 * 90) * 2
    frames = _frames(7, sizes, fmt, 31)               # chunks of 3, 3, 1: the last one partial
    pinned = [[cuda.from_numpy(x).pin_memory() for x in f] for f in frames]
    out = hb.process(pinned)
    hb.sync_status()
    for f in range(7):
        for p, r in enumerate((rl, rc, rc)):
            assert np.array_equal(out[f][p].numpy(), r.process([frames[f][p]])), (f, p)
    # Second call reuses the slots (and their captured graphs); pageable numpy buffers.
    frames2 = _frames(5, sizes, fmt, 32)
    out2 = hb.process(frames2)
    for f in range(5):
        for p, r in enumerate((rl, rc, rc)):
            assert np.array_equal(out2[f][p], r.process([frames2[f][p]])), (f, p)


@pytest.mark.parametrize("fmt,cfg,size", [
    (SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0, sharpen=0.3), (200, 120)),
    (SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0), (256, 144)),
    (SampleFormat(10), DFTConfig(block=12, overlap=9, ftype=1, sigma=6.0), (150, 98)),
], ids=["u8-fft3d32", "f32-dft16", "u10-dft12"])
def test_host_batch_formats_strided_and_in_place(cuda, fmt, cfg, size):
    w, h = size
    p = Plan(w, h, fmt, cfg)
    hb = HostBatch([p], frames_per_chunk=2, depth=3)
    frames = _frames(5, [size], fmt, 33)
    padded = []
    for f in frames:                                   # host rows longer than the plane
        big = np.zeros((h, w + 40), dtype=f[0].dtype)
        big[:, :w] = f[0]
        padded.append([big[:, :w]])
    out = hb.process(padded)
    exp = [p.process([f[0]]) for f in frames]
    for f in range(5):
        assert np.array_equal(out[f][0], exp[f]), f
    inplace = [[x[0].copy()] for x in frames]
    hb.process(inplace, outputs=inplace)
    for f in range(5):
        assert np.array_equal(inplace[f][0], exp[f]), f


def test_host_batch_rejects_bad_inputs(cuda):
    p = Plan(64, 48, SampleFormat(8), DFTConfig(tbsize=3))
    with pytest.raises(ValueError, match="single-frame plans"):
        HostBatch([p])
    q = Plan(64, 48, SampleFormat(8), DFTConfig())
    with pytest.raises(ValueError, match="depth"):
        HostBatch([q], depth=1)
    hb = HostBatch([q])
    with pytest.raises(ValueError, match="frame dimensions"):
        hb.process([[np.zeros((40, 64), np.uint8)]])
    with pytest.raises(ValueError, match="planes"):
        hb.process([[np.zeros((48, 64), np.uint8)] * 2])
    assert hb.process([]) == []
