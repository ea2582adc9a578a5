"""DFTTest 8-bit output with dither > 0 (src/kernels/scalar/dither.cpp): the GPU wavefront
error diffusion equals the reference core bit for bit, including the hashed noise of
modes >= 2 (frame and plane coordinates), bands of more than 1024 rows and narrow planes."""
import numpy as np
import pytest

from neo_fft_b200.plan import Batch, DFTConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,mode,seed,frame,pl,tbsize", [
    (160, 120, 1, 0, 0, 0, 1),
    (160, 120, 2, 7, 5, 1, 1),
    (96, 1100, 3, 123, 2, 2, 1),
    (33, 70, 5, 1, 9, 0, 1),
    (128, 96, 2, 3, 4, 0, 3),
])
def test_dither_matches_reference(cuda, ref, w, h, mode, seed, frame, pl, tbsize):
    fmt = SampleFormat(8)
    cfg = DFTConfig(block=16, overlap=8, sigma=4.0, dither=mode, dither_seed=seed, tbsize=tbsize)
    srcs = [plane(h, w, 8, False, seed=(120, 0, f)) for f in range(tbsize)]
    p = Plan(w, h, fmt, cfg)
    out = cuda.empty((h, w), dtype=cuda.uint8, device="cuda")
    p.process_at([cuda.from_numpy(s).cuda() for s in srcs], out, frame=frame, plane=pl)
    exp = ref.RefPlan(w, h, fmt, cfg).process(srcs, frame=frame, plane=pl)
    got = out.cpu().numpy()
    assert np.array_equal(got, exp), int((got != exp).sum())
    p.sync_status()


def test_dither_ignored_for_16_bit_and_rejected_in_batches(cuda):
    cfg = DFTConfig(block=16, overlap=8, sigma=4.0, dither=2)
    p16 = Plan(64, 48, SampleFormat(16), cfg)
    ref16 = Plan(64, 48, SampleFormat(16), DFTConfig(block=16, overlap=8, sigma=4.0))
    src = plane(48, 64, 16, False, seed=(121, 0, 0))
    assert np.array_equal(p16.process(src), ref16.process(src))
    p8 = Plan(64, 48, SampleFormat(8), cfg)
    a = cuda.zeros((48, 64), dtype=cuda.uint8, device="cuda")
    # without frame and plane numbers a batch cannot seed the dither noise
    with pytest.raises(ValueError, match="dithered 8-bit DFTTest output"):
        Batch([(p8, a, cuda.empty_like(a))])


def test_dithered_items_in_indexed_batches(cuda):
    """Batches whose items carry frame and plane numbers take dithered 8-bit DFTTest planes:
    each output equals process_at(..., frame, plane) bit for bit, beside undithered planes
    of the same plan shape, plain and replayed from the graph."""
    fmt = SampleFormat(8)
    specs = [  # (w, h, dither mode, seed, frame, plane)
        (160, 120, 1, 0, 0, 0), (160, 120, 2, 7, 5, 1), (96, 1100, 3, 123, 2, 2), (33, 70, 5, 1, 9, 0),
        (128, 96, 4, 3, 4, 1),
    ]
    items, expect = [], []
    for i, (w, h, mode, seed, frame, pl) in enumerate(specs):
        p = Plan(w, h, fmt, DFTConfig(block=16, overlap=8, sigma=4.0, dither=mode, dither_seed=seed))
        src = cuda.from_numpy(plane(h, w, 8, False, seed=(122, i, 0))).cuda()
        e = cuda.empty_like(src)
        p.process_at([src], e, frame=frame, plane=pl)
        items.append((p, src, cuda.zeros_like(src), frame, pl))
        expect.append(e)
    plain = Plan(160, 120, fmt, DFTConfig(block=16, overlap=8, sigma=4.0))
    psrc = cuda.from_numpy(plane(120, 160, 8, False, seed=(122, 9, 0))).cuda()
    pexp = cuda.empty_like(psrc)
    plain.process_at([psrc], pexp)
    items.append((plain, psrc, cuda.zeros_like(psrc)))
    expect.append(pexp)
    batch = Batch(items)
    for graph in (False, True):
        for it in items:
            it[2].zero_()
        batch.launch(graph=graph)
        for it, e in zip(items, expect):
            assert cuda.equal(it[2], e), (it[0], graph)
    batch.sync_status()
