"""Index arithmetic of the Kalman step's overlap-add (kalman_ola_kernel in
neo_fft_b200/csrc/kalman.cuh), checked on the CPU over many FFT3D axes: the covering blocks
the kernel derives with one division per axis are exactly the blocks whose span holds the
pixel (at most two, since FFT3D overlaps are at most half a block), and the 2- and 4-pixel
groups it forms share their covering blocks and read inside each block's row. The axis
formula is the reference's fft3d_axis (src/spectral/geometry.hpp:15-24)."""
import itertools


def fft3d_axis(length, block, overlap):
    if overlap < 0:
        overlap = block // 3
    step = block - overlap
    count = -(-(length - overlap) // step) + 2
    return {"length": length, "block": block, "step": step, "count": count, "cover": count * step + overlap,
            "offset": step}


def covering(a, c):
    """Blocks whose span [b*step, b*step + block) holds cover coordinate c (the definition)."""
    return [b for b in range(a["count"]) if b * a["step"] <= c < b * a["step"] + a["block"]]


def kernel_range(a, c):
    """The kernel's derivation: the last block starting at or before c, and the one before it
    when c lies within that block's length."""
    b1 = min(a["count"] - 1, c // a["step"])
    b0 = b1 - 1 if b1 > 0 and c - (b1 - 1) * a["step"] < a["block"] else b1
    return b0, b1


def width_of(a):
    m = a["step"] | a["block"] | a["offset"]
    return 4 if m % 4 == 0 else 2 if m % 2 == 0 else 1


AXES = [fft3d_axis(L, B, o) for L, B, o in itertools.product(
    (33, 70, 95, 96, 120, 160, 200, 257, 1080, 1920), (4, 8, 12, 16, 20, 32, 48), (-1, 0, 1, 3, 5, 8, 10, 16, 24))
    if o <= B // 2 and L >= B]


def test_covering_blocks_match_the_definition():
    for a in AXES:
        for c in range(a["offset"], a["offset"] + a["length"]):
            b0, b1 = kernel_range(a, c)
            assert list(range(b0, b1 + 1)) == covering(a, c), (a, c)
            assert 1 <= b1 - b0 + 1 <= 2


def test_pixel_groups_share_blocks_and_stay_in_rows():
    for a in AXES:
        V = width_of(a)
        for x in range(0, a["length"], V):
            c = x + a["offset"]
            b0, b1 = kernel_range(a, c)
            for e in range(V):
                if x + e < a["length"]:  # stored pixels: the same covering blocks
                    assert kernel_range(a, c + e) == (b0, b1), (a, x, e)
                for b in range(b0, b1 + 1):  # every loaded sample lies in its block's row
                    assert 0 <= c + e - b * a["step"] < a["block"], (a, x, e, b)
            if V > 1:  # the vector load starts on a V-element boundary of the row
                for b in range(b0, b1 + 1):
                    assert (c - b * a["step"]) % V == 0


def test_axis_formula_equals_reference(ref):
    """The axis formula above is the reference's own: every axis of the sweep that the
    reference accepts as a plane width equals the geometry of a reference FFT3D plan built on
    it (the oracle library)."""
    from neo_fft_b200.plan import FFT3DConfig, SampleFormat
    checked = 0
    for a in AXES:
        if a["length"] > 400:  # the wide planes add nothing to the formula check
            continue
        overlap = a["block"] - a["step"]
        try:
            plan = ref.RefPlan(a["length"], 32, SampleFormat(8), FFT3DConfig(bw=a["block"], bh=8, ow=overlap, oh=0,
                                                                              bt=0, sigma=2.0))
        except ValueError:  # padding beyond one reflection of a narrow plane: no plan to compare
            continue
        assert {k: plan.x[k] for k in ("length", "block", "step", "count", "cover", "offset")} == \
            {k: a[k] for k in ("length", "block", "step", "count", "cover", "offset")}, a
        checked += 1
    assert checked > 100
