"""CPU checks that pin the oracle: the reference core compiled from source, checked
against the known answers published in the reference's docs and unit tests, and
the shared transform arithmetic checked against the reference codelets.
"""
import numpy as np
import pytest

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, SampleFormat


def test_codelet_replica_bit_exact(ref):
    """fft_core.cuh's 8/16/32 networks equal the reference AVX2 codelets bit for bit
    (src/spectral/codelets/*_avx2.cpp), forward and inverse."""
    lib = ref.load()
    rng = np.random.default_rng(1)
    for n in (8, 16, 32):
        k = n // 2 + 1
        for trial in range(40):
            x = (rng.standard_normal((n, n)) * rng.choice([1e-3, 1, 300])).astype(np.float32)
            a = np.zeros((n, k, 2), np.float32)
            b = np.zeros((n, k, 2), np.float32)
            lib.ref_fft_r2c(n, n, ref.fp(x), ref.fp(a))
            lib.ref_replica_r2c(n, n, ref.fp(x), ref.fp(b))
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
            ya = np.zeros((n, n), np.float32)
            yb = np.zeros((n, n), np.float32)
            lib.ref_fft_c2r(n, n, ref.fp(a), ref.fp(ya))
            lib.ref_replica_c2r(n, n, ref.fp(a), ref.fp(yb))
            assert np.array_equal(ya.view(np.uint32), yb.view(np.uint32)), n


@pytest.mark.parametrize("h,w", [(12, 12), (48, 48), (6, 8), (5, 7), (9, 9), (3, 3), (20, 20), (64, 64), (2, 4),
                                 (1, 1), (8, 16), (24, 24), (15, 15), (7, 11)])
def test_project_transform_vs_binary64(ref, h, w):
    """The project mixed-radix transform (stand-in for PocketFFT) agrees with a
    binary64 DFT within the reference's FFT test tolerances (tests/unit/foundation.cpp:65-75)."""
    rng = np.random.default_rng(h * 100 + w)
    x = rng.standard_normal((h, w)).astype(np.float32)
    got = ref.r2c(x)
    exp = np.fft.rfft2(x.astype(np.float64))
    assert np.abs(got - exp).max() <= 3e-5 * max(1.0, np.abs(exp).max())
    spec = np.stack([got.real, got.imag], -1).astype(np.float32)
    y = np.zeros((h, w), np.float32)
    ref.load().ref_fft_c2r(h, w, ref.fp(spec), ref.fp(y))
    assert np.abs(y - x).max() <= 2e-6 * max(1.0, np.abs(x).max()) * 4


def test_fft3d_worked_example(ref):
    """docs/knowledge/en/fft3d.md:128-150: rows [10,14] -> [10,13] with bw=bh=4,
    ow=oh=0, sigma=4, degrid=0."""
    img = np.tile(np.array([10, 14], np.uint8), (16, 8))
    plan = ref.RefPlan(16, 16, SampleFormat(8), FFT3DConfig(bw=4, bh=4, ow=0, oh=0, bt=1, sigma=4, beta=1, degrid=0))
    out = plan.process(img)
    assert np.array_equal(out, np.tile(np.array([10, 13], np.uint8), (16, 8)))


def test_dfttest_mean_example(ref):
    """docs/knowledge/en/dfttest.md:27-33 and tests/unit/algorithms.cpp:119-153:
    [1,2,6] -> 3 with zmean, 0 without."""
    srcs = [np.array([[v]], np.uint8) for v in (1, 2, 6)]
    c = DFTConfig(block=1, mode=0, tbsize=3, swin=7, twin=7, ftype=2, sigma=0, zmean=True)
    assert ref.RefPlan(1, 1, SampleFormat(8), c).process(srcs)[0, 0] == 3
    c.zmean = False
    assert ref.RefPlan(1, 1, SampleFormat(8), c).process(srcs)[0, 0] == 0
    fsrc = [np.array([[v / 255]], np.float32) for v in (1, 2, 6)]
    c.zmean = True
    out = ref.RefPlan(1, 1, SampleFormat(32, True), c).process(fsrc)
    assert abs(out[0, 0] - 3 / 255) < 1e-7


def test_temporal_identities(ref):
    """tests/unit/algorithms.cpp:155-200: bt=3 and tbsize=3 sigma=0 identities."""
    f = [np.full((16, 16), v, np.uint8) for v in (10, 20, 30)]
    p = ref.RefPlan(16, 16, SampleFormat(8), FFT3DConfig(bw=8, bh=8, ow=4, oh=4, bt=3, sigma=0))
    assert np.array_equal(p.process(f), f[1])
    p = ref.RefPlan(16, 16, SampleFormat(8), DFTConfig(block=8, overlap=4, mode=1, tbsize=3, swin=7, twin=7,
                                                       ftype=2, sigma=1.0, zmean=False))
    assert np.array_equal(p.process(f), f[1])
    with pytest.raises(ValueError, match="DFTTest sources size must match plan temporal_size"):
        p.process(f[:2])


def test_dfttest_temporal_ola_example(ref):
    """docs/knowledge/en/dfttest/temporal-ola.md:33-37: amplitudes [0,2,4,6,8,10],
    T=4, O=2, ftype=2, sigma=0, zmean -> output n=2 is 5."""
    from neo_fft_b200.plan import DFTConfig
    vals = [0, 2, 4, 6, 8, 10]
    frames = [np.array([[v]], np.uint8) for v in vals]
    c = DFTConfig(block=1, mode=0, tbsize=4, swin=7, twin=7, ftype=2, sigma=0, zmean=True, temporal_mode=1,
                  temporal_overlap=2)
    p = ref.RefPlan(1, 1, SampleFormat(8), c)
    # covering blocks of n=2 for N=6: starts 0 and 2 -> targets 2 and 0
    srcs = [frames[min(max(s + z, 0), 5)] for s in (0, 2) for z in range(4)]
    out = p.process(srcs, targets=[2, 0])
    assert out[0, 0] == 5


def test_golden_fixtures_match_reference(ref):
    """tests/golden/smoke.npz was produced by the reference core; regenerating it
    from oracle/_ref gives identical outputs."""
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "smoke.npz")
    d = ref.RefPlan(128, 96, SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0,
                                                         slocation=[0, 8, 1, 8])).process(g["dft_in"])
    assert np.array_equal(d, g["dft_out"])
    f = ref.RefPlan(160, 96, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0)).process(g["fft3d_in"])
    assert np.array_equal(f, g["fft3d_out"])


def test_temporal_lattice_examples():
    """docs/knowledge/en/dfttest/temporal-ola.md:20-29 table and endpoint example."""
    from neo_fft_b200.temporal import temporal_blocks
    cases = {(4, 2, 0): ([-2, 0], [2, 0]), (4, 2, 3): ([0, 2], [3, 1]), (5, 2, 0): ([-3, 0], [3, 0]),
             (5, 2, 2): ([0], [2]), (4, 0, 4): ([4], [0])}
    for (t, o, n), (starts, targets) in cases.items():
        b = temporal_blocks(n, 20, t, o)
        assert [x["start"] for x in b] == starts and [x["target"] for x in b] == targets
    b = temporal_blocks(4, 5, 4, 2)
    assert [x["slots"] for x in b] == [[2, 3, 4, 4], [4, 4, 4, 4]]
    with pytest.raises(ValueError, match="DFTTest temporal heavy overlap requires divisible step"):
        temporal_blocks(0, 10, 5, 3)


def test_temporal_lattice_equals_reference(ref):
    """neo_fft_b200.temporal.temporal_blocks (the tmode 1 frame selection of the clip forms,
    the frame server and the shards) equals the reference's temporal_grid.hpp:24-40 for every
    tbsize 1..15, every tosize 0..tbsize (invalid and heavy ones included), clips of tbsize - 1
    to 40 frames and every frame index from -1 to the clip length: the same blocks, targets and
    clamped slots, or the same error text."""
    from neo_fft_b200.temporal import temporal_blocks
    checked = rejected = 0
    for size in range(1, 16):
        for overlap in range(0, size + 1):
            for length in sorted({size - 1, size, size + 1, 2 * size + 3, 40}):
                for frame in range(-1, length + 1):
                    try:
                        want = ref.temporal_blocks(frame, length, size, overlap)
                    except ValueError as e:
                        with pytest.raises(ValueError) as mine:
                            temporal_blocks(frame, length, size, overlap)
                        assert str(mine.value) == str(e), (frame, length, size, overlap)
                        rejected += 1
                        continue
                    assert temporal_blocks(frame, length, size, overlap) == want, (frame, length, size, overlap)
                    checked += 1
    assert checked == 7888 and rejected > 0, (checked, rejected)  # 7,888 valid (frame, clip, tbsize, tosize)


def test_kernel_bin_arithmetic_equals_reference_kernels(ref):
    """The kernels' per-bin arithmetic (neo_fft_b200/csrc/device_plan.cuh: spectral_bin for FFT3D
    Wiener with floor, table, template and enhancement, DFTTest ftype 0..4 and every ftype 0
    exponent mode; ratio_bin; enhancement_gain; kalman_bin), compiled as host code, against the
    reference's own scalar kernels (spectral.cpp, fft3d_profile.cpp, kalman.cpp) from the oracle
    library: 40,000 seeded random bins per case over many decades, with zeros, subnormals and
    bins on the thresholds, equal bit for bit (tests/native/bin_math_check.cpp). Bins the
    reference rejects are flagged too, except those whose only non-finite intermediate is an
    overflowing sharpen or ftype 4 denominator at powers above 1e19."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    if not (ref.REFERENCE / "src" / "kernels" / "spectral.hpp").exists():
        pytest.skip("reference sources absent")
    exe = root / "tests" / "_build" / "bin_math_check"
    exe.parent.mkdir(exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O1", "-fno-fast-math", "-ffp-contract=off", "-DNEO_FFT_ENABLE_HIGHWAY=0",
                    f"-I{ref.REFERENCE / 'src'}", f"-I{root / 'oracle' / 'shim'}", f"-I{root / 'include'}",
                    f"-I{root / 'neo_fft_b200' / 'csrc'}", str(root / "tests" / "native" / "bin_math_check.cpp"),
                    "-o", str(exe), f"-L{ref.LIB.parent}", "-lneofft_ref", f"-Wl,-rpath,{ref.LIB.parent}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    counts = dict(line.split() for line in r.stdout.splitlines())
    assert r.returncode == 0, r.stdout
    assert len(counts) == 15 and all(int(v) == 0 for k, v in counts.items() if k != "overflow_only"), counts


def test_project_transform_random_shapes_vs_binary64(ref):
    """The 2-D real transforms of non-codelet block shapes (fft_core.cuh block_r2c/block_c2r,
    reached through the oracle's stand-in backend) against binary64 for 48 seeded random shapes
    with sides 1..128 whose prime factors are at most 64: forward within 3e-5 of the largest
    output (tests/unit/foundation.cpp:65-75), the round trip within 8e-6 of the largest input."""
    rng = np.random.default_rng(64)
    lib = ref.load()
    done = 0
    while done < 48:
        h, w = (int(v) for v in rng.integers(1, 129, 2))
        if any(max(p for p in range(1, n + 1) if n % p == 0 and all(p % q for q in range(2, p))) > 64
               for n in (h, w)) or (h == w and w in (8, 16, 32)):
            continue
        x = rng.standard_normal((h, w)).astype(np.float32)
        got = ref.r2c(x)
        exp = np.fft.rfft2(x.astype(np.float64))
        assert np.abs(got - exp).max() <= 3e-5 * max(1.0, np.abs(exp).max()), (h, w)
        spec = np.ascontiguousarray(np.stack([got.real, got.imag], -1).astype(np.float32))
        y = np.zeros((h, w), np.float32)
        lib.ref_fft_c2r(h, w, ref.fp(spec), ref.fp(y))
        assert np.abs(y - x).max() <= 8e-6 * max(1.0, np.abs(x).max()), (h, w)
        done += 1


def test_volume_transform_vs_binary64(ref):
    """The 3-D real transform of DFTTest volumes (the reference's RealFFT3D over the stand-in
    backend: the spatial 2-D transform per slice, then the temporal axis, the order the volume
    kernels use) against a binary64 3-D DFT for every temporal length 2..15 on codelet and
    non-codelet block shapes: forward within 3e-5 of the largest output, the inverse round trip
    within 8e-6 of the largest input."""
    lib = ref.load()
    rng = np.random.default_rng(65)
    for d in range(2, 16):
        for h, w in ((8, 8), (12, 12), (16, 16), (9, 10), (5, 7)):
            x = rng.standard_normal((d, h, w)).astype(np.float32)
            out = np.zeros((d, h, w // 2 + 1, 2), np.float32)
            lib.ref_fft_r2c_3d(d, h, w, ref.fp(x), ref.fp(out))
            got = out[..., 0] + 1j * out[..., 1]
            exp = np.fft.rfftn(x.astype(np.float64))
            assert np.abs(got - exp).max() <= 3e-5 * np.abs(exp).max(), (d, h, w)
            y = np.zeros_like(x)
            lib.ref_fft_c2r_3d(d, h, w, ref.fp(out), ref.fp(y))
            assert np.abs(y - x).max() <= 8e-6 * np.abs(x).max(), (d, h, w)
