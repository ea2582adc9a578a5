"""Creation-time tables of the product (neo_fft_b200/csrc/plan_build.cpp) against the
reference core's own tables (oracle/_ref), bit for bit, plus configuration errors
with the reference's texts. CPU only: the product's table builder is compiled into
a small host shim (tests/native/tables_shim.cpp)."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from neo_fft_b200 import _capi as C
from neo_fft_b200.plan import DFTConfig, FFT3DConfig, SampleFormat

ROOT = Path(__file__).resolve().parents[1]
SHIM = ROOT / "tests" / "_build" / "libtables_shim.so"


@pytest.fixture(scope="module")
def tb():
    srcs = [ROOT / "tests" / "native" / "tables_shim.cpp", ROOT / "neo_fft_b200" / "csrc" / "plan_build.cpp"]
    SHIM.parent.mkdir(exist_ok=True)
    if not SHIM.exists() or any(s.stat().st_mtime > SHIM.stat().st_mtime for s in srcs):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        f"-I{ROOT / 'include'}", f"-I{ROOT / 'neo_fft_b200' / 'csrc'}", *map(str, srcs),
                        "-o", str(SHIM)], check=True)
    lib = ctypes.CDLL(str(SHIM))
    lib.tb_dft_window_3d.argtypes = [ctypes.c_int] * 6 + [ctypes.c_float] * 2 + [ctypes.c_int] * 2 + \
        [ctypes.c_void_p, ctypes.c_void_p]
    lib.tb_plan.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, C.NfFormat, ctypes.c_void_p] + \
        [ctypes.c_void_p] * 7 + [ctypes.c_char_p, ctypes.c_size_t]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_fft3d_windows(tb, ref):
    lib = ref.load()
    for b in (4, 8, 9, 16, 32, 48):
        for o in {0, 1, b // 3, b // 2}:
            for t in (0, 1, 2):
                a1, s1, a2, s2 = (np.zeros(b, np.float32) for _ in range(4))
                assert tb.tb_fft3d_window(b, o, t, _p(a1), _p(s1)) == 0
                err = ctypes.create_string_buffer(256)
                assert lib.ref_fft3d_window(b, o, t, ref.fp(a2), ref.fp(s2), err, 256) == 0
                assert np.array_equal(a1, a2) and np.array_equal(s1, s2)


def test_dft_windows(tb, ref):
    lib = ref.load()
    for (tbs, b, o, mode, tmode, tov) in [(1, 16, 12, 1, 0, 0), (1, 12, 9, 1, 0, 0), (5, 12, 9, 1, 1, 0),
                                          (3, 8, 4, 1, 0, 0), (1, 9, 0, 0, 0, 0), (4, 6, 3, 1, 1, 2)]:
        for sw in range(12):
            n = tbs * b * b
            h1, h2 = np.zeros(n, np.float32), np.zeros(n, np.float32)
            w1, w2 = np.zeros(1, np.float32), np.zeros(1, np.float32)
            assert tb.tb_dft_window_3d(tbs, b, o, mode, sw, 7 if sw % 2 else sw, 2.5, 2.5, tmode, tov, _p(h1),
                                       _p(w1)) == 0
            err = ctypes.create_string_buffer(256)
            assert lib.ref_dft_window_3d(tbs, b, o, mode, sw, 7 if sw % 2 else sw, 2.5, 2.5, tmode, tov,
                                         ref.fp(h2), ref.fp(w2), err, 256) == 0
            assert np.array_equal(h1, h2) and w1[0] == w2[0]


def _product_tables(tb, algo, w, h, fmt, cfg):
    sizes = np.zeros(16, np.int32)
    big = [np.zeros(1 << 16, np.float32) for _ in range(5)]
    scal = np.zeros(16, np.float32)
    err = ctypes.create_string_buffer(256)
    if algo == 0:
        c = cfg.to_c()
    else:
        c, keep = cfg.to_c()
    fm = C.NfFormat(fmt.bits, int(fmt.floating), int(fmt.chroma))
    rc = tb.tb_plan(algo, w, h, fm, ctypes.addressof(c), _p(sizes), *[_p(x) for x in big], _p(scal), err, 256)
    if rc:
        raise (ValueError if rc == 1 else RuntimeError)(err.value.decode())
    return sizes, big, scal


FFT3D_CASES = [
    (640, 360, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0)),
    (960, 540, SampleFormat(10, chroma=True), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3)),
    (200, 120, SampleFormat(16), FFT3DConfig(bw=16, bh=8, sigma=2, sigma2=3, sigma3=1, sigma4=4, dehalo=0.5)),
    (100, 80, SampleFormat(32, True), FFT3DConfig(bw=12, bh=12, bt=0, sigma=2.5, kratio=2.0)),
]


@pytest.mark.parametrize("w,h,fmt,cfg", FFT3D_CASES)
def test_fft3d_plan_tables_match_reference(tb, ref, w, h, fmt, cfg):
    """Geometry, noise, enhancement and degrid template equal the reference's
    (src/algorithms/plan.cpp:91-169). The template is compared through the whole
    filter in the GPU tests; here it is checked against the reference's FFT of the
    same window block."""
    sizes, big, scal = _product_tables(tb, 0, w, h, fmt, cfg)
    rp = ref.RefPlan(w, h, fmt, cfg)
    assert (sizes[5], sizes[6], sizes[7], sizes[8], sizes[9], sizes[10]) == (
        rp.x["count"], rp.y["count"], rp.x["cover"], rp.y["cover"], rp.x["offset"], rp.y["offset"])
    # degrid template: FFT(peak * wy * wx) through the reference transform
    if cfg.degrid:
        a = np.zeros(cfg.bw, np.float32)
        s = np.zeros(cfg.bw, np.float32)
        ay = np.zeros(cfg.bh, np.float32)
        sy = np.zeros(cfg.bh, np.float32)
        tb.tb_fft3d_window(cfg.bw, rp.x["overlap"], cfg.wintype, _p(a), _p(s))
        tb.tb_fft3d_window(cfg.bh, rp.y["overlap"], cfg.wintype, _p(ay), _p(sy))
        peak = np.float32(1.0 if fmt.floating else (1 << fmt.bits) - 1)
        block = ((peak * ay[:, None]).astype(np.float32) * a[None, :]).astype(np.float32)
        exp = ref.r2c(block).astype(np.complex64)
        got = big[0][: 2 * sizes[0]].view(np.complex64).reshape(exp.shape)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))
    if cfg.sigma2 is not None:
        sig = np.array([cfg.sigma, cfg.sigma2, cfg.sigma3, cfg.sigma4], np.float32) * np.float32(1 << (fmt.bits - 8))
        exp = np.zeros(cfg.bh * (cfg.bw // 2 + 1), np.float32)
        err = ctypes.create_string_buffer(256)
        ref.load().ref_fft3d_profile(cfg.bw, cfg.bh, ref.fp(sig), ref.fp(exp), err, 256)
        assert np.array_equal(big[1][: sizes[1]], exp)


DFT_CASES = [
    (1920, 1080, SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])),
    (1920, 1080, SampleFormat(32, True), DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1)),
    (257, 131, SampleFormat(8), DFTConfig(block=8, overlap=4, tbsize=3, ftype=3, sigma=2, sigma2=0.5, pmin=1, pmax=80,
                                          ssx=[0, 1, 0.5, 3, 1, 5], ssystem=0)),
    (100, 64, SampleFormat(10), DFTConfig(block=9, mode=0, ftype=4, sigma=1.5, pmin=2, pmax=60,
                                          slocation=[0, 1, 0.4, 4, 1, 9], ssystem=1)),
]


@pytest.mark.parametrize("w,h,fmt,cfg", DFT_CASES)
def test_dft_plan_tables_match_reference(tb, ref, w, h, fmt, cfg):
    sizes, big, scal = _product_tables(tb, 1, w, h, fmt, cfg)
    rp = ref.RefPlan(w, h, fmt, cfg)
    assert (sizes[5], sizes[6], sizes[7], sizes[8], sizes[9], sizes[10]) == (
        rp.x["count"], rp.y["count"], rp.x["cover"], rp.y["cover"], rp.x["offset"], rp.y["offset"])
    # primary table against the reference profile builder
    if sizes[1]:
        c, keep = cfg.to_c()
        exp = np.zeros(sizes[1], np.float32)
        err = ctypes.create_string_buffer(256)
        ref.load().ref_dft_profile(ctypes.byref(c), np.float32(1.0 / scal[5]) if cfg.ftype < 2 else np.float32(1),
                                   ref.fp(exp), err, 256)
        # the reference divides by wscale (scale = 1/E); recompute through its own window
        h = np.zeros(sizes[4], np.float32)
        w1 = np.zeros(1, np.float32)
        ref.load().ref_dft_window_3d(cfg.tbsize, cfg.block, 0 if cfg.mode == 0 else cfg.overlap, cfg.mode, cfg.swin,
                                     cfg.twin, cfg.sbeta, cfg.tbeta, cfg.temporal_mode, cfg.temporal_overlap,
                                     ref.fp(h), ref.fp(w1), err, 256)
        assert np.array_equal(h, big[4][: sizes[4]])
        div = w1[0] if cfg.ftype < 2 else np.float32(1)
        ref.load().ref_dft_profile(ctypes.byref(c), div, ref.fp(exp), err, 256)
        assert np.array_equal(big[1][: sizes[1]], exp)


@pytest.mark.parametrize("cfg,msg", [
    (FFT3DConfig(bw=1), "FFT3D bw/bh must be >=2"),
    (FFT3DConfig(ow=17), "FFT3D ow/oh exceeds half block"),
    (FFT3DConfig(bt=6), "FFT3D bt outside -1..5"),
    (FFT3DConfig(beta=0.5), "FFT3D beta must be >=1"),
    (FFT3DConfig(sigma=-1), "invalid FFT3D sigma"),
    (FFT3DConfig(smin=30), "FFT3D smin exceeds smax"),
    (DFTConfig(ftype=5), "DFTTest ftype outside 0..4"),
    (DFTConfig(mode=0, block=16), "DFTTest center mode requires odd sbsize"),
    (DFTConfig(overlap=11), "DFTTest heavy overlap requires divisible step"),
    (DFTConfig(tbsize=2), "DFTTest centered tbsize must be odd"),
    (DFTConfig(slocation=[0, 1, 0.5]), "DFTTest curve requires frequency/value pairs"),
    (DFTConfig(slocation=[0.1, 1, 1, 2]), "DFTTest curve requires endpoints 0 and 1"),
    (DFTConfig(pmin=5, pmax=1), "DFTTest pmin exceeds pmax"),
    (FFT3DConfig(bw=64, bh=64, ow=16, oh=16, pfactor=1.0), "FFT3D automatic pattern search requires a 5x5 grid"),
    (FFT3DConfig(pfactor=1.0, px=40, py=1), "FFT3D pattern coordinates outside grid"),
    (FFT3DConfig(bw=64, bh=64, ow=16, oh=16, pshow=True, sigma2=3.0),
     "FFT3D automatic pattern search requires a 5x5 grid"),
])
def test_config_errors_match_reference(tb, ref, cfg, msg):
    algo = 0 if isinstance(cfg, FFT3DConfig) else 1
    with pytest.raises(ValueError, match=msg):
        _product_tables(tb, algo, 128, 96, SampleFormat(8), cfg)
    with pytest.raises(ValueError, match=msg):
        ref.RefPlan(128, 96, SampleFormat(8), cfg)


def test_project_transform_forms_identical():
    """fft_core.cuh: the unrolled compile-time transform (kernels) and the runtime
    loop form (host builders, oracle backend) produce identical bits."""
    src = ROOT / "tests" / "native" / "fft_forms_check.cpp"
    lib_path = ROOT / "tests" / "_build" / "libfft_forms.so"
    lib_path.parent.mkdir(exist_ok=True)
    if not lib_path.exists() or src.stat().st_mtime > lib_path.stat().st_mtime or \
            (ROOT / "neo_fft_b200" / "csrc" / "fft_core.cuh").stat().st_mtime > lib_path.stat().st_mtime:
        subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        f"-I{ROOT / 'neo_fft_b200' / 'csrc'}", str(src), "-o", str(lib_path)], check=True)
    lib = ctypes.CDLL(str(lib_path))
    assert lib.fft_forms_mismatches() == 0
    # the team form (a transform shared by four lanes, used by the 48x48 kernels) too
    assert lib.fft_team_mismatches() == 0
    # the real-row forms of the 16-point codelet transform (row_forward/row_inverse<16>):
    # identical bits on generic rows; on rows of zeros, repeats, infinities and NaNs
    # identical values, the sign of an exact zero aside
    assert lib.fft16_real_mismatches(0) == 0
    assert lib.fft16_real_mismatches(1) == 0
    # and of the 32-point one
    assert lib.fft32_real_mismatches(0) == 0
    assert lib.fft32_real_mismatches(1) == 0


def _largest_prime_factor(n):
    p, m, best = 2, n, 1
    while m > 1:
        while m % p == 0:
            m //= p
            best = p
        p += 1
    return best


def test_project_transform_every_length_vs_binary64():
    """The project transform (the stand-in for PocketFFT on every non-codelet length: block
    sides, 48-point team transforms, temporal axes) against a binary64 DFT for every length
    1..128 whose prime factors are at most 64, forward and inverse, on seeded complex data:
    within the reference's FFT test tolerance (3e-5 of the largest output,
    tests/unit/foundation.cpp:65-75). The primes 67..127 exceed the runtime transform's radix
    buffers: the transform refuses them, and so do plans (next test)."""
    import numpy as np
    src = ROOT / "tests" / "native" / "fft_forms_check.cpp"
    lib_path = ROOT / "tests" / "_build" / "libfft_forms.so"
    lib_path.parent.mkdir(exist_ok=True)
    if not lib_path.exists() or src.stat().st_mtime > lib_path.stat().st_mtime or \
            (ROOT / "neo_fft_b200" / "csrc" / "fft_core.cuh").stat().st_mtime > lib_path.stat().st_mtime:
        subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        f"-I{ROOT / 'neo_fft_b200' / 'csrc'}", str(src), "-o", str(lib_path)], check=True)
    lib = ctypes.CDLL(str(lib_path))
    fp = ctypes.POINTER(ctypes.c_float)
    lib.project_fft.argtypes = [ctypes.c_int, ctypes.c_int, fp, fp]
    rng = np.random.default_rng(128)
    worst = 0.0
    for n in range(1, 129):
        for forward in (1, 0):
            x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
            inp = np.ascontiguousarray(np.stack([x.real, x.imag], -1), np.float32)
            out = np.zeros_like(inp)
            rc = lib.project_fft(n, forward, inp.ctypes.data_as(fp), out.ctypes.data_as(fp))
            if _largest_prime_factor(n) > 64:
                assert rc == 1
                continue
            assert rc == 0
            got = out[:, 0].astype(np.float64) + 1j * out[:, 1]
            xd = x.astype(np.complex128)
            exp = np.fft.fft(xd) if forward else np.fft.ifft(xd) * n
            err = np.abs(got - exp).max() / max(1.0, np.abs(exp).max())
            worst = max(worst, err)
            assert err <= 3e-5, (n, forward, err)
    assert worst > 0.0


def test_block_sides_beyond_the_radix_limit_rejected():
    """Block sides with a prime factor above 64 (67..127) are refused at plan creation, before
    any device work, for both algorithms."""
    from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
    msg = "block side has a prime factor above 64"
    for side in (67, 97, 127):
        with pytest.raises(ValueError, match=msg):
            Plan(400, 300, SampleFormat(8), FFT3DConfig(bw=side, bh=16, ow=0, oh=0))
        with pytest.raises(ValueError, match=msg):
            Plan(400, 300, SampleFormat(8), FFT3DConfig(bw=16, bh=side, ow=0, oh=0))
        with pytest.raises(ValueError, match=msg):
            Plan(400, 300, SampleFormat(8), DFTConfig(block=side, overlap=0))


@pytest.mark.parametrize("seed", range(200))
def test_random_configuration_tables_match_reference(tb, ref, seed):
    """Seeded random configurations (both algorithms, every format, odd and non-square
    blocks, overlaps, windows, ftypes, temporal modes, curves, enhancement): the product's
    host plan builder and the reference either reject the draw with the same text, or both
    build it with the same geometry and, for DFTTest, the same 3-D window and primary table
    (FFT3D: the same sigma profile when sigma varies). A GPU limit the reference does not
    have is the only other outcome allowed."""
    from tests.test_fp64_oracle_fuzz import FORMATS, _dft, _fft3d
    rng = np.random.default_rng([800, seed])
    fmt = FORMATS[int(rng.integers(0, len(FORMATS)))]
    cfg = _dft(rng) if rng.random() < 0.55 else _fft3d(rng)
    w, h = int(rng.integers(16, 160)), int(rng.integers(16, 120))
    algo = 0 if isinstance(cfg, FFT3DConfig) else 1
    try:
        rp, ref_msg = ref.RefPlan(w, h, fmt, cfg), None
    except ValueError as e:
        rp, ref_msg = None, str(e)
    try:
        sizes, big, scal = _product_tables(tb, algo, w, h, fmt, cfg)
        msg = None
    except ValueError as e:
        msg = str(e)
    if msg is not None and ref_msg is None:
        assert "GPU" in msg, (cfg, msg)
        return
    assert msg == ref_msg, (cfg, msg, ref_msg)
    if msg is not None:
        return
    assert (sizes[5], sizes[6], sizes[7], sizes[8], sizes[9], sizes[10]) == (
        rp.x["count"], rp.y["count"], rp.x["cover"], rp.y["cover"], rp.x["offset"], rp.y["offset"]), cfg
    err = ctypes.create_string_buffer(256)
    if algo == 1:
        hwin = np.zeros(sizes[4], np.float32)
        w1 = np.zeros(1, np.float32)
        assert ref.load().ref_dft_window_3d(cfg.tbsize, cfg.block, 0 if cfg.mode == 0 else cfg.overlap, cfg.mode,
                                            cfg.swin, cfg.twin, cfg.sbeta, cfg.tbeta, cfg.temporal_mode,
                                            cfg.temporal_overlap, ref.fp(hwin), ref.fp(w1), err, 256) == 0
        assert np.array_equal(hwin, big[4][: sizes[4]]), cfg
        if sizes[1]:
            c, keep = cfg.to_c()
            exp = np.zeros(sizes[1], np.float32)
            div = w1[0] if cfg.ftype < 2 else np.float32(1)
            assert ref.load().ref_dft_profile(ctypes.byref(c), div, ref.fp(exp), err, 256) == 0
            assert np.array_equal(big[1][: sizes[1]], exp), cfg
    elif cfg.sigma2 is not None and sizes[1]:
        # the reference's sample-domain factor (plan.cpp:103): 1/255 for float planes
        factor = np.float32(1.0) / np.float32(255) if fmt.floating else np.float32(1 << (fmt.bits - 8))
        sig = np.array([cfg.sigma, cfg.sigma2, cfg.sigma3, cfg.sigma4], np.float32) * factor
        exp = np.zeros(cfg.bh * (cfg.bw // 2 + 1), np.float32)
        assert ref.load().ref_fft3d_profile(cfg.bw, cfg.bh, ref.fp(sig), ref.fp(exp), err, 256) == 0
        assert np.array_equal(big[1][: sizes[1]], exp), cfg


def test_cpp_temporal_lattice_equals_reference(tb, ref):
    """The C++ temporal lattice the clip batches and the frame server use
    (plan_build.cpp temporal_blocks) equals the reference's temporal_grid.hpp:24-40 for every
    tbsize 1..15, tosize 0..tbsize and frame of clips up to 40 frames, error texts included."""
    cap = 16
    ci, ip = ctypes.c_int, ctypes.POINTER(ctypes.c_int)
    tb.tb_temporal_blocks.argtypes = [ci, ci, ci, ci, ctypes.POINTER(ctypes.c_longlong), ip, ip, ci, ip,
                                      ctypes.c_char_p, ctypes.c_size_t]
    starts = (ctypes.c_longlong * cap)()
    targets = (ctypes.c_int * cap)()
    slots = (ctypes.c_int * (cap * 15))()
    count = ctypes.c_int()
    err = ctypes.create_string_buffer(256)
    checked = 0
    for size in range(1, 16):
        for overlap in range(0, size + 1):
            for length in sorted({size - 1, size, size + 1, 2 * size + 3, 40}):
                for frame in range(-1, length + 1):
                    rc = tb.tb_temporal_blocks(frame, length, size, overlap, starts, targets, slots, cap,
                                               ctypes.byref(count), err, 256)
                    try:
                        want = ref.temporal_blocks(frame, length, size, overlap)
                    except ValueError as e:
                        assert rc == 1 and err.value.decode() == str(e), (frame, length, size, overlap)
                        continue
                    assert rc == 0 and count.value == len(want), (frame, length, size, overlap)
                    got = [{"start": starts[i], "target": targets[i], "slots": list(slots[i * size:(i + 1) * size])}
                           for i in range(count.value)]
                    assert got == want, (frame, length, size, overlap)
                    checked += 1
    assert checked == 7888
