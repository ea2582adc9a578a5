"""The C-ABI library loads and exports every symbol include/neo_fft_b200.h declares;
host-side argument validation works without a GPU (errors raised before any device
call carry the reference's texts)."""
import ctypes
import re
from pathlib import Path

import pytest

from neo_fft_b200 import _capi as C

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "neo_fft_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nf_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    syms = declared_symbols()
    for s in ("nf_plan_create_fft3d", "nf_plan_create_dft", "nf_plan_process_device", "nf_plan_process_host",
              "nf_kalman_advance_device", "nf_kalman_render_device", "nf_plan_geometry", "nf_kernel_info"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = C.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(C.PROTOTYPES), "ctypes prototypes out of date"
    assert lib.nf_abi_version() == 1


def test_defaults_match_reference_structs():
    lib = C.load()
    c = C.NfFft3dConfig()
    lib.nf_fft3d_config_default(ctypes.byref(c))
    assert (c.bw, c.bh, c.ow, c.oh, c.bt, c.sigma, c.beta, c.degrid, c.kratio) == (32, 32, -1, -1, 1, 2.0, 1.0, 1.0, 2.0)
    d = C.NfDftConfig()
    lib.nf_dft_config_default(ctypes.byref(d))
    assert (d.block, d.overlap, d.mode, d.swin, d.twin, d.ftype, d.tbsize, d.zmean) == (16, 12, 1, 0, 7, 0, 1, 1)


def test_header_is_plain_c():
    """The C ABI compiles as C99 with warnings as errors and links against the library (the
    calls a C, cgo or FFI host makes); the entry points that need no GPU give the defaults."""
    import subprocess
    exe = ROOT / "tests" / "_build" / "c_abi_check"
    exe.parent.mkdir(exist_ok=True)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "native" / "c_abi_check.c"), "-o", str(exe), f"-L{ROOT / 'neo_fft_b200'}",
                    "-lneofft_b200", f"-Wl,-rpath,{ROOT / 'neo_fft_b200'}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["1", "32", "1", "16", "12", str(16 << 20)]


def test_invalid_config_rejected_on_host():
    from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
    with pytest.raises(ValueError, match="FFT3D bt outside -1..5"):
        Plan(64, 64, SampleFormat(8), FFT3DConfig(bt=9))
    with pytest.raises(ValueError, match="DFTTest ftype outside 0..4"):
        Plan(64, 64, SampleFormat(8), DFTConfig(ftype=7))
    with pytest.raises(ValueError, match="unsupported sample format"):
        Plan(64, 64, SampleFormat(9), DFTConfig())


def test_batch_item_shapes_checked_on_host():
    """A batch item carries both frame and plane numbers or neither; a 4-tuple is an error,
    not an item whose frame is silently dropped."""
    from neo_fft_b200.plan import Batch
    with pytest.raises(ValueError, match="batch items are"):
        Batch([(None, None, None, 3)])


def _build_facade_check():
    import subprocess
    exe = ROOT / "tests" / "_build" / "facade_check"
    exe.parent.mkdir(exist_ok=True)
    src = ROOT / "tests" / "native" / "facade_check.cpp"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Wpedantic", "-Werror", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'oracle' / 'shim'}", str(src),
                    "-o", str(exe), f"-L{ROOT / 'neo_fft_b200'}", "-lneofft_b200",
                    f"-Wl,-rpath,{ROOT / 'neo_fft_b200'}"], check=True)
    return exe


def build_roi_facade_check(reference):
    """The reference host layer's src/plugin/roi.hpp, unchanged, compiled against the facade
    (tests/native/roi_facade_check.cpp); the binary is kept in tests/_build for the GPU test."""
    import subprocess
    # kept beside its source (git-ignored, but shipped with the tree to GPU hosts, which
    # have no reference sources to build it from)
    exe = ROOT / "tests" / "native" / "_bin" / "roi_facade_check"
    exe.parent.mkdir(exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'tests' / 'native' / 'shim'}", f"-I{reference / 'src'}",
                    f"-I{ROOT / 'include'}", f"-I{ROOT / 'oracle' / 'shim'}",
                    str(ROOT / "tests" / "native" / "roi_facade_check.cpp"), "-o", str(exe),
                    f"-L{ROOT / 'neo_fft_b200'}", "-lneofft_b200", "-Wl,-rpath,$ORIGIN/../../../neo_fft_b200"],
                   check=True)
    return exe


def test_reference_roi_code_compiles_against_facade():
    """filter.hpp's ROI calls (PackedROI with plan->copy_row(), process_at over packed views,
    render_kalman and prepare_pattern through PackedROI) compile unchanged against the facade."""
    from oracle import ref as R
    if not (R.REFERENCE / "src" / "plugin" / "roi.hpp").exists():
        pytest.skip("reference sources absent")
    assert build_roi_facade_check(R.REFERENCE).exists()


def test_cpp_facade_compiles_and_links():
    """include/neo_fft_b200/plan.hpp (the reference Plan's class signature over the
    C ABI) compiles without warnings (-Wall -Wextra -Wpedantic) against a span2d provider
    and links to the library."""
    assert _build_facade_check().exists()


@pytest.mark.gpu
def test_cpp_facade_matches_python_path(cuda):
    import subprocess
    import numpy as np
    from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
    out = subprocess.run([str(_build_facade_check())], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.split(" ", 1) for line in out if line)
    w, h = 96, 64
    y, x = np.mgrid[0:h, 0:w]
    src = ((x * 37 + y * 101 + (x * y) % 17) * 29 % 60000).astype(np.uint16)
    dst = Plan(w, h, SampleFormat(16), DFTConfig(block=16, overlap=12, sigma=8, slocation=[0, 8, 1, 8])).process(src)

    def fnv(b):
        v = 1469598103934665603
        for c in b:
            v = ((v ^ c) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return v
    assert int(got["dft"]) == fnv(dst.tobytes())
    assert int(got["dft_ws"]) == int(got["dft_ws_span"]) == int(got["dft"])
    assert got["pool_capacity"] == "1" and got["pool_active"] == "2"
    assert got["pool_idle"].split()[0] == "1" and int(got["pool_idle"].split()[2]) == 2 * w * h * 2
    assert got["copy_row"] == "1"
    assert got["error"] == "FFT3D bt outside -1..5"
    fsrc = ((np.arange(w * h) * 7919) % 1000 / 1000.0).astype(np.float32).reshape(h, w)
    kp = Plan(w, h, SampleFormat(32, True), FFT3DConfig(bw=16, bh=16, bt=0, sigma=2.5, kratio=2.0))
    st = kp.initial_kalman()
    d = cuda.from_numpy(fsrc).cuda()
    for _ in range(3):
        kp.advance_kalman(d, st)
    out_t = cuda.empty_like(d)
    kp.render_kalman(d, out_t, st)
    assert int(got["kalman"]) == fnv(out_t.cpu().numpy().tobytes())
    # sampled FFT3D pattern through the facade equals the Python path
    assert got["pattern_needed"] == "1"
    idx = np.arange(w * h, dtype=np.int64)
    pa = ((idx * 131 + (idx // w) * 7) % 200 + 20).astype(np.uint8).reshape(h, w)
    pb = ((idx * 97 + (idx // w) * 13) % 180 + 30).astype(np.uint8).reshape(h, w)
    pp = Plan(w, h, SampleFormat(8), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, pfactor=1.0))
    pp.prepare_pattern(cuda.from_numpy(pa).cuda())
    assert int(got["pattern"]) == fnv(pp.process(pb).tobytes())
    # the C++ checkpoint/seek policy equals the Python mirror
    from neo_fft_b200.checkpoints import KalmanSeek
    frames = [cuda.from_numpy(((np.arange(w * h, dtype=np.int64) * 7919 + f * 104729) % 1000 / 1000.0)
                              .astype(np.float32).reshape(h, w)).cuda() for f in range(24)]
    seek = KalmanSeek([kp], warmup=4)
    for n in (5, 6, 7, 20, 3, 21):
        o = cuda.empty_like(frames[0])
        seek.frame(n, lambda f, p: frames[f], [o])
        assert int(got[f"seek{n}"]) == fnv(o.cpu().numpy().tobytes()), n


def test_missing_library_fails_loudly(tmp_path):
    """The product path has no CPU fallback: without the CUDA library, loading it raises."""
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        C.load(tmp_path / "libneofft_b200.so")


def test_product_modules_do_not_import_the_oracle():
    """Nothing under neo_fft_b200/ imports, links or runs oracle/ (the oracle is test
    infrastructure); the package's sources name it nowhere."""
    pkg = ROOT / "neo_fft_b200"
    offenders = [p for p in list(pkg.glob("*.py")) + list((pkg / "csrc").glob("*"))
                 if p.is_file() and re.search(r"\boracle\b", p.read_text(errors="replace"))]
    assert not offenders, offenders
