"""Test infrastructure (oracle only): ctypes wrapper over the neo-fft reference core
compiled from its own sources into oracle/_ref/libneofft_ref.so (see oracle/Makefile).

Used by tests/ and by bench.py's CPU-baseline leg only; the product never imports it.
The configuration objects are the product's public dataclasses so both sides get
identical parameters.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libneofft_ref.so"
# The neo-fft sources: $NEO_FFT_REFERENCE, else a checkout named `reference` beside this repository.
REFERENCE = Path(os.environ.get("NEO_FFT_REFERENCE", HERE.parent.parent / "reference"))

_lib = None


def build(quiet: bool = True) -> bool:
    """Build the reference oracle if the reference sources are present."""
    if LIB.exists():
        return True
    if not (REFERENCE / "src" / "algorithms" / "plan.cpp").exists():
        return False
    out = subprocess.run(["make", "-C", str(HERE), "-j8", f"REF={REFERENCE}"], capture_output=quiet)
    return out.returncode == 0 and LIB.exists()


def available() -> bool:
    return LIB.exists() or build()


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference oracle not built (oracle/_ref/libneofft_ref.so)")
        from neo_fft_b200 import _capi as C
        lib = ctypes.CDLL(str(LIB))
        vp, ci, cs = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
        cp = ctypes.c_char_p
        FP = ctypes.POINTER(ctypes.c_float)
        sig = {
            "ref_plan_create_fft3d": (ci, [ci, ci, C.NfFormat, ctypes.POINTER(C.NfFft3dConfig), ctypes.POINTER(vp), cp, cs]),
            "ref_plan_create_dft": (ci, [ci, ci, C.NfFormat, ctypes.POINTER(C.NfDftConfig), ctypes.POINTER(vp), cp, cs]),
            "ref_plan_destroy": (None, [vp]),
            "ref_plan_geometry": (ci, [vp, ctypes.POINTER(C.NfAxis), ctypes.POINTER(C.NfAxis),
                                       ctypes.POINTER(ci), ctypes.POINTER(ci)]),
            "ref_plan_process": (ci, [vp, ci, ctypes.POINTER(C.NfConstPlane), ci, ctypes.POINTER(ci), ci, C.NfPlane,
                                      ci, ci, cp, cs]),
            "ref_plan_process_many": (ci, [vp, ci, ctypes.POINTER(C.NfConstPlane), ci, ctypes.POINTER(C.NfPlane), ci, ci,
                                           cp, cs]),
            "ref_kalman_create": (ci, [vp, ctypes.POINTER(vp), cp, cs]),
            "ref_kalman_destroy": (None, [vp]),
            "ref_kalman_bins": (cs, [vp]),
            "ref_kalman_read": (ci, [vp, FP, FP, FP]),
            "ref_kalman_advance": (ci, [vp, ci, C.NfConstPlane, vp, cp, cs]),
            "ref_kalman_render": (ci, [vp, ci, C.NfConstPlane, C.NfPlane, vp, cp, cs]),
            "ref_fft_r2c": (ci, [ci, ci, FP, FP]),
            "ref_fft_c2r": (ci, [ci, ci, FP, FP]),
            "ref_fft_r2c_3d": (ci, [ci, ci, ci, FP, FP]),
            "ref_fft_c2r_3d": (ci, [ci, ci, ci, FP, FP]),
            "ref_replica_r2c": (ci, [ci, ci, FP, FP]),
            "ref_replica_c2r": (ci, [ci, ci, FP, FP]),
            "ref_fft3d_window": (ci, [ci, ci, ci, FP, FP, cp, cs]),
            "ref_dft_window_3d": (ci, [ci, ci, ci, ci, ci, ci, ctypes.c_float, ctypes.c_float, ci, ci, FP, FP, cp, cs]),
            "ref_dft_profile": (ci, [ctypes.POINTER(C.NfDftConfig), ctypes.c_float, FP, cp, cs]),
            "ref_fft3d_profile": (ci, [ci, ci, FP, FP, cp, cs]),
            "ref_plan_prepare_noise": (ci, [vp, FP, ci, FP, ci, cp, cs]),
            "ref_plan_pattern_candidate": (ci, [vp, ci, C.NfConstPlane, FP, ci, cp, cs]),
            "ref_plan_publish_pattern": (ci, [vp, FP, ci, cp, cs]),
            "ref_dither": (ci, [FP, ci, ci, ci, ctypes.POINTER(ctypes.c_ubyte), ci, ci, ci, ci, ci, cp, cs]),
            "ref_dither_hash": (ctypes.c_uint, [ctypes.c_uint] * 5),
            "ref_temporal_blocks": (ci, [ci, ci, ci, ci, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ci),
                                         ctypes.POINTER(ci), ci, ctypes.POINTER(ci), cp, cs]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _lib = lib
    return _lib


def _raise(rc: int, err) -> None:
    if rc == 0:
        return
    msg = err.value.decode(errors="replace")
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        from neo_fft_b200._capi import NonFiniteError
        raise NonFiniteError(msg)
    raise RuntimeError(msg)


def _storage(a: np.ndarray) -> int:
    return {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 4}[a.dtype]


class RefPlan:
    """The reference `neo_fft::Plan`, compiled from its own sources."""

    def __init__(self, width, height, fmt, config):
        from neo_fft_b200 import _capi as C
        from neo_fft_b200.plan import DFTConfig
        self.lib = load()
        err = ctypes.create_string_buffer(512)
        h = ctypes.c_void_p()
        f = C.NfFormat(fmt.bits, int(fmt.floating), int(fmt.chroma))
        if isinstance(config, DFTConfig):
            cfg, self._keep = config.to_c()
            rc = self.lib.ref_plan_create_dft(width, height, f, ctypes.byref(cfg), ctypes.byref(h), err, 512)
        else:
            cfg = config.to_c()
            rc = self.lib.ref_plan_create_fft3d(width, height, f, ctypes.byref(cfg), ctypes.byref(h), err, 512)
        _raise(rc, err)
        self.h = h
        x, y = C.NfAxis(), C.NfAxis()
        t, b = ctypes.c_int(), ctypes.c_int()
        self.lib.ref_plan_geometry(h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(t), ctypes.byref(b))
        self.x = {n: getattr(x, n) for n, _ in C.NfAxis._fields_}
        self.y = {n: getattr(y, n) for n, _ in C.NfAxis._fields_}
        self.temporal_size, self.bins = t.value, b.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_plan_destroy(self.h)
            self.h = None

    def process(self, sources, dst=None, targets=(), frame=0, plane=0):
        from neo_fft_b200 import _capi as C
        if not isinstance(sources, (list, tuple)):
            sources = [sources]
        sources = [np.asarray(s) for s in sources]
        if dst is None:
            dst = np.zeros_like(sources[0])
        arr = (C.NfConstPlane * len(sources))(*[C.NfConstPlane(s.ctypes.data, s.shape[1], s.shape[0], s.strides[0])
                                                for s in sources])
        d = C.NfPlane(dst.ctypes.data, dst.shape[1], dst.shape[0], dst.strides[0])
        tg = np.asarray(list(targets), np.int32)
        tgp = tg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if tg.size else None
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_plan_process(self.h, _storage(sources[0]), arr, len(sources), tgp, int(tg.size), d,
                                       frame, plane, err, 512)
        _raise(rc, err)
        return dst

    def process_many(self, frames, threads: int):
        """frames: list of source lists (equal slot counts); returns outputs.
        Frames run concurrently on `threads` host threads (one shared plan)."""
        from neo_fft_b200 import _capi as C
        nslots = len(frames[0])
        srcs = [np.asarray(s) for f in frames for s in f]
        outs = [np.zeros_like(f[len(f) // 2]) for f in frames]
        arr = (C.NfConstPlane * len(srcs))(*[C.NfConstPlane(s.ctypes.data, s.shape[1], s.shape[0], s.strides[0])
                                             for s in srcs])
        darr = (C.NfPlane * len(outs))(*[C.NfPlane(o.ctypes.data, o.shape[1], o.shape[0], o.strides[0]) for o in outs])
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_plan_process_many(self.h, _storage(srcs[0]), arr, nslots, darr, len(outs), threads, err, 512)
        _raise(rc, err)
        return outs

    def prepare_noise(self, slices: np.ndarray) -> np.ndarray:
        """DFTNoise::prepare of this plan's sampled model from gathered slices
        [location][tbsize][sbsize][sbsize]; returns the published power table."""
        slices = np.ascontiguousarray(slices, np.float32)
        out = np.zeros(self.temporal_size * self.bins, np.float32)
        err = ctypes.create_string_buffer(512)
        _raise(self.lib.ref_plan_prepare_noise(self.h, fp(slices), int(slices.shape[0]), fp(out), out.size, err, 512),
               err)
        return out

    def pattern_candidate(self, src) -> np.ndarray:
        from neo_fft_b200 import _capi as C
        src = np.asarray(src)
        out = np.zeros(self.bins, np.float32)
        err = ctypes.create_string_buffer(512)
        _raise(self.lib.ref_plan_pattern_candidate(self.h, _storage(src), C.NfConstPlane(src.ctypes.data, src.shape[1],
               src.shape[0], src.strides[0]), fp(out), out.size, err, 512), err)
        return out

    def publish_pattern(self, power) -> None:
        p = np.ascontiguousarray(power, np.float32)
        err = ctypes.create_string_buffer(512)
        _raise(self.lib.ref_plan_publish_pattern(self.h, fp(p), p.size, err, 512), err)

    # Kalman
    def kalman_state(self):
        return RefKalman(self)

    def advance_kalman(self, src, state):
        from neo_fft_b200 import _capi as C
        src = np.asarray(src)
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_kalman_advance(self.h, _storage(src), C.NfConstPlane(src.ctypes.data, src.shape[1],
                                         src.shape[0], src.strides[0]), state.h, err, 512)
        _raise(rc, err)

    def render_kalman(self, src, state, dst=None):
        from neo_fft_b200 import _capi as C
        src = np.asarray(src)
        dst = np.zeros_like(src) if dst is None else dst
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ref_kalman_render(self.h, _storage(src),
                                        C.NfConstPlane(src.ctypes.data, src.shape[1], src.shape[0], src.strides[0]),
                                        C.NfPlane(dst.ctypes.data, dst.shape[1], dst.shape[0], dst.strides[0]),
                                        state.h, err, 512)
        _raise(rc, err)
        return dst


class RefKalman:
    def __init__(self, plan: RefPlan):
        self.lib = plan.lib
        self.h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        _raise(self.lib.ref_kalman_create(plan.h, ctypes.byref(self.h), err, 512), err)

    def read(self):
        n = self.lib.ref_kalman_bins(self.h)
        last = np.zeros((n, 2), np.float32)
        cov = np.zeros(n, np.float32)
        proc = np.zeros(n, np.float32)
        FP = ctypes.POINTER(ctypes.c_float)
        self.lib.ref_kalman_read(self.h, last.ctypes.data_as(FP), cov.ctypes.data_as(FP), proc.ctypes.data_as(FP))
        return last, cov, proc

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_kalman_destroy(self.h)
            self.h = None


def temporal_blocks(frame: int, length: int, size: int, overlap: int) -> list[dict]:
    """The reference's covering temporal blocks of an output frame
    (src/algorithms/temporal_grid.hpp:24-40): start, target slice and clamped slots."""
    cap = 16
    starts = (ctypes.c_longlong * cap)()
    targets = (ctypes.c_int * cap)()
    slots = (ctypes.c_int * (cap * 15))()
    count = ctypes.c_int()
    err = ctypes.create_string_buffer(256)
    _raise(load().ref_temporal_blocks(frame, length, size, overlap, starts, targets, slots, cap, ctypes.byref(count),
                                      err, 256), err)
    assert count.value <= cap
    return [{"start": starts[i], "target": targets[i], "slots": list(slots[i * size:(i + 1) * size])}
            for i in range(count.value)]


def fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def r2c(x: np.ndarray) -> np.ndarray:
    h, w = x.shape
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros((h, w // 2 + 1, 2), np.float32)
    load().ref_fft_r2c(h, w, fp(x), fp(out))
    return out[..., 0] + 1j * out[..., 1]
