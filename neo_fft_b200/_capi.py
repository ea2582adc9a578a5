"""ctypes binding of the C ABI in include/neo_fft_b200.h.

The shared library is built in-tree (``neo_fft_b200/libneofft_b200.so``) by
``neo_fft_b200.build``. Loading fails loudly when it is missing: there is no CPU
fallback for the pipeline.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libneofft_b200.so"

NF_OK, NF_INVALID_ARGUMENT, NF_NON_FINITE, NF_DEVICE_ERROR = 0, 1, 2, 3

c_int, c_float, c_void_p, c_size_t = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_size_t
c_ptrdiff = ctypes.c_ssize_t


class NfFormat(ctypes.Structure):
    _fields_ = [("bits", c_int), ("floating", c_int), ("chroma", c_int)]


class NfFft3dConfig(ctypes.Structure):
    _fields_ = [(n, c_int) for n in ("bw", "bh", "ow", "oh", "wintype", "opt", "bt")] + \
        [(n, c_float) for n in ("sigma", "beta", "degrid", "kratio")] + \
        [(n, c_int) for n in ("has_sigma2", "has_sigma3", "has_sigma4")] + \
        [(n, c_float) for n in ("sigma2", "sigma3", "sigma4")] + \
        [(n, c_float) for n in ("sharpen", "scutoff", "svr", "smin", "smax", "dehalo", "hr", "ht")] + \
        [(n, c_float) for n in ("pfactor", "pcutoff")] + \
        [(n, c_int) for n in ("pframe", "px", "py", "pshow")] + \
        [(n, c_int) for n in ("left", "top", "right", "bottom", "interlaced")] + \
        [(n, c_int) for n in ("cache_frames", "cache_mb", "kalman_warmup")]


_FP = ctypes.POINTER(c_float)
_IP = ctypes.POINTER(c_int)


class NfDftConfig(ctypes.Structure):
    _fields_ = [(n, c_int) for n in ("block", "overlap", "mode", "swin", "twin", "ftype", "opt", "tbsize")] + \
        [(n, c_float) for n in ("sbeta", "tbeta", "sigma", "sigma2", "pmin", "pmax", "f0beta")] + \
        [(n, c_int) for n in ("zmean", "temporal_mode", "temporal_overlap", "dither", "dither_seed")] + \
        [("slocation", _FP), ("n_slocation", c_int), ("ssx", _FP), ("n_ssx", c_int),
         ("ssy", _FP), ("n_ssy", c_int), ("sst", _FP), ("n_sst", c_int), ("ssystem", c_int),
         ("nlocation", _IP), ("n_nlocation", c_int), ("has_alpha", c_int), ("alpha", c_float)]


class NfAxis(ctypes.Structure):
    _fields_ = [(n, c_int) for n in ("length", "block", "overlap", "step", "count", "cover", "offset")]


class NfConstPlane(ctypes.Structure):
    _fields_ = [("data", c_void_p), ("width", c_int), ("height", c_int), ("stride_bytes", c_ptrdiff)]


class NfPlane(ctypes.Structure):
    _fields_ = [("data", c_void_p), ("width", c_int), ("height", c_int), ("stride_bytes", c_ptrdiff)]


class NfBatchItem(ctypes.Structure):
    _fields_ = [("plan", c_void_p), ("source", NfConstPlane), ("dst", NfPlane)]


class NfRoi(ctypes.Structure):
    _fields_ = [("left", c_int), ("top", c_int), ("width", c_int), ("height", c_int), ("interlaced", c_int)]


class NfClipItem(ctypes.Structure):
    _fields_ = [("plan", c_void_p), ("frames", ctypes.POINTER(NfConstPlane)), ("dsts", ctypes.POINTER(NfPlane)),
                ("nframes", c_int)]


# Every symbol the header declares, with its prototype: (restype, argtypes).
PROTOTYPES = {
    "nf_abi_version": (c_int, []),
    "nf_fft3d_config_default": (None, [ctypes.POINTER(NfFft3dConfig)]),
    "nf_dft_config_default": (None, [ctypes.POINTER(NfDftConfig)]),
    "nf_plan_create_fft3d": (c_int, [c_int, c_int, NfFormat, ctypes.POINTER(NfFft3dConfig),
                                     ctypes.POINTER(c_void_p), ctypes.c_char_p, c_size_t]),
    "nf_plan_create_dft": (c_int, [c_int, c_int, NfFormat, ctypes.POINTER(NfDftConfig),
                                   ctypes.POINTER(c_void_p), ctypes.c_char_p, c_size_t]),
    "nf_plan_destroy": (None, [c_void_p]),
    "nf_plan_geometry": (c_int, [c_void_p, ctypes.POINTER(NfAxis), ctypes.POINTER(NfAxis), _IP, _IP]),
    "nf_plan_process_device": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), c_int, _IP, c_int, NfPlane,
                                       c_int, c_int, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_plan_process_host": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), c_int, _IP, c_int, NfPlane,
                                     c_int, c_int, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_plan_sync_status": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_kalman_state_create": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p), ctypes.c_char_p, c_size_t]),
    "nf_kalman_state_destroy": (None, [c_void_p]),
    "nf_kalman_state_copy": (c_int, [c_void_p, c_void_p, c_void_p]),
    "nf_kalman_state_clone": (c_int, [c_void_p, ctypes.POINTER(c_void_p), c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_kalman_state_bytes": (c_size_t, [c_void_p]),
    "nf_kalman_advance_device": (c_int, [c_void_p, NfConstPlane, c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_kalman_render_device": (c_int, [c_void_p, NfConstPlane, NfPlane, c_void_p, c_void_p,
                                        ctypes.c_char_p, c_size_t]),
    "nf_kalman_step_device": (c_int, [c_void_p, NfConstPlane, NfPlane, c_void_p, c_void_p,
                                        ctypes.c_char_p, c_size_t]),
    "nf_kalman_advance_host": (c_int, [c_void_p, NfConstPlane, c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_kalman_render_host": (c_int, [c_void_p, NfConstPlane, NfPlane, c_void_p, c_void_p, ctypes.c_char_p,
                                      c_size_t]),
    "nf_kalman_state_read": (c_int, [c_void_p, _FP, _FP, _FP, c_size_t]),
    "nf_batch_create": (c_int, [ctypes.POINTER(NfBatchItem), c_int, ctypes.POINTER(c_void_p), ctypes.c_char_p,
                                c_size_t]),
    "nf_batch_create_indexed": (c_int, [ctypes.POINTER(NfBatchItem), _IP, _IP, c_int, ctypes.POINTER(c_void_p),
                                        ctypes.c_char_p, c_size_t]),
    "nf_batch_launch": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_batch_graph_launch": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_batch_destroy": (None, [c_void_p]),
    "nf_batch_geometry_count": (c_int, [c_void_p]),
    "nf_batch_mapped_planes": (c_int, [c_void_p]),
    "nf_batch_geometry": (c_int, [c_void_p]),
    "nf_batch_select_geometry": (c_int, [c_void_p, c_int, ctypes.c_char_p, c_size_t]),
    "nf_plan_process_planes_device": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfPlane), c_int,
                                              c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_clip_batch_create": (c_int, [ctypes.POINTER(NfClipItem), c_int, ctypes.POINTER(c_void_p), ctypes.c_char_p,
                                     c_size_t]),
    "nf_clip_batch_launch": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_clip_batch_graph_launch": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_clip_batch_destroy": (None, [c_void_p]),
    "nf_host_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_int, ctypes.POINTER(c_void_p),
                                     ctypes.c_char_p, c_size_t]),
    "nf_host_batch_process": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfPlane), c_int,
                                      c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_host_batch_device_bytes": (c_size_t, [c_void_p]),
    "nf_host_batch_destroy": (None, [c_void_p]),
    "nf_frame_server_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_int, c_void_p, c_void_p,
                                       ctypes.POINTER(c_void_p), ctypes.c_char_p, c_size_t]),
    "nf_frame_server_request": (c_int, [c_void_p, c_int, ctypes.POINTER(c_int), c_int, ctypes.POINTER(c_int),
                                        ctypes.c_char_p, c_size_t]),
    "nf_frame_server_get": (c_int, [c_void_p, c_int, ctypes.POINTER(NfPlane), ctypes.c_char_p, c_size_t]),
    "nf_frame_server_counters": (None, [c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_longlong)]),
    "nf_frame_server_destroy": (None, [c_void_p]),
    "nf_dft_noise_power": (c_int, [ctypes.POINTER(NfDftConfig), c_void_p, c_int, c_void_p, c_int, ctypes.c_char_p,
                                   c_size_t]),
    "nf_plan_set_noise_model": (c_int, [c_void_p, c_void_p, c_int, ctypes.c_char_p, c_size_t]),
    "nf_plan_model_state": (c_int, [c_void_p]),
    "nf_plan_pattern_candidate": (c_int, [c_void_p, NfConstPlane, c_void_p, c_int, c_void_p, ctypes.c_char_p,
                                          c_size_t]),
    "nf_plan_prepare_pattern": (c_int, [c_void_p, NfConstPlane, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_plan_pattern_candidate_host": (c_int, [c_void_p, NfConstPlane, c_void_p, c_int, c_void_p, ctypes.c_char_p,
                                               c_size_t]),
    "nf_plan_prepare_pattern_host": (c_int, [c_void_p, NfConstPlane, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_roi_make": (c_int, [c_int] * 9 + [ctypes.POINTER(NfRoi), ctypes.c_char_p, c_size_t]),
    "nf_roi_pack_device": (c_int, [ctypes.POINTER(NfRoi), NfConstPlane, NfPlane, c_int, c_void_p, ctypes.c_char_p,
                                   c_size_t]),
    "nf_roi_unpack_device": (c_int, [ctypes.POINTER(NfRoi), NfConstPlane, NfPlane, c_int, c_void_p, ctypes.c_char_p,
                                     c_size_t]),
    "nf_plan_set_primary": (c_int, [c_void_p, c_void_p, c_int, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_plan_get_primary": (c_int, [c_void_p, c_void_p, c_int, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_dft_backward_scratch_bytes": (c_int, [c_void_p, c_int, ctypes.POINTER(c_size_t)]),
    "nf_dft_backward_device": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfConstPlane),
                                       ctypes.POINTER(NfPlane), c_int, c_void_p, c_void_p, c_size_t, c_void_p,
                                       ctypes.c_char_p, c_size_t]),
    "nf_fft3d_backward_device": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfConstPlane),
                                         ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfPlane), c_int, c_void_p,
                                         c_void_p, c_size_t, c_void_p, ctypes.c_char_p, c_size_t]),
    "nf_dft_backward_static_capacity": (c_size_t, []),
    "nf_dft_backward_device_static": (c_int, [c_void_p, ctypes.POINTER(NfConstPlane), ctypes.POINTER(NfConstPlane),
                                              ctypes.POINTER(NfPlane), c_int, c_void_p, c_void_p, ctypes.c_char_p,
                                              c_size_t]),
    "nf_kernel_info": (c_int, [ctypes.c_char_p, c_size_t, ctypes.c_char_p, c_size_t, ctypes.c_char_p,
                               c_size_t, _IP]),
    "nf_copy_row": (None, [c_void_p, c_void_p, c_size_t]),
    "nf_stream_create": (c_int, [ctypes.POINTER(c_void_p), ctypes.c_char_p, c_size_t]),
    "nf_stream_destroy": (None, [c_void_p]),
}

_lib = None


def load(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"neo_fft_b200 CUDA library not built: {p} is missing "
                           "(run `python -m neo_fft_b200.build`); there is no CPU fallback")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class NonFiniteError(RuntimeError):
    """std::runtime_error("non-finite sample or intermediate") of the reference."""


class DeviceError(RuntimeError):
    """CUDA launch/allocation failure."""


def raise_for(status: int, message: bytes | str) -> None:
    """Map a status to the reference's exception types (checked.hpp:13-41)."""
    if status == NF_OK:
        return
    msg = message.decode(errors="replace") if isinstance(message, bytes) else message
    if status == NF_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == NF_NON_FINITE:
        raise NonFiniteError(msg)
    raise DeviceError(msg)
