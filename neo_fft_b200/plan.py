"""Python mirror of neo-fft's core `Plan` (src/algorithms/plan.hpp:18-140) over the C ABI.

Same names and argument meaning as the reference: ``SampleFormat``, ``FFT3DConfig``,
``DFTConfig`` and ``Plan(width, height, format, config)`` with ``process``,
``process_at``, ``initial_kalman``, ``advance_kalman`` and ``render_kalman``.
Errors follow the reference's exception types: configuration/geometry errors raise
``ValueError`` (std::invalid_argument) and non-finite samples raise
``NonFiniteError`` (a RuntimeError, like std::runtime_error).

Planes are 2-D arrays: numpy arrays run through the host-memory entry point (copies
in and out on the plan's stream), CUDA torch tensors through the device entry
point (asynchronous on the current torch stream).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi as C


@dataclass
class SampleFormat:
    bits: int = 8
    floating: bool = False
    chroma: bool = False


@dataclass
class FFT3DConfig:
    """FFT3DConfig with EnhancementConfig fields (plan.hpp:24-36, fft3d_profile.hpp:6-9)."""
    bw: int = 32
    bh: int = 32
    ow: int = -1
    oh: int = -1
    wintype: int = 0
    opt: int = 0
    bt: int = 1
    sigma: float = 2.0
    beta: float = 1.0
    degrid: float = 1.0
    kratio: float = 2.0
    sigma2: Optional[float] = None
    sigma3: Optional[float] = None
    sigma4: Optional[float] = None
    sharpen: float = 0.0
    scutoff: float = 0.3
    svr: float = 1.0
    smin: float = 4.0
    smax: float = 20.0
    dehalo: float = 0.0
    hr: float = 2.0
    ht: float = 50.0
    pfactor: float = 0.0
    pcutoff: float = 0.1
    pframe: int = 0
    px: int = 0
    py: int = 0
    pshow: bool = False
    left: int = 0
    top: int = 0
    right: int = 0
    bottom: int = 0
    interlaced: bool = False
    cache_frames: int = -1
    cache_mb: int = 128
    kalman_warmup: int = 8

    def to_c(self) -> C.NfFft3dConfig:
        c = C.NfFft3dConfig()
        for name, _ in C.NfFft3dConfig._fields_:
            if name.startswith("has_"):
                continue
            if name in ("sigma2", "sigma3", "sigma4"):
                v = getattr(self, name)
                setattr(c, "has_" + name, 0 if v is None else 1)
                setattr(c, name, 0.0 if v is None else float(v))
            else:
                setattr(c, name, type(getattr(c, name))(getattr(self, name)))
        return c


@dataclass
class DFTConfig:
    """DFTConfig with DFTCurves (plan.hpp:37-46, profile.hpp:7-12)."""
    block: int = 16
    overlap: int = 12
    mode: int = 1
    swin: int = 0
    twin: int = 7
    ftype: int = 0
    opt: int = 0
    tbsize: int = 1
    sbeta: float = 2.5
    tbeta: float = 2.5
    sigma: float = 8.0
    sigma2: float = 8.0
    pmin: float = 0.0
    pmax: float = 500.0
    f0beta: float = 1.0
    zmean: bool = True
    temporal_mode: int = 0
    temporal_overlap: int = 0
    dither: int = 0
    dither_seed: int = 0
    slocation: Sequence[float] = field(default_factory=list)
    ssx: Sequence[float] = field(default_factory=list)
    ssy: Sequence[float] = field(default_factory=list)
    sst: Sequence[float] = field(default_factory=list)
    ssystem: int = 0
    nlocation: Sequence[int] = field(default_factory=list)
    alpha: Optional[float] = None

    def to_c(self):
        c = C.NfDftConfig()
        keep = []
        for name, typ in C.NfDftConfig._fields_:
            if name.startswith("n_") or name in ("slocation", "ssx", "ssy", "sst", "nlocation", "has_alpha", "alpha"):
                continue
            setattr(c, name, typ(getattr(self, name)).value)
        for name in ("slocation", "ssx", "ssy", "sst"):
            v = np.ascontiguousarray(np.asarray(getattr(self, name), dtype=np.float32))
            keep.append(v)
            setattr(c, name, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if v.size else None)
            setattr(c, "n_" + name, int(v.size))
        loc = np.ascontiguousarray(np.asarray(self.nlocation, dtype=np.int32).reshape(-1))
        keep.append(loc)
        c.nlocation = loc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if loc.size else None
        c.n_nlocation = int(loc.size // 4)
        c.has_alpha = 0 if self.alpha is None else 1
        c.alpha = 0.0 if self.alpha is None else float(self.alpha)
        return c, keep


@dataclass
class Axis:
    length: int
    block: int
    overlap: int
    step: int
    count: int
    cover: int
    offset: int


@dataclass
class Geometry:
    x: Axis
    y: Axis


_DTYPES = {1: np.uint8, 2: np.uint16, 4: np.float32}


def _storage(fmt: SampleFormat) -> int:
    return 4 if fmt.floating else (1 if fmt.bits == 8 else 2)


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _plane(a, const: bool):
    """2-D array -> nf plane (data pointer, width, height, signed byte stride)."""
    cls = C.NfConstPlane if const else C.NfPlane
    if _is_torch(a):
        if a.dim() != 2 or a.stride(1) != 1:
            raise ValueError("planes must be 2-D with contiguous rows")
        return cls(a.data_ptr(), a.shape[1], a.shape[0], a.stride(0) * a.element_size())
    a = np.asarray(a)
    if a.ndim != 2 or a.strides[1] != a.itemsize:
        raise ValueError("planes must be 2-D with contiguous rows")
    return cls(a.ctypes.data, a.shape[1], a.shape[0], a.strides[0])


class Plan:
    """B200 per-plane compiled filter; drop-in for neo_fft::Plan."""

    def __init__(self, width: int, height: int, format: SampleFormat, config):
        self._lib = C.load()
        self.format = format
        self.config = config
        err = ctypes.create_string_buffer(512)
        handle = ctypes.c_void_p()
        fmt = C.NfFormat(format.bits, int(format.floating), int(format.chroma))
        if isinstance(config, FFT3DConfig):
            cfg = config.to_c()
            st = self._lib.nf_plan_create_fft3d(width, height, fmt, ctypes.byref(cfg), ctypes.byref(handle), err, 512)
            self.algorithm = "FFT3D"
        elif isinstance(config, DFTConfig):
            cfg, keep = config.to_c()
            st = self._lib.nf_plan_create_dft(width, height, fmt, ctypes.byref(cfg), ctypes.byref(handle), err, 512)
            self.algorithm = "DFTTest"
        else:
            raise TypeError("config must be FFT3DConfig or DFTConfig")
        C.raise_for(st, err.value)
        self._h = handle
        x, y = C.NfAxis(), C.NfAxis()
        t, b = ctypes.c_int(), ctypes.c_int()
        self._lib.nf_plan_geometry(self._h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(t), ctypes.byref(b))
        self.geometry = Geometry(Axis(*[getattr(x, n) for n, _ in C.NfAxis._fields_]),
                                 Axis(*[getattr(y, n) for n, _ in C.NfAxis._fields_]))
        self.temporal_size = t.value
        self.bins = b.value
        self.dtype = _DTYPES[_storage(format)]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_plan_destroy(h)
            self._h = None

    # -- frame processing -------------------------------------------------------
    def process_at(self, sources, dst, frame: int = 0, plane: int = 0, targets: Sequence[int] = (),
                   stream=None):
        """Plan::process_at (plan.hpp:77-80): filter `sources` (temporal slots) into `dst`."""
        if not isinstance(sources, (list, tuple)):
            sources = [sources]
        if not sources:
            raise ValueError("sources must not be empty")
        device = _is_torch(sources[0])
        srcs = (C.NfConstPlane * len(sources))(*[_plane(s, True) for s in sources])
        d = _plane(dst, False)
        tg = np.ascontiguousarray(np.asarray(list(targets), dtype=np.int32))
        tgp = tg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if tg.size else None
        err = ctypes.create_string_buffer(512)
        if device:
            import torch
            s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
            st = self._lib.nf_plan_process_device(self._h, srcs, len(sources), tgp, int(tg.size), d, frame, plane,
                                                  ctypes.c_void_p(s), err, 512)
        else:
            st = self._lib.nf_plan_process_host(self._h, srcs, len(sources), tgp, int(tg.size), d, frame, plane,
                                                ctypes.c_void_p(stream or 0), err, 512)
        C.raise_for(st, err.value)
        return dst

    def process_planes(self, sources, dsts, stream=None):
        """Several single-frame planes (device tensors) in one launch per 32 planes;
        equal to process_at per plane."""
        import torch
        if len(sources) != len(dsts):
            raise ValueError("sources and dsts differ in length")
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        for start in range(0, len(sources), 32):
            chunk = range(start, min(start + 32, len(sources)))
            srcs = (C.NfConstPlane * len(chunk))(*[_plane(sources[i], True) for i in chunk])
            ds = (C.NfPlane * len(chunk))(*[_plane(dsts[i], False) for i in chunk])
            C.raise_for(self._lib.nf_plan_process_planes_device(self._h, srcs, ds, len(chunk), ctypes.c_void_p(s),
                                                                err, 512), err.value)
        return dsts

    def process(self, sources, dst=None):
        """Plan::process (plan.hpp:58-75); allocates dst like the first source when omitted."""
        if dst is None:
            first = sources[0] if isinstance(sources, (list, tuple)) else sources
            if _is_torch(first):
                import torch
                dst = torch.empty_like(first)
            else:
                dst = np.empty_like(np.asarray(first))
        return self.process_at(sources, dst)

    @property
    def model_state(self) -> int:
        """0: no sampled noise model; 1: waiting for one; 2: ready."""
        return int(self._lib.nf_plan_model_state(self._h))

    @property
    def needs_pattern_frame(self) -> bool:
        """FFT3D pfactor > 0 with denoising (plan.hpp:90)."""
        return self.model_state != 0 and isinstance(self.config, FFT3DConfig)

    @property
    def pattern_ready(self) -> bool:
        return self.model_state == 2

    def pattern_candidate(self, source, stream=None) -> np.ndarray:
        """plan.cpp:271-277 on a device plane: the chosen block's scaled power (bins floats)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        out = np.zeros(self.bins, np.float32)
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_plan_pattern_candidate(self._h, _plane(source, True), ctypes.c_void_p(out.ctypes.data),
                                                        out.size, ctypes.c_void_p(s), err, 512), err.value)
        return out

    def prepare_pattern(self, source, stream=None) -> None:
        """prepare_pattern (plan.hpp:95-97): search and publish unless a model is published."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_plan_prepare_pattern(self._h, _plane(source, True), ctypes.c_void_p(s), err, 512),
                    err.value)

    def publish_pattern(self, power) -> None:
        self.set_noise_model(power)

    def set_noise_model(self, power) -> None:
        p = np.ascontiguousarray(power, np.float32)
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_plan_set_noise_model(self._h, ctypes.c_void_p(p.ctypes.data), p.size, err, 512),
                    err.value)

    def sync_status(self, stream=None) -> None:
        """Raise NonFiniteError if any device launch met a non-finite value."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_plan_sync_status(self._h, ctypes.c_void_p(s), err, 512), err.value)

    # -- Kalman (bt=0) -------------------------------------------------------------
    def initial_kalman(self, fp64_variance: bool = False) -> "KalmanState":
        return KalmanState(self, fp64_variance)

    def advance_kalman(self, source, state: "KalmanState", stream=None) -> None:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        st = self._lib.nf_kalman_advance_device(self._h, _plane(source, True), state._h, ctypes.c_void_p(s), err, 512)
        C.raise_for(st, err.value)

    def render_kalman(self, source, dst, state: "KalmanState", stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        st = self._lib.nf_kalman_render_device(self._h, _plane(source, True), _plane(dst, False), state._h,
                                               ctypes.c_void_p(s), err, 512)
        C.raise_for(st, err.value)
        return dst

    def step_kalman(self, source, dst, state: "KalmanState", stream=None):
        """advance_kalman(source, state) then render_kalman(source, dst, state) in one pass
        over the blocks (nf_kalman_step_device): the same results and errors."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        st = self._lib.nf_kalman_step_device(self._h, _plane(source, True), _plane(dst, False), state._h,
                                             ctypes.c_void_p(s), err, 512)
        C.raise_for(st, err.value)
        return dst


class KalmanState:
    """Device-resident Kalman state (kernels/kalman.hpp:5-14)."""

    def __init__(self, plan: Plan, fp64_variance: bool = False):
        self._lib = plan._lib
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        st = self._lib.nf_kalman_state_create(plan._h, int(fp64_variance), ctypes.byref(self._h), err, 512)
        C.raise_for(st, err.value)
        g = plan.geometry
        self.count = g.x.count * g.y.count * plan.bins

    def read(self):
        last = np.zeros((self.count, 2), np.float32)
        cov = np.zeros(self.count, np.float32)
        proc = np.zeros(self.count, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        C.raise_for(self._lib.nf_kalman_state_read(self._h, last.ctypes.data_as(fp), cov.ctypes.data_as(fp),
                                                   proc.ctypes.data_as(fp), self.count), b"state read failed")
        return last, cov, proc

    def copy_from(self, other: "KalmanState", stream=None) -> None:
        C.raise_for(self._lib.nf_kalman_state_copy(self._h, other._h, ctypes.c_void_p(stream or 0)),
                    b"state copy failed")

    def clone(self, stream=None) -> "KalmanState":
        """A new device state with the same plan, precision and contents (the copy a
        checkpoint takes, filter.hpp:171)."""
        out = KalmanState.__new__(KalmanState)
        out._lib, out.count = self._lib, self.count
        out._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_kalman_state_clone(self._h, ctypes.byref(out._h), ctypes.c_void_p(stream or 0),
                                                    err, 512), err.value)
        return out

    @property
    def nbytes(self) -> int:
        return int(self._lib.nf_kalman_state_bytes(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_kalman_state_destroy(h)
            self._h = None


class Batch:
    """Batched/persistent form: many single-frame planes (CUDA tensors) filtered by one
    persistent launch per block shape with a device work queue; `launch(graph=True)`
    replays a captured CUDA graph. Outputs equal per-plane `Plan.process_at`."""

    def __init__(self, items):
        """items: iterable of (plan, source_tensor, dst_tensor) or (plan, source_tensor,
        dst_tensor, frame, plane); frame and plane (default 0) are process_at's, and items
        that carry them may be dithered 8-bit DFTTest planes (nf_batch_create_indexed)."""
        self._lib = C.load()
        items = [tuple(it) for it in items]
        if any(len(it) not in (3, 5) for it in items):
            raise ValueError("batch items are (plan, source, dst) or (plan, source, dst, frame, plane)")
        self._keep = items  # planes must stay alive while the batch exists
        arr = (C.NfBatchItem * len(items))(*[C.NfBatchItem(it[0]._h.value, _plane(it[1], True), _plane(it[2], False))
                                             for it in items])
        self._plans = [it[0] for it in items]
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if any(len(it) == 5 for it in items):
            frames = (ctypes.c_int * len(items))(*[int(it[3]) if len(it) == 5 else 0 for it in items])
            planes = (ctypes.c_int * len(items))(*[int(it[4]) if len(it) == 5 else 0 for it in items])
            C.raise_for(self._lib.nf_batch_create_indexed(arr, frames, planes, len(items), ctypes.byref(self._h), err,
                                                          512), err.value)
        else:
            C.raise_for(self._lib.nf_batch_create(arr, len(items), ctypes.byref(self._h), err, 512), err.value)

    def launch(self, graph: bool = False, stream=None) -> None:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        fn = self._lib.nf_batch_graph_launch if graph else self._lib.nf_batch_launch
        C.raise_for(fn(self._h, ctypes.c_void_p(s), err, 512), err.value)

    @property
    def geometry_count(self) -> int:
        """Candidate strip geometries (the first launch times them and keeps the fastest)."""
        return int(self._lib.nf_batch_geometry_count(self._h))

    @property
    def mapped_planes(self) -> int:
        """Planes staged through bulk-tensor copies (2-D tensor maps) in the geometry in use."""
        return int(self._lib.nf_batch_mapped_planes(self._h))

    @property
    def geometry(self) -> int:
        """Index of the geometry in use; -1 before the first launch has tuned."""
        return int(self._lib.nf_batch_geometry(self._h))

    def select_geometry(self, index: int) -> None:
        """Fix the geometry (skips tuning; a captured graph is dropped)."""
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_batch_select_geometry(self._h, int(index), err, 512), err.value)

    def sync_status(self) -> None:
        for p in {id(p): p for p in self._plans}.values():
            p.sync_status()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_batch_destroy(h)
            self._h = None


class HostBatch:
    """Streamed host form: frames of single-frame planes in host memory (numpy arrays
    or CPU torch tensors; page-locked ones let the copies overlap the filtering)
    pass through a ring of `depth` device slots of `frames_per_chunk` frames.
    `plans[p]` filters plane p of every frame. Outputs equal `Plan.process` per plane."""

    def __init__(self, plans, frames_per_chunk: int = 1, depth: int = 4):
        self._lib = C.load()
        self._plans = list(plans)
        arr = (ctypes.c_void_p * len(self._plans))(*[p._h.value for p in self._plans])
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_host_batch_create(arr, len(self._plans), int(frames_per_chunk), int(depth),
                                                   ctypes.byref(self._h), err, 512), err.value)

    @property
    def device_bytes(self) -> int:
        return int(self._lib.nf_host_batch_device_bytes(self._h))

    def process(self, frames, outputs=None, stream=None, wait: bool = True):
        """frames[f][p] -> outputs[f][p] (allocated like the sources when omitted).
        Enqueued after the work on `stream` (torch's current stream by default); with
        wait=False the outputs are complete once that stream is synchronised."""
        import torch
        planes = len(self._plans)
        frames = [list(f) for f in frames]
        if any(len(f) != planes for f in frames):
            raise ValueError(f"every frame must hold {planes} planes")
        if outputs is None:
            outputs = [[torch.empty_like(x) if _is_torch(x) else np.empty_like(np.asarray(x)) for x in f]
                       for f in frames]
        n = len(frames)
        srcs = (C.NfConstPlane * max(1, n * planes))(*[_plane(x, True) for f in frames for x in f])
        dsts = (C.NfPlane * max(1, n * planes))(*[_plane(x, False) for f in outputs for x in f])
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_host_batch_process(self._h, srcs, dsts, n, ctypes.c_void_p(s), err, 512),
                    err.value)
        if wait:
            torch.cuda.synchronize()
        return outputs

    def sync_status(self) -> None:
        for p in {id(p): p for p in self._plans}.values():
            p.sync_status()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_host_batch_destroy(h)
            self._h = None


_FRAME_SOURCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(C.NfConstPlane))


class FrameServer:
    """Host request layer (src/plugin/filter.hpp:253-528): output frames of a clip of
    `num_frames` frames, filtered in ranges of about `range_frames` frames per batched
    launch with the host layer's frame selection. `source(frame, plane)` returns a 2-D
    plane (numpy array or torch tensor, host or CUDA); `plans[p]` None passes plane p
    through. `get(n)` returns frame n's planes; `request(n)` the source frames it reads."""

    def __init__(self, plans, num_frames: int, source, range_frames: int = 16):
        self._lib = C.load()
        self._plans = list(plans)
        self._source = source
        self._held = []
        self._error = None

        def fetch(_user, frame, plane, view):
            try:
                a = source(frame, plane)
                self._held.append(a)
                view[0] = _plane(a, True)
                return 0
            except Exception as e:  # reported through the status of the calling entry point
                self._error = e
                return 1

        self._fetch = _FRAME_SOURCE(fetch)
        arr = (ctypes.c_void_p * len(self._plans))(*[p._h.value if p is not None else None for p in self._plans])
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_frame_server_create(arr, len(self._plans), int(num_frames), int(range_frames),
                                                     ctypes.cast(self._fetch, ctypes.c_void_p), None,
                                                     ctypes.byref(self._h), err, 512), err.value)

    def request(self, n: int) -> list[int]:
        frames = (ctypes.c_int * 512)()
        count = ctypes.c_int()
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_frame_server_request(self._h, int(n), frames, 512, ctypes.byref(count), err, 512),
                    err.value)
        return list(frames[:count.value])

    def get(self, n: int, outputs=None):
        """Output frame n: outputs[p] (allocated as numpy arrays when omitted)."""
        if outputs is None:
            outputs = []
            for p, plan in enumerate(self._plans):
                if plan is None:
                    a = np.asarray(self._source(n, p))
                    outputs.append(np.empty_like(a))
                else:
                    g = plan.geometry
                    outputs.append(np.empty((g.y.length, g.x.length), dtype=plan.dtype))
        dsts = (C.NfPlane * len(outputs))(*[_plane(o, False) for o in outputs])
        err = ctypes.create_string_buffer(512)
        self._held, self._error = [], None
        try:
            st = self._lib.nf_frame_server_get(self._h, int(n), dsts, err, 512)
        finally:
            self._held = []
        e, self._error = self._error, None
        if st != C.NF_OK and e is not None:
            raise e  # the frame source's own exception
        C.raise_for(st, err.value)
        return outputs

    @property
    def counters(self) -> tuple[int, int]:
        """(output frames computed, source frames fetched) so far."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._lib.nf_frame_server_counters(self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_frame_server_destroy(h)
            self._h = None


def gather_noise(frames, location, z, block: int, fmt: SampleFormat) -> np.ndarray:
    """The host layer's sample gather (src/plugin/filter.hpp:381-389): rows
    y..y+block, columns x..x+block of plane `location[1]` of frame location[0] + z,
    decoded to 8-bit amplitude units. `frames(frame, plane)` returns a 2-D array."""
    frame, plane, y, x = location
    src = np.asarray(frames(frame + z, plane))
    if x > src.shape[1] - block or y > src.shape[0] - block:
        raise ValueError("sample frame rectangle differs from plan")
    scale = np.float32(255.0) if fmt.floating else np.float32(1.0 / float(1 << (fmt.bits - 8)))
    return (src[y:y + block, x:x + block].astype(np.float32) - np.float32(0)) * scale


class DFTNoise:
    """DFTNoise (src/algorithms/dft_noise.hpp:9-30): the sampled noise model shared by
    the DFTTest plans of one filter (nlocation, ftype 0/1). prepare(gather) builds the
    per-bin table from gathered sample volumes — gather(location, z) returns the
    block x block slice z of a location in 8-bit amplitude units (see gather_noise) —
    and publish(*plans) hands it to the plans."""

    def __init__(self, config: DFTConfig):
        loc = list(config.nlocation)
        if len(loc) % 4:
            raise ValueError("DFTTest nlocation requires quadruples")
        self.config = config
        self.locations = [tuple(loc[i:i + 4]) for i in range(0, len(loc), 4)]
        self.temporal_size, self.block_size = config.tbsize, config.block
        self.power = None

    def prepare(self, gather) -> np.ndarray:
        if self.power is not None:
            return self.power
        T, S = self.temporal_size, self.block_size
        slices = np.zeros((len(self.locations), T, S, S), np.float32)
        for i, location in enumerate(self.locations):
            for z in range(T):
                slices[i, z] = gather(location, z)
        lib = C.load()
        cfg, keep = self.config.to_c()
        out = np.zeros(T * S * (S // 2 + 1), np.float32)
        err = ctypes.create_string_buffer(512)
        C.raise_for(lib.nf_dft_noise_power(ctypes.byref(cfg), ctypes.c_void_p(slices.ctypes.data), len(self.locations),
                                           ctypes.c_void_p(out.ctypes.data), out.size, err, 512), err.value)
        del keep
        self.power = out
        return out

    def publish(self, *plans) -> None:
        if self.power is None:
            raise ValueError("DFTTest sample model not initialized")
        for p in plans:
            p.set_noise_model(self.power)


@dataclass
class ROI:
    """Region of interest of a plane (src/plugin/roi.hpp:6-11); `interlaced` packs the top
    field's rows, then the bottom field's rows in reverse order."""
    left: int
    top: int
    width: int
    height: int
    interlaced: bool = False

    @staticmethod
    def make(width, height, sub_w, sub_h, left=0, top=0, right=0, bottom=0, interlaced=False) -> "ROI":
        """make_roi (roi.hpp:13-23): margins in luma pixels, reduced by the subsampling."""
        r = C.NfRoi()
        err = ctypes.create_string_buffer(256)
        C.raise_for(C.load().nf_roi_make(width, height, sub_w, sub_h, left, top, right, bottom, int(interlaced),
                                         ctypes.byref(r), err, 256), err.value)
        return ROI(r.left, r.top, r.width, r.height, bool(r.interlaced))

    def row(self, y: int) -> int:
        if not self.interlaced:
            return y
        return 2 * y if y < self.height // 2 else 2 * (self.height - 1 - y) + 1

    def _c(self):
        return C.NfRoi(self.left, self.top, self.width, self.height, int(self.interlaced))

    def pack(self, plane, packed=None, stream=None):
        """Copies the ROI of a device plane into its packed image (PackedROI, roi.hpp:25-35)."""
        import torch
        if packed is None:
            packed = torch.empty((self.height, self.width), dtype=plane.dtype, device=plane.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(256)
        C.raise_for(C.load().nf_roi_pack_device(ctypes.byref(self._c()), _plane(plane, True), _plane(packed, False),
                                                plane.element_size(), ctypes.c_void_p(s), err, 256), err.value)
        return packed

    def unpack(self, packed, dst, stream=None):
        """Writes a packed image back into the ROI of a device plane (PackedROI::write)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(256)
        C.raise_for(C.load().nf_roi_unpack_device(ctypes.byref(self._c()), _plane(packed, True), _plane(dst, False),
                                                  packed.element_size(), ctypes.c_void_p(s), err, 256), err.value)
        return dst


class ClipBatch:
    """Temporal clips in batched form: `clips` is a list of (plan, frames, dsts) with
    device tensors; every output frame is filtered with the host layer's frame selection
    (FFT3D bt 2..5: temporal.fft3d_slots; DFTTest tmode 1: temporal.temporal_blocks;
    DFTTest tmode 0: the clamped centred window). FFT3D and DFTTest tmode 1 with tosize 0
    share each frame's transforms between outputs (two passes); the other DFTTest modes run
    one filter call per output frame inside the batch's launch and graph. Equal to
    per-frame process_at."""

    def __init__(self, clips):
        self._lib = C.load()
        self._keep = []
        items = []
        for plan, frames, dsts in clips:
            if len(frames) != len(dsts):
                raise ValueError("frames and dsts differ in length")
            fa = (C.NfConstPlane * len(frames))(*[_plane(f, True) for f in frames])
            da = (C.NfPlane * len(dsts))(*[_plane(d, False) for d in dsts])
            self._keep.append((plan, list(frames), list(dsts), fa, da))
            items.append(C.NfClipItem(plan._h.value, fa, da, len(frames)))
        arr = (C.NfClipItem * len(items))(*items)
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        C.raise_for(self._lib.nf_clip_batch_create(arr, len(items), ctypes.byref(self._h), err, 512), err.value)

    def launch(self, graph: bool = False, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        err = ctypes.create_string_buffer(512)
        fn = self._lib.nf_clip_batch_graph_launch if graph else self._lib.nf_clip_batch_launch
        C.raise_for(fn(self._h, ctypes.c_void_p(s), err, 512), err.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.nf_clip_batch_destroy(h)
            self._h = None


def kernel_info() -> dict:
    """KernelInfo (docs/api/en/kernel-info.md): labels of the active implementation."""
    lib = C.load()
    a, b, c = (ctypes.create_string_buffer(64) for _ in range(3))
    lanes = ctypes.c_int()
    lib.nf_kernel_info(a, 64, b, 64, c, 64, ctypes.byref(lanes))
    return {"fft_backend": a.value.decode(), "target": b.value.decode(), "fft": c.value.decode(),
            "fft_lanes": lanes.value}
