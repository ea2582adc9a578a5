"""Test infrastructure (oracle only): a binary64 re-evaluation of the reference core's
per-plane pipeline, with numpy's float64 FFTs. Never used by the product.

It is independent of the product's arithmetic: every transform is numpy.fft in binary64
(the pattern of the reference's own direct-DFT oracle, tests/reference/dft.hpp:4-33), and
every formula is restated here in binary64 from the reference core. The plan's binary32
creation-time tables are inputs: the FFT3D and DFTTest windows, DFTTest's wscale and its
sigma-curve table come from the compiled reference (oracle/_ref); the FFT3D sigma profile,
the enhancement windows and the degrid/zmean templates are re-evaluated in binary64 from
their formulas. Geometry and argument validation are the reference's (the same plan is
built there first).

Steps and where they come from:
  * decode (sample - base) * scale and single reflection into the cover plane
    (src/algorithms/pad.hpp:16-45, src/kernels/scalar/model.cpp:6-9);
  * FFT3D blocks: (padded * wy) * wx (src/kernels/scalar/spatial.cpp:12-16), rfft2;
    bt=1 Wiener max((q - a) / q, floor) with q = |X - M|^2 + 1e-15, M = degrid * X[0]/G[0] * G
    (src/kernels/scalar/spectral.cpp:5-53), sharpen/dehalo factor
    (src/algorithms/fft3d_profile.cpp:69-81) fused or as a second pass (plan.cpp:325-329,
    460-467); bt=2..5 temporal DFT, Wiener per temporal frequency with noise T*a, inverse at
    slot T/2, times 1/T (spectral.cpp:90-160); inverse rfft2 scaled 1/(bw*bh), synthesis
    wx * wy and overlap-add (plan.cpp:520-535); output clamp((z + 0.5) + base) or clamp(z, 0, 1)
    (plan.cpp:609-640, spatial.cpp:89-129);
  * FFT3D bt=0 (Kalman): per bin the reset-or-blend update of src/kernels/scalar/kalman.cpp:3-24
    on a binary64 state, render from the state's estimate with the enhancement pass
    (plan.cpp:293-321, 451-459);
  * DFTTest: blocks * h, rfft2 (tbsize 1) or rfftn over (time, y, x), zmean template
    M = X[0]/G[0] * G with G = FFT(255 h), gains of ftype 0..4 (spectral.cpp:5-53), inverse,
    synthesis h * volume (tmode 0: slice T/2) or (U * volume) * h (tmode 1, target slice),
    overlap-add or centre assignment (plan.cpp:538-607); output z / 255 (float) or
    clamp(trunc(z * 2^(bits-8) + 0.5)) (integer).

`process` returns the real-valued output before quantisation (the integer formats' value
in sample units); `quantize` applies the reference's final rounding and clamping.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import ref as R

EPS = 1e-15


def _reflect(length: int, offset: int, cover: int) -> np.ndarray:
    j = np.arange(cover) - offset
    return np.where(j < 0, -j, np.where(j < length, j, 2 * length - 2 - j))


@dataclass
class _Axis:
    length: int
    block: int
    overlap: int
    step: int
    count: int
    cover: int
    offset: int


def _blocks(padded: np.ndarray, ax: _Axis, ay: _Axis, rows: slice) -> np.ndarray:
    """Blocks of block rows `rows` as [nby, nx, bh, bw] (a copy)."""
    v = np.lib.stride_tricks.sliding_window_view(padded, (ay.block, ax.block))
    return np.array(v[::ay.step, ::ax.step][rows, :ax.count])


def _overlap_add(acc: np.ndarray, blk: np.ndarray, ax: _Axis, ay: _Axis, by0: int) -> None:
    """acc[by*sy + dy, bx*sx + dx] += blk[by - by0, bx, dy, dx]."""
    nby, nx, bh, bw = blk.shape
    y0 = by0 * ay.step
    for dy in range(bh):
        rows = slice(y0 + dy, y0 + dy + (nby - 1) * ay.step + 1, ay.step)
        for dx in range(bw):
            acc[rows, dx:dx + (nx - 1) * ax.step + 1:ax.step] += blk[:, :, dy, dx]


def _row_chunks(count: int, per: int):
    for a in range(0, count, per):
        yield slice(a, min(count, a + per)), a


class _Enhancement:
    """Sharpen/dehalo windows and constants in binary64 (fft3d_profile.cpp:30-68, table.cpp:40-49)."""

    def __init__(self, w: int, h: int, factor: float, c):
        self.sharpen, self.dehalo = float(c.sharpen), float(c.dehalo)
        self.active = self.sharpen != 0 or self.dehalo != 0
        if not self.active:
            return
        norm = 1.0 / (w * h)
        K = w // 2 + 1
        self.a = self.b = self.c = 0.0
        cutoff = 1.0
        if self.sharpen:
            lo, hi = c.smin * factor, c.smax * factor
            self.a, self.b = lo * lo / norm, hi * hi / norm
            cutoff = 2.0 * c.scutoff * c.scutoff
        if self.dehalo:
            self.c = c.ht * c.ht / norm
        x2 = np.arange(K, dtype=np.float64) ** 2 / float(w // 2) ** 2
        dy = np.array([y if y < h // 2 else h - y for y in range(h)], np.float64)
        y2 = dy * dy * c.svr * c.svr / float(h // 2) ** 2
        d2 = y2[:, None] + x2[None, :]
        self.sw = (1.0 - np.exp(-d2 / cutoff)).ravel()
        hw = np.exp(-0.7 * d2 * c.hr * c.hr) - np.exp(-d2 * c.hr * c.hr)
        self.hw = (hw / hw.max()).ravel() if self.dehalo else None

    def gain(self, q: np.ndarray) -> np.ndarray:
        s = np.ones_like(q)
        d = np.ones_like(q)
        if self.sharpen and self.b != 0:
            s = 1.0 + self.sharpen * self.sw * np.sqrt(q * self.b / ((q + self.a) * (q + self.b)))
        if self.dehalo:
            qc = q + self.c
            d = qc / (qc + self.dehalo * self.hw * q)
        return s * d


def _fft3d_profile(w: int, h: int, sigmas, norm: float) -> np.ndarray:
    """Analytic sigma profile of varying sigma1..4 in binary64 (fft3d_profile.cpp:13-27, table.cpp:5-17)."""
    K = w // 2 + 1
    fx = np.arange(K, dtype=np.float64) / K
    out = np.empty((h, K))
    a, b = np.sqrt(0.5) / 4, np.sqrt(0.5) / 2
    s = [float(v) for v in sigmas]
    for y in range(h):
        fy = (h - 2 * abs(y - h // 2)) / h
        f = np.sqrt((fy * fy + fx * fx) / 2.0)
        v = np.where(f < a, s[3] + (s[2] - s[3]) * f / a,
                     np.where(f < b, s[2] + (s[1] - s[2]) * (f - a) / (b - a), s[0] + (s[1] - s[0]) * (1 - f) / (1 - b)))
        out[y] = v * v / norm
    return out.ravel()


class FP64Plan:
    """Binary64 re-evaluation of one reference Plan (either algorithm)."""

    def __init__(self, width: int, height: int, fmt, config):
        from neo_fft_b200.plan import DFTConfig
        self.ref = R.RefPlan(width, height, fmt, config)  # validation and geometry
        self.w, self.h, self.fmt, self.c = width, height, fmt, config
        self.ax, self.ay = _Axis(**self.ref.x), _Axis(**self.ref.y)
        self.ix = _reflect(width, self.ax.offset, self.ax.cover)
        self.iy = _reflect(height, self.ay.offset, self.ay.cover)
        self.dft = isinstance(config, DFTConfig)
        self.peak = 1.0 if fmt.floating else float((1 << fmt.bits) - 1)
        if self.dft:
            self._init_dft()
        else:
            self._init_fft3d()

    # ---- creation-time tables ------------------------------------------------------
    def _init_fft3d(self):
        c, fmt = self.c, self.fmt
        bw, bh = c.bw, c.bh
        self.wxa, self.wxs = self._window(bw, self.ax.overlap, c.wintype)
        self.wya, self.wys = self._window(bh, self.ay.overlap, c.wintype)
        factor = 1.0 / 255.0 if fmt.floating else float(1 << (fmt.bits - 8))
        self.base = float(1 << (fmt.bits - 1)) if (not fmt.floating and fmt.chroma) else 0.0
        self.norm = 1.0 / (bw * bh)
        sig = [c.sigma, c.sigma if c.sigma2 is None else c.sigma2, c.sigma if c.sigma3 is None else c.sigma3,
               c.sigma if c.sigma4 is None else c.sigma4]
        sig = [float(np.float32(s)) * factor for s in sig]
        self.sigma_eff = sig[0]
        self.sbins = bh * (bw // 2 + 1)
        varying = any(s != sig[0] for s in sig[1:])
        if c.pfactor > 0 or c.pshow:
            raise ValueError("the binary64 re-evaluation covers plans without pattern sampling or preview")
        self.T = max(1, c.bt)
        self.kalman = c.bt == 0
        self.denoise = c.bt != -1
        self.floor = (c.beta - 1.0) / c.beta
        self.table = _fft3d_profile(bw, bh, sig, self.norm) if varying else None
        self.a = self.sigma_eff * self.sigma_eff / self.norm
        self.enh = _Enhancement(bw, bh, factor, c)
        self.fused_enh = self.enh.active and not varying and self.denoise
        self.mean_scale = float(c.degrid)
        self.grid = None
        if c.degrid != 0:
            self.grid = np.fft.rfft2(self.peak * np.outer(self.wya, self.wxa)).ravel()
        self.kratio2 = float(c.kratio) * float(c.kratio)

    def _init_dft(self):
        c, fmt = self.c, self.fmt
        B, T = c.block, c.tbsize
        h = np.zeros(T * B * B, np.float32)
        ws = np.zeros(1, np.float32)
        err = ctypes.create_string_buffer(256)
        rc = R.load().ref_dft_window_3d(T, B, 0 if c.mode == 0 else c.overlap, c.mode, c.swin, c.twin, c.sbeta,
                                        c.tbeta, c.temporal_mode, c.temporal_overlap, R.fp(h), R.fp(ws), err, 256)
        if rc:
            raise ValueError(err.value.decode())
        self.hwin = h.astype(np.float64).reshape(T, B, B)
        self.wscale = float(ws[0])
        self.T = T
        self.scale_in = 255.0 if fmt.floating else 1.0 / float(1 << (fmt.bits - 8))
        if c.ftype < 2 and len(c.nlocation):
            raise ValueError("the binary64 re-evaluation covers plans without sampled noise locations")
        scale = self.wscale if c.ftype < 2 else 1.0
        curves = any(len(getattr(c, n)) for n in ("slocation", "ssx", "ssy", "sst"))
        K = B // 2 + 1
        self.bins = T * B * K
        if curves:
            out = np.zeros(self.bins, np.float32)
            cfg, keep = c.to_c()
            rc = R.load().ref_dft_profile(ctypes.byref(cfg), np.float32(scale), R.fp(out), err, 256)
            if rc:
                raise ValueError(err.value.decode())
            self.table = out.astype(np.float64)
        else:
            self.table = None
        # SpectralParams (plan.cpp:199-207) in binary64
        self.a = 0.0 if curves else c.sigma / scale
        self.b = c.sigma2 / scale
        self.low, self.high = c.pmin / self.wscale, c.pmax / self.wscale
        self.exponent = float(c.f0beta)
        self.mean_scale = 1.0 if c.zmean else 0.0
        self.grid = None
        if c.zmean:
            self.grid = (np.fft.rfft2(255.0 * self.hwin[0]) if T == 1 else np.fft.rfftn(255.0 * self.hwin)).ravel()
        self.tmode1 = c.temporal_mode == 1
        self.center = c.mode == 0

    @staticmethod
    def _window(block, overlap, wintype):
        a = np.zeros(block, np.float32)
        s = np.zeros(block, np.float32)
        err = ctypes.create_string_buffer(256)
        if R.load().ref_fft3d_window(block, overlap, wintype, R.fp(a), R.fp(s), err, 256):
            raise ValueError(err.value.decode())
        return a.astype(np.float64), s.astype(np.float64)

    # ---- pipeline ------------------------------------------------------------------
    def _pad(self, src: np.ndarray, base: float, scale: float) -> np.ndarray:
        x = (np.asarray(src).astype(np.float64) - base) * scale
        return x[self.iy][:, self.ix]

    def _mean(self, spec: np.ndarray, force_zero: bool = False) -> np.ndarray:
        """M = scale * G per block; spec [..., bins]."""
        if self.grid is None:
            return np.zeros_like(spec)
        if force_zero:
            return np.zeros_like(spec)
        g = self.mean_scale * spec[..., :1].real / self.grid[0].real
        return g * self.grid

    def _enhance(self, X: np.ndarray) -> np.ndarray:
        M = self._mean(X)
        Rr = X - M
        q = Rr.real ** 2 + Rr.imag ** 2 + EPS
        return self.enh.gain(q) * Rr + M

    def _output(self, acc: np.ndarray) -> np.ndarray:
        z = acc[self.ay.offset:self.ay.offset + self.h, self.ax.offset:self.ax.offset + self.w]
        if self.dft:
            return z / 255.0 if self.fmt.floating else z * float(1 << (self.fmt.bits - 8))
        return np.clip(z, 0.0, 1.0) if self.fmt.floating else z + self.base

    def quantize(self, v: np.ndarray) -> np.ndarray:
        """The reference's final conversion of `process`'s values (integer formats)."""
        if self.fmt.floating:
            return v.astype(np.float32)
        q = np.clip(v + 0.5, 0.0, self.peak).astype(np.int64)
        return q.astype(np.uint8 if self.fmt.bits == 8 else np.uint16)

    def process(self, sources, targets=(), rows_per_chunk: int = 24) -> np.ndarray:
        if not isinstance(sources, (list, tuple)):
            sources = [sources]
        if self.dft:
            return self._process_dft(list(sources), list(targets), rows_per_chunk)
        return self._process_fft3d(list(sources), rows_per_chunk)

    def _synth_fft3d(self, X: np.ndarray, acc: np.ndarray, by0: int) -> None:
        c = self.c
        blk = np.fft.irfft2(X.reshape(*X.shape[:2], c.bh, c.bw // 2 + 1), s=(c.bh, c.bw))
        _overlap_add(acc, blk * np.outer(self.wys, self.wxs), self.ax, self.ay, by0)

    def _process_fft3d(self, sources, rows_per_chunk):
        c = self.c
        if self.kalman:
            raise ValueError("Kalman plans run through FP64Kalman")
        T = len(sources)
        if T not in (1, self.T):
            raise ValueError("FFT3D sources size must match plan temporal_size or single-frame fallback")
        padded = [self._pad(s, self.base, 1.0) for s in sources]
        acc = np.zeros((self.ay.cover, self.ax.cover))
        win = np.outer(self.wya, self.wxa)
        for rows, by0 in _row_chunks(self.ay.count, rows_per_chunk):
            spec = [np.fft.rfft2(_blocks(p, self.ax, self.ay, rows) * win).reshape(rows.stop - by0, self.ax.count, -1)
                    for p in padded]
            if T == 1:
                X = spec[0]
                if self.denoise:
                    M = self._mean(X)
                    Rr = X - M
                    q = Rr.real ** 2 + Rr.imag ** 2 + EPS
                    a = self.table if self.table is not None else self.a
                    gain = np.maximum((q - a) / q, self.floor)
                    if self.fused_enh:
                        gain = gain * self.enh.gain(q)
                    X = gain * Rr + M
                    if self.table is not None and self.enh.active:
                        X = self._enhance(X)
                elif self.enh.active:
                    X = self._enhance(X)
            else:
                X = self._temporal(spec)
                if self.enh.active:
                    X = self._enhance(X)
            self._synth_fft3d(X, acc, by0)
        return self._output(acc)

    def _temporal(self, spec):
        """FFT3D bt=2..5 per bin (spectral.cpp:90-160) in binary64."""
        T = len(spec)
        c = T // 2
        M = self._mean(spec[c])
        gT = M * T
        j = np.arange(T)
        fwd = np.exp(-2j * np.pi * np.outer(j, j) / T)   # [m][j]
        inv = np.exp(2j * np.pi * c * j / T)              # [m]
        noise = T * (self.table if self.table is not None else self.a)
        y = np.zeros_like(spec[0])
        for m in range(T):
            F = sum(spec[jj] * fwd[m, jj] for jj in range(T))
            Rr = F - gT if m == 0 else F
            q = Rr.real ** 2 + Rr.imag ** 2 + EPS
            gain = np.maximum((q - noise) / q, self.floor)
            Fo = gain * Rr + (gT if m == 0 else 0)
            y = y + Fo * inv[m]
        return y / T

    # ---- DFTTest ----------------------------------------------------------------
    def _gain_dft(self, q_power: np.ndarray) -> np.ndarray:
        c = self.c
        p = q_power
        a = self.table if self.table is not None else self.a
        if c.ftype == 0:
            wiener = np.maximum((p - a) / (p + EPS), 0.0)
            if abs(self.exponent - 1.0) < 5e-5:
                return wiener
            if abs(self.exponent - 0.5) < 5e-5:
                return np.sqrt(wiener)
            return wiener ** self.exponent
        if c.ftype == 1:
            return np.where(p < a, 0.0, 1.0)
        if c.ftype == 2:
            return np.broadcast_to(a, p.shape).astype(np.float64)
        if c.ftype == 3:
            return np.where((p >= self.low) & (p <= self.high), a, self.b)
        q = p + EPS
        return a * np.sqrt(q * self.high / ((q + self.low) * (q + self.high)))

    def block_outputs(self, sources, rows_per_chunk: int = 24) -> list:
        """DFTTest tmode 1: the outputs of one temporal block for every target slice
        0..T-1 (each equal to process(sources, targets=[z])), filtering the block once."""
        if not (self.dft and self.tmode1):
            raise ValueError("block_outputs is for DFTTest tmode 1 plans")
        return [self._output(a) for a in self._dft_accumulate(list(sources), list(range(self.T)), rows_per_chunk,
                                                               per_target=True)]

    def _process_dft(self, sources, targets, rows_per_chunk):
        return self._output(self._dft_accumulate(sources, targets, rows_per_chunk)[0])

    def _dft_accumulate(self, sources, targets, rows_per_chunk, per_target=False):
        c = self.c
        T, B = self.T, c.block
        K = B // 2 + 1
        nblocks = len(targets) if self.tmode1 else 1
        if self.tmode1 and per_target:
            if len(sources) != T:
                raise ValueError("invalid temporal block inputs")
        elif self.tmode1:
            if not targets or len(sources) != len(targets) * T:
                raise ValueError("invalid temporal block inputs")
        elif len(sources) != T:
            raise ValueError("DFTTest sources size must match plan temporal_size")
        if per_target:
            nblocks = 1
        accs = [np.zeros((self.ay.cover, self.ax.cover)) for _ in range(len(targets) if per_target else 1)]
        vol = float(T * B * B)
        for tb in range(nblocks):
            padded = [self._pad(s, 0.0, self.scale_in) for s in sources[tb * T:(tb + 1) * T]]
            for rows, by0 in _row_chunks(self.ay.count, rows_per_chunk):
                vols = np.stack([_blocks(p, self.ax, self.ay, rows) for p in padded], axis=2)  # [nby,nx,T,B,B]
                vols = vols * self.hwin
                if T == 1:
                    X = np.fft.rfft2(vols[:, :, 0]).reshape(*vols.shape[:2], -1)
                else:
                    X = np.fft.rfftn(vols, axes=(2, 3, 4)).reshape(*vols.shape[:2], -1)
                zero_mean = T > 1 and (self.mean_scale == 0 or (self.grid is not None and self.grid[0].real == 0))
                M = self._mean(X, force_zero=zero_mean)
                Rr = X - M
                p = Rr.real ** 2 + Rr.imag ** 2
                X = self._gain_dft(p) * Rr + M
                if T == 1:
                    full = np.fft.irfft2(X.reshape(*X.shape[:2], B, K), s=(B, B))[:, :, None]
                else:
                    full = np.fft.irfftn(X.reshape(*X.shape[:2], T, B, K), s=(T, B, B), axes=(2, 3, 4))
                for i, acc in enumerate(accs):
                    centre = (targets[i] if per_target else targets[tb]) if self.tmode1 else T // 2
                    inv = full[:, :, centre if T > 1 else 0]
                    if self.tmode1:
                        blk = (inv * vol) * self.hwin[centre]
                    else:
                        blk = inv * (self.hwin[centre] * vol)
                    if self.center:
                        cy, cx = B // 2, B // 2
                        ys = by0 * self.ay.step + cy + np.arange(blk.shape[0]) * self.ay.step
                        xs = cx + np.arange(blk.shape[1]) * self.ax.step
                        if self.tmode1:
                            acc[np.ix_(ys, xs)] += blk[:, :, cy, cx]
                        else:
                            acc[np.ix_(ys, xs)] = blk[:, :, cy, cx]
                    else:
                        _overlap_add(acc, blk, self.ax, self.ay, by0)
        return accs


class FP64Kalman:
    """FFT3D bt=0 in binary64: a state (estimate, covariance, process variance) per bin,
    advanced per frame and rendered through the enhancement pass, inverse and overlap-add."""

    def __init__(self, plan: FP64Plan):
        if not plan.kalman:
            raise ValueError("not a Kalman plan")
        self.p = plan
        n = plan.ay.count * plan.ax.count * plan.sbins
        r0 = plan.sigma_eff * plan.sigma_eff / plan.norm
        self.r0 = r0
        self.ambiguous = 0  # motion-test decisions within binary32 rounding of the threshold
        self.last = np.zeros(n, np.complex128)
        self.cov = np.full(n, r0)
        self.proc = np.full(n, r0)

    def advance(self, src) -> None:
        p = self.p
        padded = p._pad(src, p.base, 1.0)
        win = np.outer(p.wya, p.wxa)
        X = np.fft.rfft2(_blocks(padded, p.ax, p.ay, slice(0, p.ay.count)) * win).ravel()
        if p.table is not None:
            r = np.tile(np.maximum(p.table, 1e-15), p.ay.count * p.ax.count)
        else:
            r = np.full(X.shape, self.r0)
        thr = r * p.kratio2
        d = X - self.last
        reset = (d.real ** 2 > thr) | (d.imag ** 2 > thr)
        # decisions a binary32 evaluation can take the other way: a squared difference
        # within 1e-5 (relative) of the threshold
        near = (np.abs(d.real ** 2 - thr) <= 1e-5 * thr) | (np.abs(d.imag ** 2 - thr) <= 1e-5 * thr)
        self.ambiguous += int(near.sum())
        if p.table is None and self.r0 == 0:
            reset[:] = True
        s = self.cov + self.proc
        g = s / (s + r)
        nq = g * g * r
        nc = (1.0 - g) * s
        nl = g * X + (1.0 - g) * self.last
        self.last = np.where(reset, X, nl)
        self.cov = np.where(reset, r, nc)
        self.proc = np.where(reset, r, nq)

    def render(self) -> np.ndarray:
        p = self.p
        acc = np.zeros((p.ay.cover, p.ax.cover))
        X = self.last.reshape(p.ay.count, p.ax.count, -1)
        if p.enh.active:
            X = p._enhance(X)
        p._synth_fft3d(X, acc, 0)
        return p._output(acc)
