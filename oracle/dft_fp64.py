"""Test infrastructure (oracle only): a binary64, differentiable PyTorch restatement of
the reference DFTTest spatial path (tbsize 1, smode 1, float planes, ftype 0/1/2), used
as the gradient oracle for the sm_100a adjoint kernels. Never used by the product.

Steps, each following the reference core:
  * decode and reflect-pad: padded = 255 * src[reflect(y - offset_y), reflect(x - offset_x)]
    over cover_h x cover_w (src/algorithms/pad.hpp:41-45 and :65-80);
  * per block at (by*step, bx*step): analysis window h (src/algorithms/windows.cpp, taken from
    the reference's own dft_window_3d), forward r2c (unnormalised), spectrum layout
    [row][bin] with bin = 0..sbsize/2 (src/algorithms/plan.cpp:563-570);
  * zmean: scale = spectrum[0].re / grid[0].re with grid = r2c(255 * h) (plan.cpp:213-224, :575);
  * spectral gain per bin k with threshold a = table[k] (src/kernels/scalar/spectral.cpp:7-52):
    ftype 0: max((p - a) / (p + 1e-15), 0); ftype 1: p < a ? 0 : 1; ftype 2: a,
    applied to the mean-removed bin and the mean added back;
  * normalised c2r, times h * sbsize^2 (h_synthesis, plan.cpp:616-617), summed into the
    accumulator (scatter_dfttest, plan.cpp:596-598);
  * output = accum[offset_y + y][offset_x + x] / 255 (plan.cpp:604-609).

Parity of this restatement is pinned by `forward` agreeing with the reference plan's own
float32 output (tests/test_gpu_adjoint.py checks it on each configuration it uses).
"""
from __future__ import annotations

import ctypes

import numpy as np


def reference_tables(config):
    """(h [b, b] float32, wscale) from the reference's own window builder."""
    from . import ref
    b = config.block
    h = np.zeros(b * b, np.float32)
    w1 = np.zeros(1, np.float32)
    err = ctypes.create_string_buffer(256)
    rc = ref.load().ref_dft_window_3d(1, b, config.overlap, 1, config.swin, config.twin, config.sbeta,
                                      config.tbeta, config.temporal_mode, config.temporal_overlap,
                                      ref.fp(h), ref.fp(w1), err, 256)
    if rc:
        raise ValueError(err.value.decode())
    return h.reshape(b, b), float(w1[0])


def _reflect_index(length: int, offset: int, cover: int):
    j = np.arange(cover) - offset
    j = np.where(j < 0, -j, np.where(j < length, j, 2 * length - 2 - j))
    return j


class DFTTestFP64:
    """forward(x [B, H, W] float64 tensor, table [b*(b/2+1)] float64 tensor) -> [B, H, W]."""

    def __init__(self, width: int, height: int, config):
        from . import ref
        from neo_fft_b200.plan import SampleFormat
        if config.tbsize != 1 or config.mode != 1 or config.ftype not in (0, 1, 2):
            raise ValueError("restatement covers tbsize 1, smode 1, ftype 0..2")
        rp = ref.RefPlan(width, height, SampleFormat(32, True), config)
        self.gx, self.gy = rp.x, rp.y
        self.width, self.height, self.config = width, height, config
        self.h, self.wscale = reference_tables(config)
        self.iy = _reflect_index(height, self.gy["offset"], self.gy["cover"])
        self.ix = _reflect_index(width, self.gx["offset"], self.gx["cover"])

    def forward(self, x, table):
        import torch
        import torch.nn.functional as F
        b = self.config.block
        step = b - self.config.overlap
        dev = x.device
        h = torch.from_numpy(self.h.astype(np.float64)).to(dev)
        iy = torch.from_numpy(self.iy).to(dev)
        ix = torch.from_numpy(self.ix).to(dev)
        padded = 255.0 * x[:, iy][:, :, ix]                           # [B, Ch, Cw]
        B, ch, cw = padded.shape
        ny, nx = self.gy["count"], self.gx["count"]
        blocks = padded.unfold(1, b, step).unfold(2, b, step)       # [B, ny, nx, b, b]
        blocks = blocks[:, :ny, :nx] * h
        spec = torch.fft.rfft2(blocks)                              # [B, ny, nx, b, b/2+1]
        a = table.reshape(b, b // 2 + 1)
        if self.config.zmean:
            grid = torch.fft.rfft2(255.0 * h)
            mean = (spec[..., 0, 0].real / grid[0, 0].real)[..., None, None] * grid
        else:
            mean = torch.zeros_like(spec)
        re = spec - mean
        power = re.real ** 2 + re.imag ** 2
        if self.config.ftype == 0:
            gain = torch.clamp((power - a) / (power + 1e-15), min=0.0)
        elif self.config.ftype == 1:
            gain = (power >= a).to(power.dtype)
        else:
            gain = a.expand_as(power)
        filtered = gain * re + mean
        out_blocks = torch.fft.irfft2(filtered, s=(b, b)) * (h * float(b * b))
        cols = out_blocks.permute(0, 3, 4, 1, 2).reshape(B, b * b, ny * nx)
        acc = F.fold(cols, output_size=(ch, cw), kernel_size=b, stride=step)[:, 0]
        oy, ox = self.gy["offset"], self.gx["offset"]
        return acc[:, oy:oy + self.height, ox:ox + self.width] / 255.0

    def kink_distance(self, x, table):
        """Per block [B, ny, nx]: the smallest relative distance |p - a| / a of any bin's power
        from the threshold where the ftype 0 gain has its kink (binary64)."""
        import torch
        with torch.no_grad():
            b = self.config.block
            step = b - self.config.overlap
            h = torch.from_numpy(self.h.astype(np.float64))
            padded = 255.0 * x[:, torch.from_numpy(self.iy)][:, :, torch.from_numpy(self.ix)]
            ny, nx = self.gy["count"], self.gx["count"]
            spec = torch.fft.rfft2(padded.unfold(1, b, step).unfold(2, b, step)[:, :ny, :nx] * h)
            a = table.reshape(b, b // 2 + 1)
            if self.config.zmean:
                grid = torch.fft.rfft2(255.0 * h)
                spec = spec - (spec[..., 0, 0].real / grid[0, 0].real)[..., None, None] * grid
            p = spec.real ** 2 + spec.imag ** 2
            return (torch.abs(p - a) / a).amin(dim=(-2, -1))

    def uniform_table(self):
        """The table a DFTTest plan without curves uses: sigma / wscale for ftype 0/1, sigma for 2."""
        c = self.config
        b = c.block
        v = np.float32(c.sigma) / np.float32(self.wscale) if c.ftype < 2 else np.float32(c.sigma)
        return np.full(b * (b // 2 + 1), v, np.float32)


class FFT3DFP64:
    """Binary64, differentiable restatement of the reference FFT3D bt=1 path for float planes
    (src/algorithms/plan.cpp:432-537): decode (no scale), single reflection into the cover,
    blocks (v*wy)*wx, r2c, degrid template M = degrid * X0/G0 * G with G = r2c(wy*wx),
    gain max((q - a)/q, floor) with q = |X - M|^2 + 1e-15 (kernels/scalar/spectral.cpp:18-22)
    times the sharpen/dehalo factor S(q)D(q) (algorithms/fft3d_profile.cpp:69-81; windows in
    binary64 as in oracle/fp64_pipeline.py), Y = gain*R + M; for varying-sigma plans the
    enhancement is a second pass on Y with its own template term (plan.cpp:476-481, 325-329);
    c2r / (bw*bh), synthesis wxs*wys,
    overlap-add, output clamp(z, 0, 1) whose gradient passes where 0 < z < 1.

    forward(x [B, H, W] float64 tensor, table [bh*(bw/2+1)] float64 tensor) -> [B, H, W]; the
    table is the per-bin noise power a (uniform sigma: sigma^2/norm in every bin)."""

    def __init__(self, width: int, height: int, config):
        from . import ref
        from .fp64_pipeline import FP64Plan
        from neo_fft_b200.plan import SampleFormat
        if config.bt != 1 or config.pfactor > 0 or config.pshow:
            raise ValueError("restatement covers FFT3D bt=1 without pattern sampling")
        self.fp = FP64Plan(width, height, SampleFormat(32, True), config)
        rp = self.fp.ref
        self.gx, self.gy = rp.x, rp.y
        self.width, self.height, self.config = width, height, config
        self.iy = _reflect_index(height, self.gy["offset"], self.gy["cover"])
        self.ix = _reflect_index(width, self.gx["offset"], self.gx["cover"])

    def forward(self, x, table):
        import torch
        import torch.nn.functional as F
        fp, c = self.fp, self.config
        bh, bw = c.bh, c.bw
        dev = x.device
        t = lambda a: torch.from_numpy(np.asarray(a, np.float64)).to(dev)  # noqa: E731
        wa = t(np.outer(fp.wya, fp.wxa))
        ws = t(np.outer(fp.wys, fp.wxs))
        padded = x[:, torch.from_numpy(self.iy).to(dev)][:, :, torch.from_numpy(self.ix).to(dev)]
        B, ch, cw = padded.shape
        sy, sx = self.gy["step"], self.gx["step"]
        ny, nx = self.gy["count"], self.gx["count"]
        blocks = padded.unfold(1, bh, sy).unfold(2, bw, sx)[:, :ny, :nx] * wa
        spec = torch.fft.rfft2(blocks)
        K = bw // 2 + 1
        if fp.grid is not None:
            grid = t(fp.grid.real).reshape(bh, K) + 1j * t(fp.grid.imag).reshape(bh, K)
            mean = (fp.mean_scale * spec[..., 0, 0].real / grid[0, 0].real)[..., None, None] * grid
        else:
            mean = torch.zeros_like(spec)
        R = spec - mean
        q = R.real ** 2 + R.imag ** 2 + 1e-15
        a = table.reshape(bh, K)
        r = (q - a) / q
        gain = torch.where(r >= fp.floor, r, torch.full_like(r, fp.floor))
        e = fp.enh

        def enhancement(qq):  # S(q) * D(q)
            s = torch.ones_like(qq)
            d = torch.ones_like(qq)
            if e.sharpen and e.b != 0:
                s = 1.0 + e.sharpen * t(e.sw).reshape(bh, K) * torch.sqrt(qq * e.b / ((qq + e.a) * (qq + e.b)))
            if e.dehalo:
                qc = qq + e.c
                d = qc / (qc + e.dehalo * t(e.hw).reshape(bh, K) * qq)
            return s * d

        if e.active and fp.table is None:  # uniform sigma: enhancement fused into the Wiener gain
            gain = gain * enhancement(q)
        Y = gain * R + mean
        if e.active and fp.table is not None:
            # varying sigma (plan.cpp:476-481): the Wiener output is enhanced in a second pass
            # whose template term is recomputed from that output's DC (enhance, plan.cpp:325-329)
            if fp.grid is not None:
                mean2 = (fp.mean_scale * Y[..., 0, 0].real / grid[0, 0].real)[..., None, None] * grid
            else:
                mean2 = torch.zeros_like(Y)
            R2 = Y - mean2
            Y = enhancement(R2.real ** 2 + R2.imag ** 2 + 1e-15) * R2 + mean2
        out_blocks = torch.fft.irfft2(Y, s=(bh, bw)) * ws
        cols = out_blocks.permute(0, 3, 4, 1, 2).reshape(B, bh * bw, ny * nx)
        acc = F.fold(cols, output_size=(ch, cw), kernel_size=(bh, bw), stride=(sy, sx))[:, 0]
        oy, ox = self.gy["offset"], self.gx["offset"]
        z = acc[:, oy:oy + self.height, ox:ox + self.width]
        self.last_z, self.last_kink = z.detach(), None
        # per block: smallest relative distance of q from the kink of max((q - a)/q, floor),
        # q = a / (1 - floor)
        qk = a.detach() / (1.0 - fp.floor)
        self.last_kink = (torch.abs(q.detach() - qk) / qk).amin(dim=(-2, -1))
        return torch.where((z > 0) & (z < 1), z, z.detach().clamp(0.0, 1.0))

    def uniform_table(self):
        """The table of a uniform-sigma plan: a = sigma_eff^2 / norm in every bin (binary32)."""
        c = self.config
        sig = np.float32(np.float32(c.sigma) * np.float32(1.0 / 255.0))
        a = np.float32(np.float32(sig * sig) / np.float32(1.0 / (np.float32(c.bw) * np.float32(c.bh))))
        return np.full(c.bh * (c.bw // 2 + 1), a, np.float32)
