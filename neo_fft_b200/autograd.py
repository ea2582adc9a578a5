"""Differentiable DFTTest (tbsize=1, smode=1, float planes, ftype 0/1/2) and FFT3D (bt=1,
float planes, sharpen/dehalo fused into the gain) for PyTorch.

`DFTTestFunction.apply(x, table, plan)` filters a batch of float32 CUDA planes
x[B, H, W] with the primary table `table` (the per-bin threshold the Wiener gain
compares with, [sbsize * (sbsize//2+1)], already calibrated) and differentiates with
respect to both. Forward runs the sm_100a strip kernel over up to 32 planes per launch (results
identical to `Plan.process`); backward runs the hand-written adjoint kernels through the C ABI
(nf_dft_backward_device), recomputing block spectra instead of storing them.

`FFT3DFunction.apply(x, table, plan)` does the same for an FFT3D plan, whose table is the
per-bin noise power a of the Wiener gain max((q - a)/q, floor) (a uniform-sigma plan starts
from sigma^2/norm in every bin); its backward (nf_fft3d_backward_device) also takes the
forward output, because the float output is clamped to [0, 1].

`SigmaTableDenoiser` wraps either as a module with a learnable table; in data-parallel
training its table gradient is all-reduced once per step (`allreduce_table_grad`).
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi as C
from .plan import DFTConfig, FFT3DConfig, Plan, SampleFormat


def _set_primary(plan: Plan, table: torch.Tensor, stream) -> torch.Tensor:
    t = table.detach()
    if t.dtype != torch.float32 or not t.is_contiguous():
        t = t.contiguous().to(torch.float32)
    err = ctypes.create_string_buffer(256)
    C.raise_for(plan._lib.nf_plan_set_primary(plan._h, ctypes.c_void_p(t.data_ptr()), t.numel(), stream, err, 256),
                err.value)
    return t


def _plane_array(t: torch.Tensor, start: int, n: int, const: bool):
    """ctypes array of n planes t[start:start+n] of a contiguous [B, H, W] float32 tensor,
    built from the base pointer (no per-plane tensor views)."""
    cls = C.NfConstPlane if const else C.NfPlane
    _, h, w = t.shape
    step = h * w * 4
    base = t.data_ptr() + start * step
    return (cls * n)(*[cls(base + i * step, w, h, w * 4) for i in range(n)])


class DFTTestFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, table: torch.Tensor, plan: Plan):
        if x.dim() != 3 or x.dtype != torch.float32 or not x.is_cuda:
            raise ValueError("x must be a float32 CUDA tensor [batch, height, width]")
        x = x.contiguous()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        keep = _set_primary(plan, table, stream)
        out = torch.empty_like(x)
        err = ctypes.create_string_buffer(256)
        for start in range(0, x.shape[0], 32):
            n = min(32, x.shape[0] - start)
            C.raise_for(plan._lib.nf_plan_process_planes_device(plan._h, _plane_array(x, start, n, True),
                                                                _plane_array(out, start, n, False), n, stream,
                                                                err, 256), err.value)
        ctx.save_for_backward(x, keep)
        ctx.plan = plan
        return out

    @staticmethod
    def backward(ctx, gout: torch.Tensor):
        x, table = ctx.saved_tensors
        plan: Plan = ctx.plan
        gout = gout.contiguous()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        keep = _set_primary(plan, table, stream)  # noqa: F841 (kept alive until the launch is enqueued)
        gx = torch.empty_like(x)
        lib = plan._lib
        err = ctypes.create_string_buffer(256)
        nb = x.shape[0]
        chunks = [(s0, min(32, nb - s0)) for s0 in range(0, nb, 32)]
        parts = torch.empty((len(chunks), table.numel()), dtype=torch.float32, device=x.device)
        need = ctypes.c_size_t()
        lib.nf_dft_backward_scratch_bytes(plan._h, chunks[0][1], ctypes.byref(need))
        scratch = torch.empty(max(1, need.value), dtype=torch.uint8, device=x.device)
        for c, (start, n) in enumerate(chunks):
            st = lib.nf_dft_backward_device(plan._h, _plane_array(x, start, n, True), _plane_array(gout, start, n, True),
                                            _plane_array(gx, start, n, False), n,
                                            ctypes.c_void_p(parts[c].data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
                                            need.value, stream, err, 256)
            C.raise_for(st, err.value)
        gtab = parts[0] if len(chunks) == 1 else parts.sum(0)
        return gx, gtab.to(table.dtype).view_as(table), None


class FFT3DFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, table: torch.Tensor, plan: Plan):
        if x.dim() != 3 or x.dtype != torch.float32 or not x.is_cuda:
            raise ValueError("x must be a float32 CUDA tensor [batch, height, width]")
        x = x.contiguous()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        keep = _set_primary(plan, table, stream)
        out = torch.empty_like(x)
        err = ctypes.create_string_buffer(256)
        for start in range(0, x.shape[0], 32):
            n = min(32, x.shape[0] - start)
            C.raise_for(plan._lib.nf_plan_process_planes_device(plan._h, _plane_array(x, start, n, True),
                                                                _plane_array(out, start, n, False), n, stream,
                                                                err, 256), err.value)
        ctx.save_for_backward(x, keep, out)
        ctx.plan = plan
        return out

    @staticmethod
    def backward(ctx, gout: torch.Tensor):
        x, table, out = ctx.saved_tensors
        plan: Plan = ctx.plan
        gout = gout.contiguous()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        keep = _set_primary(plan, table, stream)  # noqa: F841 (kept alive until the launch is enqueued)
        gx = torch.empty_like(x)
        lib = plan._lib
        err = ctypes.create_string_buffer(256)
        nb = x.shape[0]
        chunks = [(s0, min(32, nb - s0)) for s0 in range(0, nb, 32)]
        parts = torch.empty((len(chunks), table.numel()), dtype=torch.float32, device=x.device)
        need = ctypes.c_size_t()
        lib.nf_dft_backward_scratch_bytes(plan._h, chunks[0][1], ctypes.byref(need))
        scratch = torch.empty(max(1, need.value), dtype=torch.uint8, device=x.device)
        for c, (start, n) in enumerate(chunks):
            st = lib.nf_fft3d_backward_device(plan._h, _plane_array(x, start, n, True), _plane_array(out, start, n, True),
                                              _plane_array(gout, start, n, True), _plane_array(gx, start, n, False), n,
                                              ctypes.c_void_p(parts[c].data_ptr()),
                                              ctypes.c_void_p(scratch.data_ptr()), need.value, stream, err, 256)
            C.raise_for(st, err.value)
        gtab = parts[0] if len(chunks) == 1 else parts.sum(0)
        return gx, gtab.to(table.dtype).view_as(table), None


class SigmaTableDenoiser(torch.nn.Module):
    """DFTTest or FFT3D with a learnable per-frequency table: DFTTest's threshold table
    (sbsize x (sbsize//2+1)) or FFT3D's noise power table (bh x (bw//2+1))."""

    def __init__(self, width: int, height: int, config, initial: torch.Tensor | None = None):
        super().__init__()
        self.fft3d = isinstance(config, FFT3DConfig)
        if self.fft3d:
            if config.bt != 1 or config.pfactor > 0 or config.pshow:
                raise ValueError("differentiable FFT3D needs bt=1 without pattern sampling or preview")
            k = config.bh * (config.bw // 2 + 1)
        else:
            if config.tbsize != 1 or config.mode != 1 or config.ftype not in (0, 1, 2):
                raise ValueError("differentiable DFTTest needs tbsize=1, smode=1 and ftype 0, 1 or 2")
            k = config.block * (config.block // 2 + 1)
        self.plan = Plan(width, height, SampleFormat(32, True), config)
        if initial is None:
            initial = torch.empty(k, dtype=torch.float32, device="cuda")
            err = ctypes.create_string_buffer(256)
            stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            C.raise_for(self.plan._lib.nf_plan_get_primary(self.plan._h, ctypes.c_void_p(initial.data_ptr()), k,
                                                           stream, err, 256), err.value)
        self.table = torch.nn.Parameter(initial.clone().float().cuda())

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        return (FFT3DFunction if self.fft3d else DFTTestFunction).apply(x, self.table, self.plan)


def shard(n: int, rank: int, world: int) -> range:
    """Contiguous shard of n patches for data-parallel training."""
    per = (n + world - 1) // world
    return range(min(n, rank * per), min(n, (rank + 1) * per))


def allreduce_grad(grad: torch.Tensor, group=None) -> torch.Tensor:
    """Sum a gradient tensor over the ranks of `group` in place (NCCL for CUDA tensors,
    gloo for CPU ones); a no-op outside torch.distributed."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def allreduce_table_grad(module: SigmaTableDenoiser, group=None) -> None:
    """Data-parallel step: sum the table gradient over the ranks (one all-reduce of
    sbsize*(sbsize//2+1) floats per step); pixel gradients stay local. Each rank's loss
    must be normalised by the global batch, so that the sum is the full-batch gradient."""
    if module.table.grad is not None:
        allreduce_grad(module.table.grad, group)
