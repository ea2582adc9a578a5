"""nf_dft_backward_device_static: the DFTTest backward with its scratch in the library's
fixed device buffer. Two calls in a row agree with nf_dft_backward_device (caller
scratch) on the same inputs, even after another plan's call has left different data in
the buffer; neither torch's allocator nor the device's free memory changes across a
call; calls whose scratch need exceeds the buffer are rejected with a clear message, and
invalid plans or plane counts get the same error as the caller-scratch form.
(Named to be collected last; it also passes alone in a fresh process.)"""
import ctypes

import numpy as np
import pytest

from neo_fft_b200 import _capi as C
from neo_fft_b200.plan import DFTConfig, Plan, SampleFormat, _plane
from tests.synth import noisy_patches

pytestmark = pytest.mark.gpu


def _planes(t, const):
    cls = C.NfConstPlane if const else C.NfPlane
    return (cls * t.shape[0])(*[_plane(t[i], const) for i in range(t.shape[0])])


def _backward_caller_scratch(torch, plan, x, g):
    n = x.shape[0]
    gx = torch.empty_like(x)
    gt = torch.empty(plan.bins, dtype=torch.float32, device=x.device)
    need = ctypes.c_size_t()
    assert plan._lib.nf_dft_backward_scratch_bytes(plan._h, n, ctypes.byref(need)) == 0
    # NaN bytes everywhere: a scratch word read before this call writes it would show
    scratch = torch.full((need.value,), 0xFF, dtype=torch.uint8, device=x.device)
    err = ctypes.create_string_buffer(256)
    st = plan._lib.nf_dft_backward_device(plan._h, _planes(x, True), _planes(g, True), _planes(gx, False), n,
                                          ctypes.c_void_p(gt.data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
                                          need.value, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                          err, 256)
    C.raise_for(st, err.value)
    return gx, gt


def _backward_static(torch, plan, x, g, gx, gt):
    err = ctypes.create_string_buffer(256)
    st = plan._lib.nf_dft_backward_device_static(plan._h, _planes(x, True), _planes(g, True), _planes(gx, False),
                                                 x.shape[0], ctypes.c_void_p(gt.data_ptr()),
                                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), err, 256)
    C.raise_for(st, err.value)


def test_static_scratch_backward_matches_caller_scratch(cuda):
    torch = cuda
    n, s = 16, 256
    plan = Plan(s, s, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0))
    noisy, clean = noisy_patches(n, s, 51)
    x = torch.from_numpy(noisy).cuda()
    g = torch.from_numpy(np.random.default_rng(52).standard_normal((n, s, s)).astype(np.float32)).cuda()
    ref_gx, ref_gt = _backward_caller_scratch(torch, plan, x, g)

    # Stale contents first: a call of another plan (other block size and overlap) on other
    # inputs fills the shared buffer with its own cover gradients and partials.
    other = Plan(192, 160, SampleFormat(32, True), DFTConfig(block=8, overlap=4, ftype=1, sigma=2.0))
    ox = torch.from_numpy(np.random.default_rng(53).random((3, 160, 192), dtype=np.float32)).cuda()
    ogx = torch.empty_like(ox)
    ogt = torch.empty(other.bins, dtype=torch.float32, device="cuda")
    _backward_static(torch, other, ox, ox, ogx, ogt)  # first call on this device: address lookup
    torch.cuda.synchronize()
    other.sync_status()

    gx = torch.empty_like(x)
    gt = torch.empty(plan.bins, dtype=torch.float32, device="cuda")
    for _ in range(2):
        gx.fill_(float("nan"))
        gt.fill_(float("nan"))
        torch.cuda.synchronize()
        alloc, reserved = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
        # whole-device free memory also counts other contexts on a shared GPU; torch's own
        # counters above are the exact check for this process
        free_before = torch.cuda.mem_get_info()[0]
        _backward_static(torch, plan, x, g, gx, gt)
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == alloc and torch.cuda.memory_reserved() == reserved
        assert torch.cuda.mem_get_info()[0] == free_before
        # deterministic kernels on identical inputs: the tolerance is zero
        assert torch.equal(gx, ref_gx) and torch.equal(gt, ref_gt)
    plan.sync_status()


def test_static_scratch_rejects_oversized_calls(cuda):
    torch = cuda
    lib = C.load()
    cap = lib.nf_dft_backward_static_capacity()
    assert cap == 16 << 20
    w, h, n = 1920, 1080, 4
    plan = Plan(w, h, SampleFormat(32, True), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0))
    need = ctypes.c_size_t()
    lib.nf_dft_backward_scratch_bytes(plan._h, n, ctypes.byref(need))
    assert need.value > cap
    x = torch.zeros((n, h, w), dtype=torch.float32, device="cuda")
    gx = torch.empty_like(x)
    gt = torch.empty(plan.bins, dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="above the 16777216-byte static buffer"):
        _backward_static(torch, plan, x, x, gx, gt)
    # an invalid call is told what is invalid, not that the buffer is too small
    many = torch.zeros((33, 8, 8), dtype=torch.float32, device="cuda")
    small = Plan(8, 8, SampleFormat(32, True), DFTConfig(block=8, overlap=4, ftype=0, sigma=4.0))
    sgt = torch.empty(small.bins, dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="1..32 planes"):
        _backward_static(torch, small, many, many, torch.empty_like(many), sgt)
    u16 = Plan(w, h, SampleFormat(16), DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0))
    with pytest.raises(ValueError, match="float DFTTest plan"):
        _backward_static(torch, u16, x, x, gx, gt)
