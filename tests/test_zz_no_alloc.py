"""nf_dft_backward_device_static: the DFTTest backward with its scratch in the library's
fixed device buffer. Two calls in a row agree with nf_dft_backward_device (caller
scratch) on the same inputs, device free memory does not change across a call, and
calls whose scratch need exceeds the buffer are rejected with a clear message.
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
    scratch = torch.empty(need.value, dtype=torch.uint8, device=x.device)
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

    gx = torch.empty_like(x)
    gt = torch.empty(plan.bins, dtype=torch.float32, device="cuda")
    _backward_static(torch, plan, x, g, gx, gt)  # first call on this device: address lookup
    torch.cuda.synchronize()
    for _ in range(2):
        gx.fill_(float("nan"))
        gt.fill_(float("nan"))
        free_before = torch.cuda.mem_get_info()[0]
        _backward_static(torch, plan, x, g, gx, gt)
        torch.cuda.synchronize()
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
