"""DFTTest sampled noise model (nlocation): the table built by nf_dft_noise_power from
gathered sample volumes equals the reference's DFTNoise bit for bit (CPU), and plans
publishing it filter exactly like the reference plan with the same model (GPU)."""
import ctypes

import numpy as np
import pytest

from neo_fft_b200 import _capi as C
from neo_fft_b200.plan import DFTConfig, DFTNoise, Plan, SampleFormat, gather_noise
from tests.synth import plane

CASES = [
    (SampleFormat(8), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, nlocation=[0, 0, 10, 20, 1, 0, 40, 60])),
    (SampleFormat(16), DFTConfig(block=12, overlap=6, tbsize=3, ftype=1, sigma=8.0, zmean=0, alpha=6.5,
                                 nlocation=[0, 0, 5, 5, 1, 0, 30, 50, 2, 0, 60, 10])),
    (SampleFormat(32, True), DFTConfig(block=8, overlap=4, mode=1, ftype=0, f0beta=0.5, sigma=3.0,
                                       nlocation=[2, 0, 0, 0])),
]
IDS = ["u8-b16", "u16-b12-t3", "f32-b8"]
W, H = 120, 96


def _frames(fmt, n=6):
    return [plane(H, W, fmt.bits, fmt.floating, seed=(99, 0, f)) for f in range(n)]


def _slices(fmt, cfg, frames):
    noise = DFTNoise(cfg)
    return noise, np.stack([np.stack([gather_noise(lambda f, p: frames[f], loc, z, cfg.block, fmt)
                                      for z in range(cfg.tbsize)]) for loc in noise.locations])


@pytest.mark.parametrize("fmt,cfg", CASES, ids=IDS)
def test_noise_model_matches_reference(ref, fmt, cfg):
    frames = _frames(fmt)
    noise, slices = _slices(fmt, cfg, frames)
    power = noise.prepare(lambda loc, z: slices[noise.locations.index(loc), z])
    exp = ref.RefPlan(W, H, fmt, cfg).prepare_noise(slices)
    assert power.dtype == np.float32 and np.array_equal(power, exp)


def test_noise_model_rejects_inactive_and_mismatched_inputs():
    lib = C.load()
    err = ctypes.create_string_buffer(256)
    c, keep = DFTConfig(ftype=2, nlocation=[0, 0, 0, 0]).to_c()
    out = np.zeros(16 * 9, np.float32)
    sl = np.zeros((1, 1, 16, 16), np.float32)
    assert lib.nf_dft_noise_power(ctypes.byref(c), ctypes.c_void_p(sl.ctypes.data), 1,
                                  ctypes.c_void_p(out.ctypes.data), out.size, err, 256) == 1
    assert b"inactive DFTTest sample model" in err.value
    c, keep = DFTConfig(nlocation=[0, 0, 0, 0, 1, 0, 0, 0]).to_c()
    assert lib.nf_dft_noise_power(ctypes.byref(c), ctypes.c_void_p(sl.ctypes.data), 1,
                                  ctypes.c_void_p(out.ctypes.data), out.size, err, 256) == 1
    assert b"slices differ from nlocation" in err.value


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,cfg", CASES, ids=IDS)
def test_plan_with_published_model_matches_reference(cuda, ref, fmt, cfg):
    frames = _frames(fmt)
    noise, slices = _slices(fmt, cfg, frames)
    p = Plan(W, H, fmt, cfg)
    assert p.model_state == 1
    T = cfg.tbsize
    srcs = [frames[j] for j in range(T)]
    with pytest.raises(ValueError, match="DFTTest sample model not initialized"):
        p.process(srcs)
    noise.prepare(lambda loc, z: slices[noise.locations.index(loc), z])
    noise.publish(p)
    assert p.model_state == 2
    got = p.process(srcs)
    rp = ref.RefPlan(W, H, fmt, cfg)
    rp.prepare_noise(slices)
    assert np.array_equal(got, rp.process(srcs))
