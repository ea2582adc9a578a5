"""Host-memory drop-in calls from several host threads (the host layer runs frames on
its own threads): each call runs on its thread's stream with its own device staging and
its own non-finite flag, so concurrent results equal serial ones and a non-finite input
fails only the call that carried it."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from neo_fft_b200 import NonFiniteError
from neo_fft_b200.plan import DFTConfig, FFT3DConfig, Plan, SampleFormat
from tests.synth import plane

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt,cfg", [
    (SampleFormat(32, True), DFTConfig(block=16, overlap=12, ftype=0, sigma=4.0)),
    (SampleFormat(16), FFT3DConfig(bw=16, bh=16, ow=8, oh=8, bt=3, sigma=600.0)),
], ids=["f32-dft16", "u16-fft3d-bt3"])
def test_threaded_host_calls_equal_serial(cuda, fmt, cfg):
    w, h = 160, 96
    p = Plan(w, h, fmt, cfg)
    T = p.temporal_size
    clips = [[plane(h, w, fmt.bits, fmt.floating, seed=(400, i, t)) for t in range(T)] for i in range(24)]
    serial = [p.process(c) for c in clips]
    with ThreadPoolExecutor(6) as pool:
        threaded = list(pool.map(p.process, clips))
    for a, b in zip(serial, threaded):
        assert np.array_equal(a, b)


def test_non_finite_fails_only_its_own_call(cuda):
    w, h = 128, 96
    fmt = SampleFormat(32, True)
    p = Plan(w, h, fmt, DFTConfig(block=16, overlap=12, ftype=0, sigma=4.0))
    planes = [plane(h, w, 32, True, seed=(401, i)) for i in range(16)]
    bad = 5
    planes[bad] = planes[bad].copy()
    planes[bad][40, 50] = np.nan

    def run(i):
        try:
            return p.process([planes[i]])
        except NonFiniteError:
            return None
    with ThreadPoolExecutor(4) as pool:
        out = list(pool.map(run, range(16)))
    for i, o in enumerate(out):
        if i == bad:
            assert o is None
        else:
            assert o is not None and np.array_equal(o, p.process([planes[i]]))
    p.sync_status()  # the plan's own flag is untouched by host-memory calls
