"""neo_fft_b200 — B200 (sm_100a) implementation of neo-fft's per-plane spectral pipeline.

The public surface mirrors the reference core's `Plan` API; see `plan.py`.
"""
from .plan import (ROI, Axis, Batch, ClipBatch, DFTConfig, DFTNoise, FFT3DConfig, FrameServer, Geometry, HostBatch, KalmanState, Plan, SampleFormat,  # noqa: F401
                   kernel_info)
from ._capi import DeviceError, NonFiniteError  # noqa: F401
