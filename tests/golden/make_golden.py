"""Regenerates the golden fixtures from the reference core compiled from source
(oracle/_ref). Run from the repository root: python tests/golden/make_golden.py

smoke.npz: inputs and reference outputs of the two smoke() cases
  dft   - DFTTest sbsize 16, sosize 12, ftype 0, sigma 8 (flat curve), u16 128x96
  fft3d - FFT3D bw=bh=32, ow=oh=16, sigma 2, u8 160x96
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from neo_fft_b200.plan import DFTConfig, FFT3DConfig, SampleFormat  # noqa: E402
from oracle import ref as R  # noqa: E402
from tests.synth import plane  # noqa: E402


def main():
    out = {}
    src = plane(96, 128, 16, False, seed=(2, 0, 0))
    out["dft_in"] = src
    out["dft_out"] = R.RefPlan(128, 96, SampleFormat(16),
                               DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])).process(src)
    src = plane(96, 160, 8, False, seed=(1, 0, 0), kind="gradient")
    out["fft3d_in"] = src
    out["fft3d_out"] = R.RefPlan(160, 96, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0)).process(src)
    np.savez_compressed(ROOT / "tests" / "golden" / "smoke.npz", **out)
    print("wrote smoke.npz")


if __name__ == "__main__":
    main()
