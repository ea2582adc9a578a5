"""Runs a few launches of one workload's dominant kernel, for profilers.

  python -m neo_fft_b200.profile_case --workload dft16 --launches 3

Workloads (one plane per launch, seeded synthetic content):
  dft16    DFTTest sbsize 16 / sosize 12, ftype 0, sigma 8 flat curve, u16 1920x1080
  dft16_batch the same configuration as one batched launch over --frames YUV420 frames
           (default 4: 4 x 1920x1080 + 8 x 960x540 planes)
  dft16_4k the same on a u16 3840x2160 plane (input+output larger than L2)
  fft3d32  FFT3D bw=bh=32, ow=oh=16, sigma 2, u8 640x360
  fft3d48  FFT3D bt=3 bw=bh=48, ow=oh=24, sigma 3, sharpen 0.3, u16 (10-bit) 3840x2160
  kalman32 FFT3D bt=0 (Kalman advance), bw=bh=32, float 1920x1080
  dft12t5  DFTTest tbsize 5 tmode 1, sbsize 12 / sosize 9, ftype 1, float 1920x1080
  clip12t5 DFTTest tbsize 5 tmode 1 sbsize 12 / sosize 9 ftype 1, float 1920x1080 clip of 10
           frames as one clip batch (volume spectra pass + slice strips) per launch
  clip48   FFT3D bt=3 48x48 ow=oh=24 sigma 3 sharpen 0.3, 1920x1080 YUV420P10 clip of 6
           frames as one clip batch (spectra pass + temporal strips) per launch
  adjoint16 differentiable DFTTest: 16 float 256x256 noisy patches, sbsize 16 / sosize 8,
           ftype 0, learnable table, MSE loss; one forward+backward per launch
"""
from __future__ import annotations

import argparse

import numpy as np


def _plane(h, w, dtype, lo, hi, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(lo, hi, (h, w))
    return v.astype(dtype)


def main():
    import torch

    from . import DFTConfig, FFT3DConfig, Plan, SampleFormat
    from .temporal import temporal_blocks

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="dft16")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--frames", type=int, default=4, help="frames of the dft16_batch workload")
    a = ap.parse_args()
    dev = torch.device("cuda", 0)
    wl = a.workload
    if wl in ("dft16", "dft16_4k"):
        w, h = (1920, 1080) if wl == "dft16" else (3840, 2160)
        plan = Plan(w, h, SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8]))
        srcs = [torch.from_numpy(_plane(h, w, np.uint16, 4096, 60000, 1)).to(dev)]
        targets = ()
    elif wl == "dft16_batch":
        from . import Batch
        cfg = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])
        luma, chroma = Plan(1920, 1080, SampleFormat(16), cfg), Plan(960, 540, SampleFormat(16), cfg)
        items = []
        for f in range(a.frames):
            for p, (w, h) in ((luma, (1920, 1080)), (chroma, (960, 540)), (chroma, (960, 540))):
                s_ = torch.from_numpy(_plane(h, w, np.uint16, 4096, 60000, f)).to(dev)
                items.append((p, s_, torch.empty_like(s_)))
        batch = Batch(items)
        for _ in range(a.launches):
            batch.launch()
        torch.cuda.synchronize()
        batch.sync_status()
        return
    elif wl == "fft3d32":
        w, h = 640, 360
        plan = Plan(w, h, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0))
        srcs = [torch.from_numpy(_plane(h, w, np.uint8, 16, 235, 1)).to(dev)]
        targets = ()
    elif wl == "fft3d48":
        w, h = 3840, 2160
        plan = Plan(w, h, SampleFormat(10), FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3))
        srcs = [torch.from_numpy(_plane(h, w, np.uint16, 64, 940, f)).to(dev) for f in range(3)]
        targets = ()
    elif wl == "kalman32":
        w, h = 1920, 1080
        plan = Plan(w, h, SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0))
        state = plan.initial_kalman()
        src = torch.from_numpy(_plane(h, w, np.float32, 0, 1, 1)).to(dev)
        for _ in range(a.launches):
            plan.advance_kalman(src, state)
        torch.cuda.synchronize()
        plan.sync_status()
        return
    elif wl == "dft12t5":
        w, h = 1920, 1080
        plan = Plan(w, h, SampleFormat(32, True), DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1,
                                                            ftype=1, sigma=8.0))
        clip = [torch.from_numpy(_plane(h, w, np.float32, 0, 1, f)).to(dev) for f in range(9)]
        blocks = temporal_blocks(4, 9, 5, 0)
        srcs = [clip[s] for b in blocks for s in b["slots"]]
        targets = [b["target"] for b in blocks]
    elif wl == "clip48":
        from . import ClipBatch
        cfg = FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3)
        pls = [Plan(1920, 1080, SampleFormat(10), cfg), Plan(960, 540, SampleFormat(10, chroma=True), cfg)]
        clips = []
        for p in range(3):
            pw, ph = (1920, 1080) if p == 0 else (960, 540)
            fr = [torch.from_numpy(_plane(ph, pw, np.uint16, 64, 940, 10 * p + f)).to(dev) for f in range(6)]
            clips.append((pls[min(p, 1)], fr, [torch.empty_like(x) for x in fr]))
        cb = ClipBatch(clips)
        for _ in range(a.launches):
            cb.launch()
        torch.cuda.synchronize()
        for p in pls:
            p.sync_status()
        return
    elif wl == "clip12t5":
        from . import ClipBatch
        cfg = DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1, sigma=8.0)
        p = Plan(1920, 1080, SampleFormat(32, True), cfg)
        fr = [torch.from_numpy(_plane(1080, 1920, np.float32, 0, 1, f)).to(dev) for f in range(10)]
        cb = ClipBatch([(p, fr, [torch.empty_like(x) for x in fr])])
        for _ in range(a.launches):
            cb.launch()
        torch.cuda.synchronize()
        p.sync_status()
        return
    elif wl == "adjoint16":
        import sys
        from pathlib import Path
        sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
        from tests.synth import noisy_patches

        from .autograd import SigmaTableDenoiser
        noisy, clean = noisy_patches(16, 256, 41)
        x0, cl = torch.from_numpy(noisy).to(dev), torch.from_numpy(clean).to(dev)
        m = SigmaTableDenoiser(256, 256, DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0))
        for _ in range(a.launches):
            x = x0.detach().requires_grad_()
            ((m(x) - cl) ** 2).mean().backward()
        torch.cuda.synchronize()
        m.plan.sync_status()
        return
    else:
        raise SystemExit(f"unknown workload {wl}")
    out = torch.empty_like(srcs[0])
    for _ in range(a.launches):
        plan.process_at(srcs, out, targets=targets)
    torch.cuda.synchronize()
    plan.sync_status()


if __name__ == "__main__":
    main()
