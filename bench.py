"""Benchmark: DFTTest (sbsize 16, sosize 12, ftype 0, sigma 8 with a flat sigma curve,
dither 0) over a 1920x1080 YUV420P16 clip of 60 frames — luma 1920x1080 and two
960x540 chroma planes per frame, synthetic seeded band-limited texture in
[4096, 60000] plus Gaussian noise sd 600.

A step is one pass of the per-plane pipeline over the whole clip (60 frames x 3
planes; ~746 MB of input and output per step, larger than the 126 MB L2, so no
flush is needed between steps). Mpx counts luma pixels per output frame.

`value` is the batched form (the whole clip in one persistent launch, replayed
from a CUDA graph); `plain` is the drop-in form (one launch per plane); `e2e`
takes every plane from pinned host memory and returns it there within each step,
through the streamed host form (HostBatch: device slots of a few frames, copies
overlapped with the batched launch).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --profile WORKLOAD [--launches N] [--frames F]   (a profiler's workload)

Multi-GPU (one process per GPU under torchrun): every rank filters its own clip
(weak scaling, no data-path collective); the time is the max over ranks.
--impl reference times the reference core's CPU implementation of the same
workload (compiled from its own sources, oracle/_ref) on all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, CW, CH, FRAMES = 1920, 1080, 960, 540, 60
HOST_CHUNK = 1  # frames per device slot of the streamed host form (4 slots)
# DRAM bytes of one batch launch over the 60-frame clip: ncu capture of a 16-frame launch of
# the same kernel (100.73 MB read + 60.34 MB written), scaled by the frames processed.
TRAFFIC_PER_LAUNCH = (100.73e6 + 60.34e6) * FRAMES / 16
METRIC = "Mpx/s per config on 1 B200 (plain vs batched/graph), fwd+bwd Mpx/s, vs host CPU"
WORKLOAD = "DFTTest tbsize=1 sbsize=16 sosize=12 ftype=0 sigma=8 flat curve, 1920x1080 YUV420P16, 60 frames"


def dft_config():
    from neo_fft_b200 import DFTConfig
    return DFTConfig(block=16, overlap=12, mode=1, ftype=0, sigma=8.0, tbsize=1, dither=0, slocation=[0, 8, 1, 8])


def make_plane(h, w, seed):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    t = gaussian_filter(rng.standard_normal((h, w)), 3.0)
    t = (t - t.min()) / max(np.ptp(t), 1e-12)
    v = 4096 + (60000 - 4096) * t + rng.standard_normal((h, w)) * 600
    return np.clip(np.round(v), 0, 65535).astype(np.uint16)


def make_clip(rank: int, frames: int):
    """Frames of (Y, U, V) planes; seeds [2, clip, frame]. Frames beyond a small
    distinct set reuse seeds to keep host generation short (content does not change
    the arithmetic per pixel)."""
    distinct = min(frames, 6)
    base = [(make_plane(H, W, [2, rank, f, 0]), make_plane(CH, CW, [2, rank, f, 1]), make_plane(CH, CW, [2, rank, f, 2]))
            for f in range(distinct)]
    return [base[f % distinct] for f in range(frames)]


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every 10 ms during the timed
    region through NVML (read-only queries), or through nvidia-smi where NVML cannot be
    loaded. The GPU is found by its PCI address, so CUDA_VISIBLE_DEVICES renumbering
    does not matter."""

    def __init__(self, index: int):
        self.index, self.samples, self._stop = index, [], threading.Event()
        try:  # NVML is opened before the timed region starts
            self._nv = self._nvml_handle()
        except Exception:
            self._nv = None
        self._t = threading.Thread(target=self._run, daemon=True)

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.index)
        try:
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _run(self):
        try:
            nv, h = self._nv
            bits = [getattr(nv, "nvmlClocksEventReason" + n, None) or getattr(nv, "nvmlClocksThrottleReason" + n)
                    for n in ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self._stop.is_set():
                r = reasons(h)
                self.samples.append([str(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), str(mx), "",
                                     *["Active" if r & b else "Not Active" for b in bits]])
                self._stop.wait(0.01)
            return
        except Exception:
            pass
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_baseline(gpu_out=None, frames_sample: int = 2):
    """The reference core (compiled from its own sources) on the host cores: frames
    run concurrently, one shared plan per plane size. With `gpu_out` (host copies of the
    GPU's outputs of the first frames of the same clip) it also checks them: against the
    reference's outputs of the timed sample, and against the binary64 re-evaluation
    (oracle/fp64_pipeline.py) on frame 0."""
    from neo_fft_b200 import SampleFormat
    from oracle import ref as R
    if not R.available():
        return None
    threads = os.cpu_count() or 1
    fmt = SampleFormat(16)
    luma = R.RefPlan(W, H, fmt, dft_config())
    chroma = R.RefPlan(CW, CH, fmt, dft_config())
    n = max(frames_sample, 2 * threads)  # about 15-20 s of CPU work over all threads
    clip = make_clip(0, n)
    t0 = time.perf_counter()
    ly = luma.process_many([[c[0]] for c in clip[:n]], threads)
    uv = chroma.process_many([[c[p]] for c in clip[:n] for p in (1, 2)], threads)
    dt = time.perf_counter() - t0
    line = {"value": n * W * H / dt / 1e6, "unit": "Mpx/s", "cores": threads, "kind": "reference",
            "sample": f"{n} frames (Y+U+V) of the same clip, frames concurrent on {threads} threads, "
                      "reference core built from source with its codelet FFT backend"}
    if gpu_out is not None:
        m = min(n, len(gpu_out))
        ref_out = [(ly[f], uv[2 * f], uv[2 * f + 1]) for f in range(m)]
        same = all(np.array_equal(gpu_out[f][p], ref_out[f][p]) for f in range(m) for p in range(3))
        from oracle.fp64_pipeline import FP64Plan
        fp64 = {}
        for p, (w, h) in enumerate([(W, H), (CW, CH), (CW, CH)]):
            fp = FP64Plan(w, h, fmt, dft_config())
            v = fp.process([clip[0][p]])
            d = np.abs(gpu_out[0][p].astype(np.int64) - fp.quantize(v).astype(np.int64))
            inside = (v > 0.5) & (v < fp.peak - 0.5)
            fp64["YUV"[p]] = {"max_steps": int(d.max()), "frac_off_by_one": float((d > 0).mean()),
                              "excess_over_half_step": float(np.abs(gpu_out[0][p] - v)[inside].max() - 0.5)}
        line["parity"] = {"vs_reference": {"frames": m, "planes": 3, "bit_identical": bool(same)},
                          "vs_fp64_frame0": fp64,
                          "fp64_note": "integer output vs the exactly rounded binary64 value: steps off, share of "
                                       "pixels one step off, and the binary32 error beyond the half step"}
    return line


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle library not built"}))
        return
    threads = os.cpu_count() or 1
    from neo_fft_b200 import SampleFormat
    fmt = SampleFormat(16)
    luma = R.RefPlan(W, H, fmt, dft_config())
    chroma = R.RefPlan(CW, CH, fmt, dft_config())
    n = FRAMES  # the same 60-frame clip as the GPU arm, every step
    clip = make_clip(0, n)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        luma.process_many([[c[0]] for c in clip], threads)
        chroma.process_many([[c[p]] for c in clip for p in (1, 2)], threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    dt = float(np.mean(times))
    value = n * W * H / dt / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpx/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "frames_per_step": n, "planes": "Y 1920x1080 + U,V 960x540 u16"},
        "cpu_baseline": {"value": value, "unit": "Mpx/s", "cores": threads, "kind": "reference",
                         "sample": f"the whole {n}-frame clip per step (Y+U+V), frames concurrent on {threads} host "
                                   "threads, reference core built from its own sources"},
        "e2e": {"value": value, "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import torch.distributed as dist

    from neo_fft_b200 import Batch, FrameServer, HostBatch, Plan, SampleFormat
    from neo_fft_b200 import _capi as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    fmt = SampleFormat(16)
    luma = Plan(W, H, fmt, dft_config())
    chroma = Plan(CW, CH, fmt, dft_config())
    lib = C.load()
    clip = make_clip(rank, FRAMES)
    # device-resident inputs and outputs
    d_in = [[torch.from_numpy(p).to(dev) for p in f] for f in clip]
    d_out = [[torch.empty_like(p) for p in f] for f in d_in]
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes_stream(stream)
    err = __import__("ctypes").create_string_buffer(256)
    plans = (luma, chroma, chroma)
    batch = Batch([(plans[p], d_in[f][p], d_out[f][p]) for f in range(FRAMES) for p in range(3)])

    def plane_call(plan, src, dst):
        srcs = (C.NfConstPlane * 1)(C.NfConstPlane(src.data_ptr(), src.shape[1], src.shape[0], src.stride(0) * 2))
        d = C.NfPlane(dst.data_ptr(), dst.shape[1], dst.shape[0], dst.stride(0) * 2)
        st = lib.nf_plan_process_device(plan._h, srcs, 1, None, 0, d, 0, 0, sptr, err, 256)
        if st:
            C.raise_for(st, err.value)

    def plain_step():
        for f in range(FRAMES):
            for p in range(3):
                plane_call(plans[p], d_in[f][p], d_out[f][p])

    def batch_step():
        batch.launch(graph=True)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    def timed(step_fn, steps, clocks=False):
        for _ in range(max(3, args.warmup)):
            step_fn()
        luma.sync_status()
        chroma.sync_status()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if clocks else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        for _ in range(steps):
            step_fn()
        e1.record(stream)
        barrier()
        if sampler:
            sampler.__exit__()
        ms = e0.elapsed_time(e1)
        luma.sync_status()
        chroma.sync_status()
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps, sampler

    # Plain drop-in: one launch per plane (180 per step).
    plain_ms, _ = timed(plain_step, args.steps)
    # Batched/graph: one persistent launch per step, replayed from a CUDA graph.
    ms_step, clocks = timed(batch_step, args.steps, clocks=True)
    value = world * FRAMES * W * H / (ms_step / 1e3) / 1e6
    plain_value = world * FRAMES * W * H / (plain_ms / 1e3) / 1e6

    # Roofline of the dominant kernel (the batch kernel: one launch per step, so its
    # average duration is the timed step); algorithmic bytes and flops per launch.
    gl, gc = luma.geometry, chroma.geometry
    plane_px = W * H + 2 * CW * CH
    alg_bytes = FRAMES * plane_px * 2 * 2           # each input sample read once + output written once
    blocks = FRAMES * (gl.x.count * gl.y.count + 2 * gc.x.count * gc.y.count)
    # per block: a forward and an inverse real 16x16 transform at 2.5 N log2 N flops each
    # (N = 256: 5120) plus 12 flops for each of the 144 bins' filter
    alg_flops = blocks * (2 * 2.5 * 256 * 8 + 144 * 12)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved_gbs = alg_bytes / (ms_step / 1e3) / 1e9
    fp32_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    achieved_tf = alg_flops / (ms_step / 1e3) / 1e12

    # End to end through the public API: pinned host frames copied in, the batch
    # replayed, outputs copied back to pinned host memory, every step.
    pin_in = [[torch.from_numpy(p).pin_memory() for p in f] for f in clip]
    pin_out = [[torch.empty(p.shape, dtype=torch.uint16).pin_memory() for p in f] for f in clip]

    host_batch = HostBatch(plans, frames_per_chunk=HOST_CHUNK, depth=4)

    def e2e_step():
        host_batch.process(pin_in, pin_out, wait=False)

    def serial_step():
        for f in range(FRAMES):
            for p in range(3):
                d_in[f][p].copy_(pin_in[f][p], non_blocking=True)
        batch.launch(graph=True)
        for f in range(FRAMES):
            for p in range(3):
                pin_out[f][p].copy_(d_out[f][p], non_blocking=True)

    e2e_ms, _ = timed(e2e_step, max(1, min(args.steps, 5)))
    serial_ms, _ = timed(serial_step, max(1, min(args.steps, 5)))
    plane_bytes = FRAMES * plane_px * 2
    e2e_value = world * FRAMES * W * H / (e2e_ms / 1e3) / 1e6
    serial_value = world * FRAMES * W * H / (serial_ms / 1e3) / 1e6
    # The host request layer: every output frame requested in order from a frame server
    # over the same pinned host frames (ranges of 4 frames, two ranges prefetched).
    server = FrameServer(plans, FRAMES, lambda f, p: pin_in[f][p].numpy(), range_frames=4)
    server_out = [[o.numpy() for o in f] for f in pin_out]
    for n in range(FRAMES):
        server.get(n, server_out[n])
    t0 = time.perf_counter()
    for n in range(FRAMES):
        server.get(n, server_out[n])
    server_value = FRAMES * W * H / (time.perf_counter() - t0) / 1e6
    del server
    # Same through the per-plane host-memory entry point (copies + launch + sync per plane).
    t0 = time.perf_counter()
    for f in range(FRAMES):
        luma.process([pin_in[f][0].numpy()], pin_out[f][0].numpy())
        chroma.process([pin_in[f][1].numpy()], pin_out[f][1].numpy())
        chroma.process([pin_in[f][2].numpy()], pin_out[f][2].numpy())
    host_plane_value = FRAMES * W * H / (time.perf_counter() - t0) / 1e6
    # The same drop-in calls from 8 host threads, each filtering its own frames (the host
    # layer's frame threads); each call synchronises only its thread's stream.
    from concurrent.futures import ThreadPoolExecutor

    def frame_job(f):
        luma.process([pin_in[f][0].numpy()], pin_out[f][0].numpy())
        chroma.process([pin_in[f][1].numpy()], pin_out[f][1].numpy())
        chroma.process([pin_in[f][2].numpy()], pin_out[f][2].numpy())
    with ThreadPoolExecutor(8) as pool:
        list(pool.map(frame_job, range(8)))  # warm-up: each thread's stream and staging
        t0 = time.perf_counter()
        list(pool.map(frame_job, range(FRAMES)))
        host_threads_value = FRAMES * W * H / (time.perf_counter() - t0) / 1e6

    train = differentiable_pass(args, dev, world)
    configs = other_configs(args, dev) if world == 1 else None
    cpu = None
    if rank == 0 and world == 1:
        batch.launch(graph=True)  # d_out as the batched form writes it
        torch.cuda.synchronize(dev)
        gpu_first = [[d_out[f][p].cpu().numpy() for p in range(3)] for f in range(min(FRAMES, 6))]
        cpu = cpu_baseline(gpu_first)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "Mpx/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "batched persistent launch replayed from a CUDA graph",
                   "frames_per_step": FRAMES, "planes": "Y 1920x1080 + U,V 960x540 u16",
                   "parallelism": f"clip-per-rank x{world}", "l2": "inputs larger than L2 (746 MB per step)"},
        "plain": {"value": plain_value, "unit": "Mpx/s", "ms_per_step": plain_ms,
                  "form": "one nf_plan_process_device launch per plane"},
        "e2e": {"value": e2e_value, "unit": "Mpx/s", "h2d_bytes_per_step": plane_bytes,
                "d2h_bytes_per_step": plane_bytes,
                "path": f"HostBatch.process (nf_host_batch_process): pinned host frames through {HOST_CHUNK}-frame "
                        "device slots, copies overlapped with the batched launch on separate streams",
                "serial_copies_value": serial_value,
                "frame_server_value": server_value,
                "per_plane_host_api_value": host_plane_value,
                "per_plane_host_api_8_threads_value": host_threads_value},
        "gpu_launches": args.steps,
        # The binding roof is the FP32 pipe (193 flops per algorithmic byte against a ridge of
        # ~11): achieved = algorithmic flops per launch / the launch's CUDA-event time; the
        # peak is nominal (no FP32 peak is measured on this pool). The HBM fraction and the
        # DRAM traffic of the same launch sit beside it.
        "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved_tf / fp32_peak, "alg_flops_per_launch": alg_flops,
                     "flops_per_block": "2 x 2.5 N log2 N (N = 256) + 144 bins x 12",
                     "peak_source": "148 SMs x 128 FP32 lanes x 2 x max SM clock (nominal)",
                     # the reference's binary32 rounding of every add and multiply rules out
                     # fused multiply-adds, so one flop per lane per clock is the ceiling
                     "peak_unfused": fp32_peak / 2, "frac_unfused": 2 * achieved_tf / fp32_peak,
                     "traffic": TRAFFIC_PER_LAUNCH,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 16-frame launch "
                                       "of the same kernel (161.1 MB), scaled by 60/16",
                     "kernel": "spatial_batch_kernel<16,16,u16,DFTTest> (whole clip per launch)", "launch_ms": ms_step,
                     "hbm": {"achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": achieved_gbs / hbm_peak,
                             "alg_bytes_per_launch": alg_bytes, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}},
        "clocks": clocks.summary() if clocks else None,
        "cpu_baseline": cpu,
        "fwd_bwd": train,
        "other_configs": configs,
    }
    print(json.dumps(line))


def differentiable_pass(args, dev, world=1):
    """Differentiable DFTTest: 16 float32 256x256 noisy patches, sbsize 16 / sosize 8, ftype 0,
    learnable 16x9 table; loss = MSE to the clean patches. Times the forward alone and
    forward+backward (gradients w.r.t. pixels and table) with CUDA events around each
    step and the L2 flushed (a 256 MB write) before every step."""
    import torch

    from neo_fft_b200 import DFTConfig
    from neo_fft_b200.autograd import SigmaTableDenoiser, allreduce_table_grad
    sys.path.insert(0, str(ROOT))
    from tests.synth import noisy_patches
    n, s = 16, 256
    noisy, clean = noisy_patches(n, s, 41)
    x0 = torch.from_numpy(noisy).to(dev)
    cl = torch.from_numpy(clean).to(dev)
    m = SigmaTableDenoiser(s, s, DFTConfig(block=16, overlap=8, ftype=0, sigma=4.0))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def fwd():
        with torch.no_grad():
            m(x0)

    def fwd_bwd():
        x = x0.detach().requires_grad_()
        m.table.grad = None
        ((m(x) - cl) ** 2).mean().backward()
        if world > 1:  # data-parallel step: one all-reduce of the 144-float table gradient
            allreduce_table_grad(m)

    def measure(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        total = 0.0
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            total += e0.elapsed_time(e1)
        m.plan.sync_status()
        return total / steps

    steps = max(5, args.steps)
    f_ms, fb_ms = measure(fwd, steps), measure(fwd_bwd, steps)
    px = n * s * s

    # The same training step captured once into a CUDA graph (static input buffer),
    # replayed per step: removes the host launch gaps between the small kernels.
    static_x = x0.detach().clone().requires_grad_()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(3):
            m.table.grad = None
            static_x.grad = None
            ((m(static_x) - cl) ** 2).mean().backward()
    torch.cuda.current_stream(dev).wait_stream(side)
    m.table.grad = None
    static_x.grad = None
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="thread_local"):
        ((m(static_x) - cl) ** 2).mean().backward()
    g_ms = measure(graph.replay, steps)
    del graph
    return {"value": px / (fb_ms / 1e3) / 1e6, "unit": "Mpx/s", "ms_per_step": fb_ms,
            "forward_value": px / (f_ms / 1e3) / 1e6, "forward_ms": f_ms, "ratio_to_forward": f_ms / fb_ms,
            "graph_value": px / (g_ms / 1e3) / 1e6, "graph_ms": g_ms, "graph_ratio_to_forward": f_ms / g_ms,
            "workload": "16 float32 256x256 patches, sbsize 16 / sosize 8, ftype 0, learnable 16x9 table, "
                        "MSE loss; gradients w.r.t. pixels and table (autograd over the C ABI adjoint kernels)",
            "l2": "flushed before every step (256 MB write)"}


def _texture(h, w, seed, lo, hi, noise_sd, dtype, peak=None):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    t = gaussian_filter(rng.standard_normal((h, w)), 3.0)
    t = lo + (hi - lo) * (t - t.min()) / max(np.ptp(t), 1e-12) + rng.standard_normal((h, w)) * noise_sd
    if peak is not None:
        t = np.clip(np.round(t), 0, peak)
    return t.astype(dtype)


def drift_base(h, w, seed, lo, hi, dev, sd_px=3.0):
    """A seeded band-limited texture in [lo, hi], wider than the frames cut from it, on the device."""
    import torch
    sys.path.insert(0, str(ROOT))
    from tests.synth import textured
    return torch.from_numpy(textured(h + 8, w + 400, seed, lo, hi, sd_px)).to(dev, torch.float32)


def drift_frames(base, n, seed, noise_sd, peak, dev, step=None):
    """n frames cut from `base` drifting right by 1-3 px per frame (or `step` px), bilinear
    between integer shifts, plus seeded Gaussian noise; rounded and clipped to [0, peak]
    as uint16 when peak is given, float32 otherwise. Generated on the device."""
    import torch
    g = torch.Generator(device=dev).manual_seed(int(np.random.default_rng(seed).integers(1 << 62)))
    rng = np.random.default_rng(seed)
    H, Wb = base.shape
    h, w = H - 8, Wb - 400
    frames, pos = [], float(rng.uniform(0, 16))
    for _ in range(n):
        i, frac = int(pos), pos - int(pos)
        v = (1 - frac) * base[4:4 + h, i:i + w] + frac * base[4:4 + h, i + 1:i + 1 + w]
        v = v + torch.randn((h, w), generator=g, device=dev) * noise_sd
        if peak is not None:
            v = v.round().clamp(0, peak).to(torch.int32).to(torch.uint16)
        frames.append(v.contiguous())
        pos += float(rng.uniform(1, 3)) if step is None else step
        if pos > 390:
            pos -= 380
    return frames


def _event_timer(dev, flush):
    import torch

    def measure(fn, steps, warmup):
        for _ in range(max(3, warmup)):
            fn()
        total = 0.0
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            total += e0.elapsed_time(e1)
        return total / steps
    return measure


def other_configs(args, dev):
    """The remaining configurations, each timed with CUDA events per step and the L2
    flushed (256 MB write) before every step. Mpx counts luma pixels per output frame."""
    import torch

    from neo_fft_b200 import Batch, ClipBatch, DFTConfig, FFT3DConfig, Plan, SampleFormat
    from neo_fft_b200.temporal import temporal_blocks
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    measure = _event_timer(dev, flush)
    steps = max(3, min(args.steps, 10))
    out = {}

    # A: FFT3D bt=1, 640x360 GRAY8, 24 frames, 32x32 blocks, overlap 16, sigma 2.
    w, h, n = 640, 360, 24
    plan = Plan(w, h, SampleFormat(8), FFT3DConfig(bw=32, bh=32, ow=16, oh=16, sigma=2.0))
    frames = [torch.from_numpy(_texture(h, w, [1, 0, f], 16, 235, 5, np.uint8, 255)).to(dev) for f in range(n)]
    outs = [torch.empty_like(f) for f in frames]
    batch = Batch([(plan, frames[f], outs[f]) for f in range(n)])
    plain_ms = measure(lambda: [plan.process_at([frames[f]], outs[f]) for f in range(n)], steps, args.warmup)
    batch_ms = measure(lambda: batch.launch(graph=True), steps, args.warmup)
    plan.sync_status()
    out["A"] = {"workload": "FFT3D bt=1 32x32 ow=oh=16 sigma 2, 640x360 GRAY8, 24 frames",
                "plain": n * w * h / (plain_ms / 1e3) / 1e6, "batched": n * w * h / (batch_ms / 1e3) / 1e6,
                "unit": "Mpx/s", "plain_ms": plain_ms, "batched_ms": batch_ms}
    del batch, frames, outs

    # C: FFT3D bt=3 48x48 ow=oh=24 sigma 3 sharpen 0.3 on YUV420P10 clips of 120 frames
    # drifting 1-3 px per frame. Batched, as stated: 32 clips (8 each of 3840x2160,
    # 1920x1080, 1280x720, 720x480) in one clip-batch launch replayed from a CUDA graph,
    # every output frame of every clip per step. Plain: one clip of each size through the
    # per-call drop-in (one two-pass call per output frame and plane).
    cfg = FFT3DConfig(bw=48, bh=48, ow=24, oh=24, bt=3, sigma=3.0, sharpen=0.3)
    sizes = [(3840, 2160), (1920, 1080), (1280, 720), (720, 480)]
    nf, per_size = 120, 8
    plans = {}
    for (w, h) in sizes:
        plans[(w, h)] = [Plan(w, h, SampleFormat(10), cfg), Plan(w // 2, h // 2, SampleFormat(10, chroma=True), cfg)]
    clips = []  # (size, [planes][frames] device tensors, outputs)
    for si, (w, h) in enumerate(sizes):
        bases = [drift_base(h >> (p > 0), w >> (p > 0), [3, si, p], 64, 940 if p == 0 else 960, dev)
                 for p in range(3)]
        for c in range(per_size):
            fr = [drift_frames(bases[p], nf, [3, si, c, p], 8.0, 1023, dev) for p in range(3)]
            clips.append(((w, h), fr, [[torch.empty_like(x) for x in fp] for fp in [fr[0], fr[1], fr[2]]]))
        del bases
    px_all = sum(nf * w * h for (w, h), _, _ in clips)
    cb = ClipBatch([(plans[sz][min(p, 1)], fr[p], outs[p]) for sz, fr, outs in clips for p in range(3)])
    cb_ms = measure(lambda: cb.launch(graph=True), 2, 1)
    del cb
    plain_clips = [clips[i * per_size] for i in range(len(sizes))]

    def c_plain():
        for sz, fr, outs in plain_clips:
            for t in range(nf):
                for p in range(3):
                    srcs = [fr[p][t]] if t in (0, nf - 1) else [fr[p][t - 1], fr[p][t], fr[p][t + 1]]
                    plans[sz][min(p, 1)].process_at(srcs, outs[p][t])
    c_ms = measure(c_plain, 2, 1)
    px_plain = sum(nf * w * h for (w, h), _, _ in plain_clips)
    for pl in plans.values():
        for p in pl:
            p.sync_status()
    out["C"] = {"workload": "FFT3D bt=3 48x48 ow=oh=24 sigma 3 sharpen 0.3, YUV420P10 clips of 120 frames drifting "
                            "1-3 px/frame + noise sd 8",
                "batched": px_all / (cb_ms / 1e3) / 1e6, "batched_ms": cb_ms,
                "batched_form": "32 clips (8 each of 3840x2160, 1920x1080, 1280x720, 720x480), all 120 output "
                                "frames of every clip per step: one clip-batch launch (spectra once per frame, "
                                "temporal strips) replayed from a CUDA graph",
                "plain": px_plain / (c_ms / 1e3) / 1e6, "plain_ms": c_ms,
                "plain_form": "one clip of each size, 120 output frames x 3 planes, one per-call two-pass filter each",
                "unit": "Mpx/s", "steps": 2, "warmup": 1, "l2": "inputs larger than L2"}
    del clips, plain_clips
    torch.cuda.empty_cache()

    # B at 4K: DFTTest 16/12 ftype 0 flat curve on a 3840x2160 YUV420P10 clip of 30 frames.
    W4, H4, n4 = 3840, 2160, 30
    dcfg = DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8])
    p4 = [Plan(W4, H4, SampleFormat(10), dcfg), Plan(W4 // 2, H4 // 2, SampleFormat(10, chroma=True), dcfg)]
    bases = [drift_base(H4 >> (p > 0), W4 >> (p > 0), [2, 4, p], 64, 940, dev) for p in range(3)]
    fr = [drift_frames(bases[p], n4, [2, 4, 0, p], 8.0, 1023, dev) for p in range(3)]
    del bases
    o4 = [[torch.empty_like(x) for x in fp] for fp in fr]
    b4 = Batch([(p4[min(p, 1)], fr[p][f], o4[p][f]) for f in range(n4) for p in range(3)])
    b4_ms = measure(lambda: b4.launch(graph=True), steps, args.warmup)
    b4p_ms = measure(lambda: [p4[min(p, 1)].process_at([fr[p][f]], o4[p][f]) for f in range(n4) for p in range(3)],
                     steps, args.warmup)
    for p in p4:
        p.sync_status()
    out["B4K"] = {"workload": "DFTTest tbsize=1 16/12 ftype 0 sigma 8 flat curve, 3840x2160 YUV420P10, 30 frames",
                  "batched": n4 * W4 * H4 / (b4_ms / 1e3) / 1e6, "batched_ms": b4_ms,
                  "plain": n4 * W4 * H4 / (b4p_ms / 1e3) / 1e6, "plain_ms": b4p_ms, "unit": "Mpx/s"}
    del b4, fr, o4

    # D1: FFT3D bt=0 Kalman 32x32 sigma 2.5 kratio 2 over 240 sequential distinct 1920x1080
    # float frames (slowly advected texture + noise sd 0.02): advance + render per frame,
    # state resident in HBM; the binary64-variance mode and the binary32 mode.
    w, h, n = 1920, 1080, 240
    kp = Plan(w, h, SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0))
    kbase = drift_base(h, w, [4, 0, 0], 0.0, 1.0, dev, sd_px=6.0)
    kf = drift_frames(kbase, n, [4, 0, 0, 1], 0.02, None, dev, step=0.3)
    del kbase
    kout = torch.empty_like(kf[0])
    d1 = {}
    for mode, fp64 in (("binary64_variance", True), ("binary32", False)):
        state = kp.initial_kalman(fp64_variance=fp64)

        def seq():
            for f in range(n):
                kp.advance_kalman(kf[f], state)
                kp.render_kalman(kf[f], kout, state)

        def seq_step():
            for f in range(n):
                kp.step_kalman(kf[f], kout, state)
        ms = measure(seq, max(2, min(steps, 3)), 1)
        ms_step = measure(seq_step, max(2, min(steps, 3)), 1)
        d1[mode] = {"plain": n * w * h / (ms / 1e3) / 1e6, "plain_ms": ms,
                    "step": n * w * h / (ms_step / 1e3) / 1e6, "step_ms": ms_step}
        del state
    kp.sync_status()
    out["D1"] = {"workload": "FFT3D bt=0 Kalman 32x32 sigma 2.5 kratio 2, 240 sequential distinct 1920x1080 float32 "
                             "frames", "unit": "Mpx/s", **d1,
                 "plain": d1["binary64_variance"]["plain"], "plain_ms": d1["binary64_variance"]["plain_ms"],
                 "step": d1["binary64_variance"]["step"], "step_ms": d1["binary64_variance"]["step_ms"],
                 "form": "binary64-variance state (the figures under plain and step; binary32 beside them); plain = "
                         "nf_kalman_advance_device + nf_kalman_render_device per frame, step = nf_kalman_step_device "
                         "per frame (one pass over the blocks, then the ordered overlap-add)"}
    del kf
    torch.cuda.empty_cache()

    # D2: DFTTest tbsize 5 tmode 1 (tosize 0), sbsize 12 sosize 9 ftype 1 sigma 8,
    # 1920x1080 float32; 8 output frames of a 12-frame clip.
    nclip, nout = 12, 8
    dp = Plan(w, h, SampleFormat(32, True), DFTConfig(block=12, overlap=9, tbsize=5, temporal_mode=1, ftype=1,
                                                      sigma=8.0))
    df = [torch.from_numpy(_texture(h, w, [4, 0, f], 0, 1, 0.02, np.float32)).to(dev) for f in range(nclip)]
    dout = torch.empty_like(df[0])
    jobs = []
    for t in range(2, 2 + nout):
        blocks = temporal_blocks(t, nclip, 5, 0)
        jobs.append(([df[s] for b in blocks for s in b["slots"]], [b["target"] for b in blocks]))
    d2_ms = measure(lambda: [dp.process_at(srcs, dout, targets=tg) for srcs, tg in jobs], steps, args.warmup)
    douts = [torch.empty_like(f) for f in df]
    cb = ClipBatch([(dp, df, douts)])
    d2b_ms = measure(lambda: cb.launch(graph=True), steps, args.warmup)
    dp.sync_status()
    del cb
    out["D2"] = {"workload": "DFTTest tbsize 5 tmode 1 sbsize 12 sosize 9 ftype 1 sigma 8, 1920x1080 float32, "
                             "12-frame clip", "plain": nout * w * h / (d2_ms / 1e3) / 1e6, "plain_ms": d2_ms,
                 "plain_form": "8 output frames, one per-call two-pass filter (volume slices, slice strip) per frame",
                 "batched": nclip * w * h / (d2b_ms / 1e3) / 1e6, "batched_ms": d2b_ms,
                 "batched_form": "all 12 output frames: clip batch (each temporal block filtered once, slice "
                                 "strips), graph", "unit": "Mpx/s"}
    return out


def _profile_plane(h, w, dtype, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (h, w)).astype(dtype)


def run_profile(a):
    """A few launches of one workload's dominant kernel, for ncu (`--profile <workload>
    --launches N`); prints nothing and times nothing.

    Workloads (one plane per launch, seeded synthetic content):
      dft16    DFTTest sbsize 16 / sosize 12, ftype 0, sigma 8 flat curve, u16 1920x1080
      dft16_batch the same configuration as one batched launch over --frames YUV420 frames
               (default 4: 4 x 1920x1080 + 8 x 960x540 planes)
      dft16_4k the same on a u16 3840x2160 plane (input+output larger than L2)
      fft3d32  FFT3D bw=bh=32, ow=oh=16, sigma 2, u8 640x360
      fft3d48  FFT3D bt=3 bw=bh=48, ow=oh=24, sigma 3, sharpen 0.3, u16 (10-bit) 3840x2160
      kalman32 FFT3D bt=0 (Kalman advance and render per launch), bw=bh=32, float 1920x1080
      kalman32_step the same as one Kalman step per launch (advance with the render's
               inverse transforms, then the ordered overlap-add)
      dft12t5  DFTTest tbsize 5 tmode 1, sbsize 12 / sosize 9, ftype 1, float 1920x1080
      clip12t5 DFTTest tbsize 5 tmode 1 sbsize 12 / sosize 9 ftype 1, float 1920x1080 clip of 10
               frames as one clip batch (volume spectra pass + slice strips) per launch
      clip48   FFT3D bt=3 48x48 ow=oh=24 sigma 3 sharpen 0.3, 1920x1080 YUV420P10 clip of 6
               frames as one clip batch (spectra pass + temporal strips) per launch
      adjoint16 differentiable DFTTest: 16 float 256x256 noisy patches, sbsize 16 / sosize 8,
               ftype 0, learnable table, MSE loss; one forward+backward per launch
    """
    import torch

    from neo_fft_b200 import DFTConfig, FFT3DConfig, Plan, SampleFormat
    from neo_fft_b200.temporal import temporal_blocks
    _plane = _profile_plane
    dev = torch.device("cuda", 0)
    wl = a.profile
    if wl in ("dft16", "dft16_4k"):
        w, h = (1920, 1080) if wl == "dft16" else (3840, 2160)
        plan = Plan(w, h, SampleFormat(16), DFTConfig(block=16, overlap=12, ftype=0, sigma=8.0, slocation=[0, 8, 1, 8]))
        srcs = [torch.from_numpy(_plane(h, w, np.uint16, 4096, 60000, 1)).to(dev)]
        targets = ()
    elif wl == "dft16_batch":
        from neo_fft_b200 import Batch
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
    elif wl in ("kalman32", "kalman32_step"):
        w, h = 1920, 1080
        plan = Plan(w, h, SampleFormat(32, True), FFT3DConfig(bw=32, bh=32, bt=0, sigma=2.5, kratio=2.0))
        state = plan.initial_kalman()
        src = torch.from_numpy(_plane(h, w, np.float32, 0, 1, 1)).to(dev)
        out = torch.empty_like(src)
        for _ in range(a.launches):
            if wl == "kalman32_step":
                plan.step_kalman(src, out, state)
            else:
                plan.advance_kalman(src, state)
                plan.render_kalman(src, out, state)
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
        from neo_fft_b200 import ClipBatch
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
        from neo_fft_b200 import ClipBatch
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
        from tests.synth import noisy_patches

        from neo_fft_b200.autograd import SigmaTableDenoiser
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




def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def spawn_ranks(args) -> int:
    """`--gpus N` outside a launcher: run N ranks (one process per GPU) under
    torch.distributed.run on this node and return its exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile", default=None, metavar="WORKLOAD",
                    help="run --launches launches of one workload's dominant kernel for a profiler")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--frames", type=int, default=4, help="frames of the dft16_batch profile workload")
    args = ap.parse_args()
    world = os.environ.get("WORLD_SIZE")
    if world is None and args.gpus > 1 and not args.profile:
        sys.exit(spawn_ranks(args))
    if world is not None and int(world) != args.gpus:
        sys.exit(f"--gpus {args.gpus} but the launcher started WORLD_SIZE={world} ranks")
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
