"""One long clip over several GPUs: contiguous output-frame ranges per rank, each rank
holding its range's source frames plus the read-only halo its windows reach, in its own
HBM. Output frames are independent functions of a bounded source window (the host
layer's frame selection, src/plugin/filter.hpp:266-305 and :433-452), so the ranges need
no exchange: every output frame is produced by exactly one rank from exactly the sources
the reference would use.

  * FFT3D bt 2..5: window n - bt//2 .. n + (bt-1)//2, or the frame alone at clip edges
    (temporal.fft3d_slots); the halo is bt//2 frames before the range and (bt-1)//2 after.
  * DFTTest tmode 0: slots clamp(n - T//2 + z, 0, N-1) (temporal.centred_slots).
  * DFTTest tmode 1: the slots of every covering temporal block, anchored on the whole
    clip's lattice (temporal.temporal_blocks), so a rank loads whole temporal blocks.
  * Single-frame plans (FFT3D bt 1 or -1, DFTTest tbsize 1): no halo.
  * FFT3D bt 0 (Kalman) is sequential in time and is not split by frames (a clip stays on
    one rank; several clips or planes spread over ranks instead).

`ClipShard` runs a rank's range: it uploads the sources it needs (host frames, or frames
already in this GPU's memory) and produces its outputs through the clip-batch form over
the range plus halo (FFT3D) or through one per-call filter per output frame with the
whole-clip window (DFTTest); the results equal the single-GPU clip bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass

from .temporal import centred_slots, fft3d_slots, temporal_blocks


@dataclass(frozen=True)
class Window:
    """What one output frame reads: source frames in slot order and, for DFTTest tmode 1,
    the target slice of each covering block."""
    sources: tuple
    targets: tuple = ()


def frame_ranges(n_frames: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, balanced [start, stop) output ranges, one per rank (some may be empty
    when there are more ranks than frames)."""
    if n_frames < 0 or world < 1:
        raise ValueError("invalid frame count or world size")
    base, extra = divmod(n_frames, world)
    out, start = [], 0
    for r in range(world):
        stop = start + base + (1 if r < extra else 0)
        out.append((start, stop))
        start = stop
    return out


def window(kind: str, n: int, length: int, size: int = 1, overlap: int = 0) -> Window:
    """The host layer's frame selection for output n of a clip of `length` frames.
    kind: "single", "fft3d" (size = bt), "dft0" (tmode 0, size = tbsize) or "dft1"
    (tmode 1, size = tbsize, overlap = tosize)."""
    if not 0 <= n < length:
        raise ValueError("frame outside clip")
    if kind == "single":
        return Window((n,))
    if kind == "fft3d":
        return Window(tuple(fft3d_slots(n, length, size)))
    if kind == "dft0":
        return Window(tuple(centred_slots(n, length, size)))
    if kind == "dft1":
        blocks = temporal_blocks(n, length, size, overlap)
        return Window(tuple(s for b in blocks for s in b["slots"]), tuple(b["target"] for b in blocks))
    raise ValueError(f"unknown window kind {kind}")


def plan_kind(plan) -> tuple[str, int, int]:
    """(kind, size, overlap) of a Plan (or anything with .config and .temporal_size) for
    `window`."""
    from .plan import FFT3DConfig
    c = plan.config
    if isinstance(c, FFT3DConfig):
        if c.bt == 0:
            raise ValueError("Kalman plans are sequential in time: keep a clip on one rank")
        t = plan.temporal_size
        return ("fft3d", t, 0) if t > 1 and not c.pshow else ("single", 1, 0)
    if c.tbsize == 1:
        return "single", 1, 0
    if c.temporal_mode == 1:
        return "dft1", c.tbsize, c.temporal_overlap
    return "dft0", c.tbsize, 0


def rank_sources(kind: str, rng: tuple[int, int], length: int, size: int = 1, overlap: int = 0) -> list[int]:
    """Sorted source frames a rank needs for its output range (range plus halo)."""
    need = set()
    for n in range(*rng):
        need.update(window(kind, n, length, size, overlap).sources)
    return sorted(need)


class ClipShard:
    """The outputs [start, stop) of one clip on this rank's GPU.

    plan: a Plan; frames: callable f -> source frame f (numpy array or CUDA tensor);
    length: frames in the whole clip. run() returns {frame: CUDA tensor output}."""

    def __init__(self, plan, frames, length: int, rng: tuple[int, int], device=None):
        import torch
        self.plan, self.length, self.rng = plan, length, rng
        self.kind, self.size, self.overlap = plan_kind(plan)
        self.dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.sources = rank_sources(self.kind, rng, length, self.size, self.overlap)
        self.local = {}
        for f in self.sources:  # host upload or device-to-device copy into this GPU's HBM
            x = frames(f)
            x = torch.from_numpy(x) if not isinstance(x, torch.Tensor) else x
            self.local[f] = x.to(self.dev, copy=True)

    def run(self) -> dict:
        import torch
        from .plan import ClipBatch
        start, stop = self.rng
        if start >= stop:
            return {}
        out = {}
        if self.kind == "fft3d":
            # the clip form over the range plus halo: interior outputs see the same windows
            # as in the whole clip, and a range that starts or ends at the clip's edge
            # falls back to the single frame exactly as the whole clip does
            lo, hi = self.sources[0], self.sources[-1]
            sub = [self.local[f] for f in range(lo, hi + 1)]
            dsts = [torch.empty_like(x) for x in sub]
            ClipBatch([(self.plan, sub, dsts)]).launch()
            out = {n: dsts[n - lo] for n in range(start, stop)}
        else:
            for n in range(start, stop):
                w = window(self.kind, n, self.length, self.size, self.overlap)
                dst = torch.empty_like(self.local[n])
                self.plan.process_at([self.local[s] for s in w.sources], dst, frame=n, targets=w.targets)
                out[n] = dst
        self.plan.sync_status()
        return out
