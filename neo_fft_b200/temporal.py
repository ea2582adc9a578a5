"""Host-side frame-slot logic of the temporal paths (what the plugin layer computes
before calling Plan::process_at):

  * temporal_blocks — DFTTest tmode=1 absolute lattice with endpoint clamping
    (src/algorithms/temporal_grid.hpp:5-40)
  * centred_slots   — DFTTest tmode=0 slots clamp(n-floor(T/2)+z, 0, N-1)
    (src/plugin/filter.hpp:446-452)
  * fft3d_slots     — FFT3D bt=2..5 window n-floor(bt/2)..n+floor((bt-1)/2), or the
    single-frame fallback at clip edges (src/plugin/filter.hpp:433-440)
"""
from __future__ import annotations


def validate_temporal(size: int, mode: int, overlap: int) -> None:
    if mode not in (0, 1):
        raise ValueError("DFTTest tmode outside 0..1")
    if not 1 <= size <= 15:
        raise ValueError("DFTTest tbsize outside 1..15")
    if mode == 0 and size % 2 != 1:
        raise ValueError("DFTTest centered tbsize must be odd")
    if mode == 1:
        if not 0 <= overlap < size:
            raise ValueError("DFTTest invalid tosize")
        if not (overlap <= size // 2 or size % (size - overlap) == 0):
            raise ValueError("DFTTest temporal heavy overlap requires divisible step")


def temporal_blocks(frame: int, length: int, size: int, overlap: int) -> list[dict]:
    """Covering temporal blocks of output `frame`: start, target slice and slots."""
    validate_temporal(size, 1, overlap)
    if not (length >= size and 0 <= frame < length):
        raise ValueError("invalid temporal clip/index")
    step = size - overlap
    anchor = -max(step, overlap)
    first = max(0, (frame - size - anchor) // step + 1)
    last = (frame - anchor) // step
    out = []
    for j in range(first, last + 1):
        start = anchor + j * step
        out.append({"start": start, "target": frame - start,
                    "slots": [min(max(start + z, 0), length - 1) for z in range(size)]})
    return out


def centred_slots(frame: int, length: int, size: int) -> list[int]:
    c = size // 2
    return [min(max(frame - c + j, 0), length - 1) for j in range(size)]


def fft3d_slots(frame: int, length: int, bt: int) -> list[int]:
    left, right = bt // 2, (bt - 1) // 2
    if bt <= 1 or frame < left or length - 1 - frame < right:
        return [frame]
    return list(range(frame - left, frame + right + 1))
