"""Kalman checkpoints and bounded-warmup seeks (Python mirror of
include/neo_fft_b200/checkpoints.hpp).

KalmanCheckpoints keeps up to four snapshots of per-plane device states with the
observable policy of the reference's runtime::Checkpoints (src/runtime/checkpoints.hpp:32-79);
KalmanSeek applies the host layer's random-access rule (src/plugin/filter.hpp:152-250) on
top of Plan's Kalman calls.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field


@dataclass
class KalmanCheckpoint:
    frame: int = 0
    planes: list = field(default_factory=lambda: [None] * 4)

    def nbytes(self) -> int:
        return 64 + sum(p.nbytes for p in self.planes if p is not None)

    def clone(self) -> "KalmanCheckpoint":
        return KalmanCheckpoint(self.frame, [p.clone() if p is not None else None for p in self.planes])


class KalmanCheckpoints:
    """At most four snapshots; acquire(frame, earliest) leases the latest snapshot in
    [earliest, frame]; publish() ignores frame < 1 and frames already held, then evicts
    least-recently used snapshots until the new one fits. Default budget 64 MiB that
    always retains one snapshot; an explicit budget is hard.

    Mirror of SnapshotShelf (include/neo_fft_b200/snapshot_shelf.hpp): a dict of frame ->
    (checkpoint, bytes, stamp), where every hit and every store takes the next value of a
    use counter and the smallest stamp is the least recently used."""

    SLOTS = 4

    def __init__(self, budget: int | None = None):
        self._budget = 64 << 20 if budget is None else int(budget)
        self._keep_oversized = budget is None
        self._held: dict[int, list] = {}  # frame -> [checkpoint, bytes, stamp]
        self._clock = 0
        self._lock = threading.Lock()

    def _stamp(self) -> int:
        self._clock += 1
        return self._clock

    def acquire(self, frame: int, earliest: int = 0):
        with self._lock:
            inside = [f for f in self._held if earliest <= f <= frame]
            if not inside:
                return None
            entry = self._held[max(inside)]
            entry[2] = self._stamp()
            return entry[0]

    def publish(self, cp: KalmanCheckpoint | None) -> None:
        if cp is None or cp.frame < 1:
            return
        size = cp.nbytes()
        cap = size if self._keep_oversized and size > self._budget else self._budget
        if size > cap:
            return
        with self._lock:
            if cp.frame in self._held:  # the snapshot already held for this frame stays
                self._held[cp.frame][2] = self._stamp()
                return
            while len(self._held) >= self.SLOTS or sum(e[1] for e in self._held.values()) + size > cap:
                lru = min(self._held, key=lambda f: self._held[f][2])
                del self._held[lru]
            self._held[cp.frame] = [cp, size, self._stamp()]

    def frames(self) -> list[int]:
        with self._lock:
            return sorted(self._held)

    def nbytes(self) -> int:
        with self._lock:
            return sum(e[1] for e in self._held.values())


class KalmanSeek:
    """Random-access Kalman frames over up to four plane plans (None = plane not
    filtered). frame(n, get_source, dsts) renders output frame n into dsts[p]:
    frame 0 passes through; otherwise the latest snapshot not older than
    n - warmup - 1 is continued, or the initial state is advanced over frames
    n - warmup .. n (1 .. n when n <= warmup); the new state is published."""

    def __init__(self, plans, warmup: int = 8, checkpoints: KalmanCheckpoints | None = None):
        self.plans = list(plans) + [None] * (4 - len(plans))
        self.warmup = warmup
        self.checkpoints = checkpoints if checkpoints is not None else KalmanCheckpoints()

    def frame(self, n: int, get_source, dsts) -> int:
        """get_source(f, p) -> device plane of source frame f, plane p. Returns the number
        of frames advanced (the replay length)."""
        def render(state):
            for p, plan in enumerate(self.plans):
                if p >= len(dsts) or dsts[p] is None:
                    continue
                src = get_source(n, p)
                if plan is None or state is None:
                    dsts[p].copy_(src)
                else:
                    plan.render_kalman(src, dsts[p], state.planes[p])
        if n == 0:
            render(None)
            return 0
        earliest = n - self.warmup - 1 if n > self.warmup else 0
        start = self.checkpoints.acquire(n, earliest)
        replay_start = start.frame if start is not None else earliest
        current = None
        steps = 0
        if replay_start < n:
            if start is not None:
                current = start.clone()
            else:
                current = KalmanCheckpoint(0, [p.initial_kalman() if p is not None else None for p in self.plans])
            for f in range(replay_start + 1, n + 1):
                for p, plan in enumerate(self.plans):
                    if plan is not None:
                        plan.advance_kalman(get_source(f, p), current.planes[p])
                current.frame = f
                steps += 1
        render(current if current is not None else start)
        if current is not None:
            self.checkpoints.publish(current)
        return steps
