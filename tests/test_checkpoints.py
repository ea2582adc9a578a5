"""Kalman checkpoint policy (neo_fft_b200/checkpoints.py, mirrored by
include/neo_fft_b200/checkpoints.hpp) and the host layer's bounded-warmup seek rule,
with fake states on the CPU; tests/test_gpu_checkpoints.py runs them on device states."""
import pytest

from neo_fft_b200.checkpoints import KalmanCheckpoint, KalmanCheckpoints, KalmanSeek


class FakeState:
    def __init__(self, nbytes=1000, history=()):
        self.nbytes, self.history = nbytes, list(history)

    def clone(self):
        return FakeState(self.nbytes, self.history)


def cp(frame, nbytes=1000):
    return KalmanCheckpoint(frame, [FakeState(nbytes), None, None, None])


def test_acquire_takes_latest_snapshot_in_window():
    c = KalmanCheckpoints()
    for f in (3, 9, 6):
        c.publish(cp(f))
    assert c.acquire(8).frame == 6
    assert c.acquire(20).frame == 9
    assert c.acquire(8, earliest=7) is None
    assert c.acquire(2) is None


def test_publish_ignores_frame_zero_and_keeps_first_snapshot_of_a_frame():
    c = KalmanCheckpoints()
    c.publish(cp(0))
    assert c.frames() == []
    first = cp(4)
    c.publish(first)
    c.publish(cp(4))
    assert c.acquire(4) is first


def test_four_slots_least_recently_used_evicted():
    c = KalmanCheckpoints()
    for f in (1, 2, 3, 4):
        c.publish(cp(f))
    c.acquire(1)  # touch the oldest
    c.publish(cp(5))
    assert c.frames() == [1, 3, 4, 5]


def test_explicit_budget_is_hard_and_default_retains_one():
    big = 40 << 20
    c = KalmanCheckpoints(budget=2 * big + (1 << 20))
    for f in (1, 2, 3):
        c.publish(cp(f, big))
    assert c.frames() == [2, 3]
    hard = KalmanCheckpoints(budget=1 << 20)
    hard.publish(cp(1, big))
    assert hard.frames() == []
    default = KalmanCheckpoints()
    default.publish(cp(1, 100 << 20))  # larger than 64 MiB: still kept (retain one)
    default.publish(cp(2, 100 << 20))
    assert default.frames() == [2]


class FakePlan:
    def initial_kalman(self):
        return FakeState()

    def advance_kalman(self, src, state):
        state.history.append(src)

    def render_kalman(self, src, dst, state):
        dst.append((src, list(state.history)))


class Sink(list):
    def copy_(self, src):
        self.append((src, None))


@pytest.mark.parametrize("warmup", [4, 8])
def test_seek_replays_bounded_warmup(warmup):
    seek = KalmanSeek([FakePlan()], warmup=warmup)
    out = {}
    for n in (5, 6, 7, 20, 3, 21, 0):
        sink = Sink()
        seek.frame(n, lambda f, p: f, [sink])
        out[n] = sink[0]
    assert out[0] == (0, None)  # frame 0 passes through
    first = lambda n: max(1, n - warmup)  # noqa: E731
    assert out[5] == (5, list(range(first(5), 6)))
    assert out[6] == (6, list(range(first(5), 7)))    # continues the snapshot of frame 5
    assert out[7] == (7, list(range(first(5), 8)))
    assert out[20] == (20, list(range(20 - warmup, 21)))  # no snapshot in reach: warmup frames
    assert out[3] == (3, [1, 2, 3])
    assert out[21] == (21, list(range(20 - warmup, 22)))


def test_cpp_snapshot_shelf_policy():
    """The C++ shelf behind KalmanCheckpoints and the frame server's Kalman snapshots
    (include/neo_fft_b200/snapshot_shelf.hpp) passes the same cases on the CPU."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    exe = root / "tests" / "_build" / "shelf_check"
    exe.parent.mkdir(exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{root / 'include'}", str(root / "tests" / "native" / "shelf_check.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert out.stdout.count("ok ") == 10
