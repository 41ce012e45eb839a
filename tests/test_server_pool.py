"""Placement of served requests over several devices' request loops
(``ServerPool``): a host request goes to the loop with the fewest
outstanding samples (then requests, then the lowest index), a request on a
CUDA tensor to its device's loop, each with the plan compiled for that
device. Checked on the CPU with stand-in loops that record what they get;
the device form runs in tests/test_gpu_serving.py."""
import numpy as np
import pytest

from processseg_b200.server import ServerPool, leastLoaded


def test_least_loaded_picks_fewest_samples_then_requests_then_index():
    assert leastLoaded([(0, 0)]) == 0
    assert leastLoaded([(3, 900), (9, 100), (1, 500)]) == 1
    assert leastLoaded([(3, 100), (2, 100), (2, 100)]) == 1
    assert leastLoaded([(0, 0), (0, 0)]) == 0
    with pytest.raises(ValueError):
        leastLoaded([])


class FakeLoop:
    """A loop on ``device`` whose outstanding work grows with what it takes."""

    def __init__(self, device, requests=0, samples=0):
        self.device = device
        self.requests, self.samples = requests, samples
        self.taken = []

    def load(self):
        return self.requests, self.samples

    def submit(self, plan, src, dst, meta):
        self.taken.append(plan)
        self.requests += 1
        self.samples += src.size
        return len(self.taken)

    def wait(self, t, timeout_ms=0):
        self.requests -= 1

    def close(self):
        pass


class FakePlan:
    def __init__(self, device):
        self.device = device
        self.twins = {}

    def forDevice(self, d):
        if d == self.device:
            return self
        return self.twins.setdefault(d, FakePlan(d))


def test_host_requests_spread_by_outstanding_samples():
    loops = [FakeLoop(0, samples=5000), FakeLoop(1), FakeLoop(2, samples=1000)]
    pool = ServerPool(loops=loops)
    plan = FakePlan(0)
    blocks = [np.zeros((10, 100), np.float32) for _ in range(6)]  # 1000 samples each
    placed = [pool.submit(plan, b, b, None)[0] for b in blocks]
    # loop 1 first (no samples); at equal samples the loop with fewer
    # requests; loop 0 (5000 outstanding) is never the least loaded here
    assert placed == [1, 2, 1, 2, 1, 2]
    assert [lp.samples for lp in loops] == [5000, 3000, 4000]
    # each loop got the plan compiled for its own device
    for lp in loops:
        assert all(p.device == lp.device for p in lp.taken)


class FakeDev:
    type = "cuda"

    def __init__(self, index):
        self.index = index


class FakeTensor:
    def __init__(self, index, size=100):
        self.device = FakeDev(index)
        self.size = size


def test_device_requests_stay_on_their_device():
    loops = [FakeLoop(0), FakeLoop(1, samples=10 ** 9)]
    pool = ServerPool(loops=loops)
    i, _ = pool.submit(FakePlan(0), FakeTensor(1), FakeTensor(1), None)
    assert i == 1 and loops[1].taken[0].device == 1
    with pytest.raises(ValueError):
        pool.place(FakeTensor(5))
