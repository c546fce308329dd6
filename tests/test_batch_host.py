"""The batch and serving module's host logic (pysurf_b200.batch), on CPU: the sweep's draw, the
memory gate's admission, the arrival stream."""
import threading
import time

import numpy as np

from pysurf_b200 import batch


def test_the_sweep_is_drawn_from_its_seed_within_its_ranges():
    a, b = batch.drawSweep(256, seed=0), batch.drawSweep(256, seed=0)
    assert a == b and len(a) == 256
    slopes = np.array([c.slope for c in a])
    heights = np.array([c.height for c in a])
    ppds = np.array([c.ppd for c in a])
    assert slopes.min() >= 1.0 / 35.0 and slopes.max() <= 1.0 / 8.0
    assert heights.min() >= 0.2 and heights.max() <= 0.6
    assert ppds.min() >= 16 and ppds.max() <= 64
    # log-uniform slopes: about half below the geometric mean
    assert 0.35 < np.mean(slopes < np.sqrt(1.0 / 35.0 / 8.0)) < 0.65
    assert batch.drawSweep(8, seed=1) != batch.drawSweep(8, seed=0)


def test_the_memory_gate_holds_work_to_its_budget():
    gate = batch.MemoryGate(100)
    peak, held, lock = [0], [0], threading.Lock()

    def work(nbytes):
        gate.acquire(nbytes)
        with lock:
            held[0] += nbytes
            peak[0] = max(peak[0], held[0])
        time.sleep(0.02)
        with lock:
            held[0] -= nbytes
        gate.release(nbytes)

    threads = [threading.Thread(target=work, args=(40,)) for _ in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert peak[0] <= 100 and gate.held == 0


def test_a_request_larger_than_the_budget_runs_alone():
    gate = batch.MemoryGate(10)
    gate.acquire(50)            # alone: admitted
    admitted = threading.Event()
    t = threading.Thread(target=lambda: (gate.acquire(1), admitted.set()))
    t.start()
    assert not admitted.wait(0.05)
    gate.release(50)
    assert admitted.wait(1.0)
    t.join()


def test_poisson_arrivals_have_the_rate():
    arrivals = batch.poissonArrivals(4000, 20.0, seed=0)
    assert np.all(np.diff(arrivals) > 0)
    assert abs(len(arrivals) / arrivals[-1] - 20.0) < 1.0
