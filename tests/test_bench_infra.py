"""Measurement infrastructure of bench.py on the CPU: the clock sampler keeps only
samples taken from the timed region on, and the reference arm's sampler bounds a
step (new runs stop at the budget, running ones at twice it) and reports per-run
busy time."""
import os
import subprocess
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libanalogsat_ref.so")


def test_clock_sampler_keeps_timed_region_samples(monkeypatch):
    import bench
    rows = "0, 1965, 1965, 500, 0x0, Not Active, Not Active, Not Active, Not Active"
    late = "0, 1965, 1965, 900, 0x4, Not Active, Not Active, Not Active, Active"
    script = f"sleep 0.2; echo '{rows}'; sleep 0.3; while true; do echo '{late}'; sleep 0.05; done"
    real = subprocess.Popen
    monkeypatch.setattr(subprocess, "Popen", lambda args, **kw: real(["bash", "-c", script], **kw))
    with bench.Clocks(0) as c:
        time.sleep(0.4)  # the "timed region"
    s = c.summary()
    assert c.skip == 1            # the sample taken before the region is dropped
    assert s["samples"] >= 1
    assert s["reasons"] == ["sw_power_cap"]
    assert s["sm_mhz"] == 1965.0


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference checker not built here")
def test_reference_sampler_bounds_a_step():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    from analogsat_b200.instances import make_instance, initial_states
    R = Reference()
    lits, lens, _ = make_instance("random", 120, 511, 3, seed=8)
    p = R.problem(lits, lens)
    x = initial_states(120, 511, 64, seed=2)
    t0 = time.perf_counter()
    r = R.solve_many([p], np.zeros(64, np.int32), list(x), eps=1e-6, maxsteps=10 ** 7, batch=50,
                     nthreads=2, wall_budget=0.3)
    wall = time.perf_counter() - t0
    assert wall < 0.3 * 2 + 0.5
    done = r["done"].astype(bool)
    assert done.sum() == r["completed"]
    assert (r["busy"][done] > 0).all() and (r["busy"][~done] == 0).all()
    assert r["busy"][done].sum() <= 2 * r["wall"] + 1e-3
