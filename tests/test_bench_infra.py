"""Measurement infrastructure of bench.py on the CPU: the clock sampler keeps only
samples taken from the timed region on, and the reference CPU sample is fixed work
(every run to its own SatResult, every run charged)."""
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
def test_reference_sample_is_fixed_work():
    """The CPU sample runs every unit to its own SatResult (no budget, none left out),
    charges every run's busy time, and gives the same solves and steps on a rerun, so
    the rate depends on the machine's speed only."""
    import bench
    from analogsat_b200.instances import make_instance, initial_states
    P, T = 3, 4
    probs = [make_instance("random", 120, 511, 3, seed=8 + i)[:2] for i in range(P)]
    pidx = np.repeat(np.arange(P), T).astype(np.int32)
    ics = np.concatenate([initial_states(120, 511, T, seed=20 + i) for i in range(P)])
    units = bench.cpu_sample_units(P, T)
    assert list(units) == [0, 4, 8, 1, 5, 9]  # trajectories 0 and 1, round-robin
    a = bench.cpu_baseline(probs, pidx, ics, units, nthreads=2, maxsteps=20000)
    b = bench.cpu_baseline(probs, pidx, ics, units[::-1], nthreads=2, maxsteps=20000)
    assert a["runs"] == b["runs"] == 6
    assert a["solved"] == b["solved"] and a["steps_mean"] == b["steps_mean"]
    assert a["value"] == pytest.approx(a["solved"] / a["busy"])
    assert a["busy"] <= a["wall"] + 1e-3
