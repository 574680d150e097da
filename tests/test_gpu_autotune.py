"""The project-written autotuner: times candidate CTA sizes / storage modes on short
fixed-length solves, caches the fastest per instance-size bucket, applies it."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_applies(tmp_path, monkeypatch):
    import analogsat_b200.autotune as AT
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    monkeypatch.setattr(AT, "CACHE", str(tmp_path / "tune.json"))
    lits, lens, _ = make_instance("planted", 300, 1275, 3, seed=3)
    p = SatProblem.from_arrays(lits, lens)
    e = AT.tune(p, trajectories=64, steps=40, candidates=(128, 320, 1024))
    assert e["threads"] in (128, 320, 1024) and e["storage"] in (1, 2)
    assert len(e["candidates"]) == 6
    assert AT.lookup(p)["threads"] == e["threads"]
    s = SatSolver([p])
    assert AT.apply(s, p)
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(20000); s.SetMaxTime(1e8)
    s.SetSatStates(np.zeros(8, np.int32), initial_states(300, 1275, 8, seed=1, dtype=np.float32))
    s.Solve()
    assert s.launch_shape()["threads"] == e["threads"]
    assert (s.results()["status"] == 0).any()
