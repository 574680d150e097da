"""The command-line frontend (analogsat_b200/frontend/analogsat_cli.cpp): the reference
frontend's run / speedtest / bench commands (Frontend/src/main.cpp, cnf_runner.cpp,
bench_runner.cpp) on the C ABI, with its option names, problem-folder layout, result
file and perf-line formats."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def cli():
    from analogsat_b200 import build
    build.build()
    return build.build_cli()


def _run(cli, *args, cwd=None):
    return subprocess.run([cli, *args], capture_output=True, text=True, cwd=cwd, timeout=600)


def test_cli_rejects_bad_usage(cli):
    """Option errors are reported before any device call, with the reference's wording."""
    for args, msg in [((), "usage"), (("solve",), "command not understood"), (("run", "-eps", "2"), "-eps"),
                      (("run", "-nogpu"), "GPU solver only"), (("run", "-batch"), "needs a value"),
                      (("bench", "-samplestart", "5", "-sampleend", "5"), "sample range")]:
        r = _run(cli, *args)
        assert r.returncode == 2 and msg in r.stderr, (args, r.stderr)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["double", "float"])
def test_cli_run_writes_minisat_compatible_result(cli, tmp_path, golden, prec):
    from analogsat_b200.instances import is_satisfied
    extra = ["-float"] if prec == "float" else []
    r = _run(cli, "run", "-problem", os.path.join(ROOT, "tests", "golden", "p50.cnf"), "-resultfolder",
             str(tmp_path), "-trajectories", "8", "-timeout", "60", *extra)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "solution found" in r.stdout and "All done." in r.stdout
    lines = (tmp_path / "p50.out").read_text().splitlines()
    assert lines[0] == "SAT"
    vals = [int(v) for v in lines[1].split()]
    assert vals[-1] == 0 and [abs(v) for v in vals[:-1]] == list(range(1, 51))
    assert is_satisfied(golden["p50/literals"], golden["p50/lengths"], np.array(vals[:-1]) > 0)


@pytest.mark.gpu
def test_cli_bench_then_speedtest(cli, tmp_path):
    """bench makes random samples (N = 20, 40), solves them and keeps the solved ones in
    the reference's problem-folder layout; speedtest then runs them back (cycled to 200
    runs per N) and writes one perf line per run."""
    pf, rf = str(tmp_path / "problems"), str(tmp_path / "results")
    common = ["-problemfolder", pf, "-resultfolder", rf, "-nstart", "1", "-nend", "2", "-nstep", "1",
              "-alpha", "4.0", "-timeout", "30", "-float"]
    r = _run(cli, "bench", "-samplestart", "0", "-sampleend", "6", *common)
    assert r.returncode == 0, r.stdout + r.stderr
    for n in (20, 40):
        d = os.path.join(pf, "3a400", f"N{n}")
        kept = sorted(os.listdir(d))
        assert kept and all(f.startswith("p") and f.endswith(".cnf") for f in kept)
        perf = open(os.path.join(rf, f"perf_K3_a400_N{n}.dat")).read().splitlines()
        assert len(perf) == 6
    r = _run(cli, "speedtest", *common)
    assert r.returncode == 0, r.stdout + r.stderr
    rates = [ln for ln in r.stdout.splitlines() if ln.startswith("N=")]
    assert len(rates) == 2 and all("RHS evals/s=" in ln for ln in rates)
    for n in (20, 40):
        perf = open(os.path.join(rf, f"perf_K3_a400_N{n}.dat")).read().splitlines()
        assert len(perf) == 6 + 200
        f = perf[-1].split("\t")
        # sample, GPU, solver, answer, wall, CPU, RHS count (bench_runner.cpp:331-343)
        assert len(f) == 7 and f[0].startswith(f"3a400/N{n}/p") and f[2] == "analogsatb200f32orig"
        assert float(f[4]) > 0 and int(f[6]) > 0
