"""The header-only C++ adapter (include/analogsat_b200.hpp) compiled with g++ and linked
against the in-tree CUDA library, driven like the reference frontend drives
CudaSatSolver<double>."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp")


@pytest.fixture(scope="module")
def adapter_bin(tmp_path_factory):
    from analogsat_b200 import build
    build.build()
    out = str(tmp_path_factory.mktemp("cpp") / "adapter_check")
    libdir = os.path.join(ROOT, "analogsat_b200")
    subprocess.run(["g++", "-std=c++14", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
                    "-L", libdir, "-lanalogsat_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return out


def test_adapter_host_behaviour(adapter_bin, tmp_path):
    r = subprocess.run([adapter_bin, "host", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    assert "host ok" in r.stdout


@pytest.mark.gpu
def test_adapter_solves_like_reference(adapter_bin, tmp_path, golden):
    """Same call sequence as the reference frontend; FP64 reproduces the reference's own
    SatSolver result for the golden IC (SatResult and step count)."""
    ic = golden["p50/solve_ics"][0]
    f = tmp_path / "ic.txt"
    np.savetxt(f, ic, fmt="%.17g")
    r = subprocess.run([adapter_bin, "gpu", os.path.join(ROOT, "tests", "golden", "p50.cnf"), str(f)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rows = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.strip().splitlines()}
    assert int(rows["f64"][0]) == golden["p50/solve_result"][0]
    assert int(rows["f64"][1]) == golden["p50/solve_steps"][0]
    assert int(rows["f64"][2]) == golden["p50/solve_rhs"][0]
    assert int(rows["f32"][0]) == 0 and int(rows["f32"][4]) == 0
    assert [int(v) for v in rows["cnf_device"]] == [50, 210, 3]
    u = np.random.Generator(np.random.Philox(key=42)).random(260)  # reference transform
    assert int(rows["rand"][0]) == 260
    assert [float(v) for v in rows["rand"][1:]] == [u[0] * 2 - 1, u[49] * 2 - 1, u[259] + 1]
