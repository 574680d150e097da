"""Structural checks of the device packing on random instances (tests/cpp/pack_check.cpp,
built with g++ against the host sources only): literal sets, contribution slots, SELL
row order, permutations and bank-group diagnostics for the FP64, FP32 and FP32-pair
layouts."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pack_structure(tmp_path):
    exe = str(tmp_path / "pack_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", exe, os.path.join(ROOT, "tests", "cpp", "pack_check.cpp"),
                    os.path.join(ROOT, "analogsat_b200", "csrc", "as_problem.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "pack ok" in r.stdout
