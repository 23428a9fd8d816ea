"""The shared-memory layout planner (host C++) yields aligned, disjoint
regions for every species shape and precision -- compiled and run on the CPU."""
import shutil
import subprocess

import pytest

from tests.conftest import ROOT


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc needed to compile the host-side layout check")
def test_layouts_are_aligned_and_disjoint(tmp_path):
    exe = tmp_path / "layout_check"
    src = ROOT / "tests" / "layout_check.cpp"
    inc = ROOT / "co_cultivation_metabolic_atlas_b200" / "csrc"
    subprocess.run(["nvcc", "-std=c++17", "-x", "cu", "-Wno-deprecated-gpu-targets", "-I", str(inc),
                    str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert "bad 0" in out.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ needed to compile the host-side check")
def test_bank_spreading_keeps_rows_and_lowers_conflicts(tmp_path):
    exe = tmp_path / "spread_check"
    csrc = ROOT / "co_cultivation_metabolic_atlas_b200" / "csrc"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(csrc), str(ROOT / "tests" / "spread_check.cpp"),
                    str(csrc / "prepare.cpp"), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    words = out.stdout.split()
    before, after = int(words[words.index("before") + 1]), int(words[words.index("after") + 1])
    assert after <= 0.85 * before, out.stdout
