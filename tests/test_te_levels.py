"""The level schedule of core_dTe's diffusion sweep (te_levels in
spilady_b200/csrc/sld_host.cpp), checked on the host: compiled with the
engine's host source and run against the sequential colour sweep on even,
odd and mixed periodic meshes (tests/csrc/te_levels_check.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_te_levels_match_the_sequential_sweep(tmp_path):
    exe = tmp_path / "te_levels_check"
    src = os.path.join(ROOT, "tests", "csrc", "te_levels_check.cpp")
    host = os.path.join(ROOT, "spilady_b200", "csrc", "sld_host.cpp")
    inc = os.path.join(ROOT, "spilady_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", inc, "-I", os.path.join(ROOT, "include"),
                    src, host, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout
    lines = out.stdout.strip().splitlines()
    assert len(lines) == 7 and all(l.endswith("diff=0") for l in lines)
    # an even mesh (8 colours) takes 7 levels instead of 16 phases
    assert any(l.startswith("16x16x16 G=8 L=7 ") for l in lines)
