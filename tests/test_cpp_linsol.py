"""The C++ linsol mirror compiles against include/bbmg_b200.h, links the library and
drives a solve (on CPU the expected outcome is the library's no-device error)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "linsol_check.cpp")
LIBDIR = os.path.join(ROOT, "nga2_b200")


def build_exe(tmp_path):
    exe = str(tmp_path / "linsol_check")
    subprocess.run(["g++", "-std=c++17", "-O2", SRC, "-o", exe, f"-L{LIBDIR}", "-lbbmg_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_cpp_mirror_builds_and_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present: covered by the gpu test")
    r = subprocess.run([build_exe(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_cpp_mirror_solves(tmp_path):
    r = subprocess.run([build_exe(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    it, rerr = r.stdout.split()
    assert 0 < int(it) < 20 and float(rerr) <= 1e-10
