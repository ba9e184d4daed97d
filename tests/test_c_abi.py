"""The C ABI from plain C: tests/c_abi_shot.c includes both headers, is compiled as strict C99
(-pedantic -Werror) and linked against the two libraries.  On the CPU it answers a host-only
call; on a B200 it runs a 3-D shot with a device gather and a checkpoint restart, and a 2-D
shot, through nothing but the C entry points."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "cmakepro_cuda_seissim_v2_b200")


def build_example(tmp_path) -> str:
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path / "c_abi_shot")
    cmd = [gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "c_abi_shot.c"), "-o", exe, "-L", PKG, "-l:libseis3d_b200.so", "-l:libseis2d_b200.so",
           "-lm", f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_headers_are_c99_and_link(tmp_path, solver_lib, solver2d_lib):
    exe = build_example(tmp_path)
    r = subprocess.run([exe, "link"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["abi", "1", "1"]


@pytest.mark.gpu
def test_shots_from_c(tmp_path, solver_lib, solver2d_lib, cuda_device):
    exe = build_example(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    words = r.stdout.split()
    assert words[0] == "gather3d" and words[2] == "restart" and words[4] == "trace2d"
    g3, restart, t2 = float(words[1]), int(words[3]), float(words[5])
    assert np.isfinite(g3) and g3 > 0 and restart == 1 and np.isfinite(t2) and t2 > 0
