"""Seis3D::extractViews3D of the header-only reference layer (include/compat/Cuda_Seis3D.cuh,
declared as in cuda/Cuda_Seis3D.cuh:24-26): tests/compat_views.cpp calls it the way the
reference's renderer does and compares it with the C entry point on the same session."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "cmakepro_cuda_seissim_v2_b200")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(tmp_path) -> str:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "compat_views")
    cmd = [gxx, "-std=c++20", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include", "compat"),
           "-I", os.path.join(CUDA_HOME, "include"), os.path.join(HERE, "compat_views.cpp"), "-o", exe,
           "-L", PKG, "-l:libseis3d_b200.so", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
           f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{os.path.join(CUDA_HOME, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_compat_layer_declares_extract_views(tmp_path, solver_lib):
    exe = build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_extract_views_through_compat_layer(tmp_path, solver_lib, cuda_device):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("views ")
