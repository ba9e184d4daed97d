"""Build the in-tree solver libraries for sm_100a with nvcc.

    python -m cmakepro_cuda_seissim_v2_b200.build [--force]

Both libraries are compiled from csrc/ with ``-gencode arch=compute_100a,code=sm_100a`` and
written next to this file so that they travel with the repository snapshot:

* ``libseis3d_b200.so`` - the 3-D solver, no fast math (the reference 3-D solver's own flags,
  CMakeLists.txt:208-236);
* ``libseis2d_b200.so`` - the 2-D P-SV solver, with ``--use_fast_math`` (the flag of the
  reference target that holds its 2-D solver, CMakeLists.txt:128-135).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIBRARIES = {
    "libseis3d_b200.so": (["seis3d_capi.cu", "seis3d_noalloc.cu"], []),
    "libseis2d_b200.so": (["seis2d_capi.cu"], ["--use_fast_math"]),
}


def _sources(names):
    return [os.path.join(CSRC, n) for n in names]


def _deps():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return deps


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the solver library needs the CUDA toolkit to build")
    return path


def build(force: bool = False, verbose: bool = False) -> list[str]:
    built = []
    newest_dep = max(os.path.getmtime(d) for d in _deps())
    for lib, (names, flags) in LIBRARIES.items():
        out = os.path.join(HERE, lib)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= newest_dep:
            continue
        cmd = [nvcc(), "-std=c++17", *ARCH, "-O3", "-lineinfo", *flags, "-Xcompiler", "-fPIC", "-shared",
               "-o", out + ".tmp", *_sources(names)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
        built.append(out)
    return built


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--force", action="store_true")
    p.add_argument("--verbose", action="store_true")
    args = p.parse_args(argv)
    for path in build(force=args.force, verbose=args.verbose):
        print("built", path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
