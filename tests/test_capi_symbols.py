"""The C-ABI library loads without a GPU and exports every entry point the header declares."""
import os
import re
import subprocess

from cmakepro_cuda_seissim_v2_b200 import capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "seis3d_capi.h")


def declared_functions():
    text = open(HEADER).read()
    return set(re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(seis3d_\w+)\s*\(", text, flags=re.M))


def test_header_declarations_match_bindings():
    declared = declared_functions()
    assert declared, "no declarations parsed"
    assert declared == set(capi.SIGNATURES), declared ^ set(capi.SIGNATURES)


def test_library_exports_every_declared_symbol(solver_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIBRARY_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = declared_functions() - exported
    assert not missing, missing
    for name in declared_functions():
        assert hasattr(solver_lib, name)


def test_abi_version_and_error_string(solver_lib):
    assert solver_lib.seis3d_abi_version() == 1
    assert isinstance(solver_lib.seis3d_last_error(), bytes)


def test_lifecycle_errors_without_gpu(solver_lib):
    # Every session call rejects a null session as a lifecycle error, before touching CUDA
    # (reference runStep3D / refreshCpml throw std::logic_error when not initialised).
    from ctypes import byref
    from cmakepro_cuda_seissim_v2_b200 import seis3d

    c = seis3d.validate_context3D(seis3d.default_context())
    s = seis3d.default_source(x3D=10, y3D=10, z3D=10)
    assert solver_lib.seis3d_run_step(None, byref(c), byref(s), 0) == capi.SEIS3D_LOGIC_ERROR
    assert solver_lib.seis3d_reset(None, byref(c)) == capi.SEIS3D_LOGIC_ERROR
    assert solver_lib.seis3d_refresh_cpml(None, byref(c)) == capi.SEIS3D_LOGIC_ERROR
    solver_lib.seis3d_release(None)  # idempotent / null-safe like releaseGpu3D


def test_storage_enum_matches_bindings():
    """enum seis3d_storage of the header and the Python constants agree, name by name."""
    text = open(HEADER).read()
    body = re.search(r"enum\s+seis3d_storage\s*\{([^}]*)\}", text).group(1)
    values = {name: int(value) for name, value in re.findall(r"SEIS3D_STORAGE_(\w+)\s*=\s*(\d+)", body)}
    assert values == {"FP32": capi.STORAGE_FP32, "FP16": capi.STORAGE_FP16, "BF16": capi.STORAGE_BF16,
                      "BF16_CPML": capi.STORAGE_BF16_CPML}
