"""Host logic of bench.py that needs no GPU: the roofline's byte model per storage mode, the CPML
slab-cell counts of the two measured 3-D workloads (300 x 300 x 400 with six CPML faces of 20
cells: 50,864,000 active cells, 16,592,000 slab cells summed over axes; 300 x 50 x 300 with a
free surface and five faces: 9,792,000 and 6,116,000), the storage labels of the `config`
object, and the storage-mode numbers against the C-ABI's enum."""
import importlib.util
import os

import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, seis3d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def context(nx, ny, nz, free_surface):
    c = seis3d.default_context(nx3D=nx, ny3D=ny, nz3D=nz, pml3D=20, freeSurface3D=int(free_surface),
                               reflecting3D=0, spacing3D=10.0)
    return seis3d.validate_context3D(c)


@pytest.mark.parametrize("nx,ny,nz,free_surface,active,slab", [
    (300, 300, 400, False, 50_864_000, 16_592_000),
    (300, 50, 300, True, 9_792_000, 6_116_000),
])
def test_byte_model_of_both_workloads(bench, solver_lib, nx, ny, nz, free_surface, active, slab):
    c = context(nx, ny, nz, free_surface)
    assert (c.gx3D - 8) * (c.gy3D - 8) * (c.gz3D - 8) == active
    assert bench.slab_cells(c) == slab
    assert bench.step_bytes(c) == 84 * active + 48 * slab
    assert bench.step_bytes(c, "bf16_cpml") == 84 * active + 24 * slab


def test_storage_modes_match_the_c_abi(bench):
    assert bench.STORAGE_MODES == {"fp32": capi.STORAGE_FP32, "bf16_cpml": capi.STORAGE_BF16_CPML}
    assert set(bench.STORAGE_LABELS) == set(bench.STORAGE_MODES)
    assert bench.STORAGE_LABELS["fp32"] == "fp32"
    assert bench.FULL_STEPS == {"size_cap": 2500, "reference_default": 2000}
    assert bench.E2E_REPEATS >= 3
