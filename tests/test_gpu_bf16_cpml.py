"""BF16 CPML memories (SEIS3D_STORAGE_BF16_CPML): the passes keep wavefields and materials in
FP32 and store only the CPML memories in BF16, each FP32 update used in full and only the kept
memory rounded to nearest even.

* Against the CPU oracle emulating exactly that storage (oracle3d_set_psi_storage(2), FP32
  arithmetic).  Rounding to 8 bits amplifies differences at the FP32 rounding level: where two
  solvers' FP32 memories straddle a BF16 rounding boundary they keep values one BF16 ulp apart,
  and that difference feeds back.  The oracle shows it on its own: its emulation with the
  source amplitude perturbed by 2e-7 drifts from the unperturbed one by 8e-7 in the first 160
  steps of the free-surface shot and by 1.3e-4 in 400, while the storage effect is 3.8e-5 and
  2.9e-4.  So the check that the kernels round the same values at the same points is made while
  the waves have entered the CPML but before the drift (the first 160 steps with a free
  surface, 120 with six CPML faces, where the waves reach the layer sooner): there the traces
  must agree with the emulation to well under a tenth of the storage effect.
* Over the whole run the traces move by a few 1e-4 against FP32 storage, inside the 1e-3 bar of
  a 16-bit mode.
* The memories take half the bytes; batched BF16 shots equal their solo runs bit for bit.
The full-size runs against FP64 are in test_gpu_headline_parity.py."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

STEPS = 400
EMULATION_TOL = 5e-6    # relative L2 over the check window, BF16-memory kernels vs the emulation
STORAGE_BAR = 1e-3      # relative L2, 16-bit storage vs full FP32 storage


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def gpu_gather(shot, storage):
    s = seis3d.Session(shot.context, storage=storage)
    try:
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        s.gather_begin(2, STEPS // 2)
        s.run_steps(shot.source, 0, STEPS)
        return s.gather_fetch()
    finally:
        s.release()


def oracle_gather(shot, psi_storage):
    lib = oracle.oracle_library()
    lib.oracle3d_set_psi_storage(psi_storage)
    try:
        o = oracle.CpuOracle(shot.context, 32)
        o.upload_model(shot.vp, shot.vs, shot.rho)
        g = o.run_gather(shot.source, 0, STEPS, shot.receivers, 2)
        o.close()
    finally:
        lib.oracle3d_set_psi_storage(0)
    return g


@pytest.mark.parametrize("free_surface,check_steps", [(True, 160), (False, 120)])
def test_bf16_memories_match_oracle_emulation(free_surface, check_steps, solver_lib, cuda_device):
    shot = models3d.small_shot(nx=32, ny=28, nz=30, steps=STEPS, free_surface=free_surface)
    ours = gpu_gather(shot, capi.STORAGE_BF16_CPML)
    fp32 = gpu_gather(shot, capi.STORAGE_FP32)
    emulated = oracle_gather(shot, 2)
    plain = oracle_gather(shot, 0)
    assert ours.shape == emulated.shape and np.all(np.isfinite(ours))
    for steps in (80, 100, 120, 160, 200, 300, 400):
        n = steps // 2
        print(f"\nfree surface {free_surface}, first {steps} steps: vs BF16 emulation {rel_l2(ours[:n], emulated[:n]):.2e}, "
              f"vs FP32 oracle {rel_l2(ours[:n], plain[:n]):.2e}, vs FP32 storage on the GPU {rel_l2(ours[:n], fp32[:n]):.2e}, "
              f"emulation vs FP32 oracle {rel_l2(emulated[:n], plain[:n]):.2e}")
    n = check_steps // 2
    early_effect = rel_l2(emulated[:n], plain[:n])
    assert early_effect > 1e-5                              # the memories are in play by then
    assert rel_l2(ours[:n], emulated[:n]) < min(EMULATION_TOL, 0.1 * early_effect)
    storage_effect = rel_l2(ours, fp32)
    assert 1e-5 < storage_effect < STORAGE_BAR
    assert rel_l2(fp32, plain) < 1e-5       # the FP32 mode is the parity mode


def test_bf16_memories_take_half_the_bytes(solver_lib, cuda_device):
    shot = models3d.small_shot(steps=4)
    a = seis3d.Session(shot.context)
    b = seis3d.Session(shot.context, storage=capi.STORAGE_BF16_CPML)
    try:
        va, vb = a.views(), b.views()
        assert va.storage == capi.STORAGE_FP32 and vb.storage == capi.STORAGE_BF16_CPML
        memory_cells = sum(int(va.slabCells3D[k]) * 6 for k in range(3))
        assert [int(vb.slabCells3D[k]) for k in range(3)] == [int(va.slabCells3D[k]) for k in range(3)]
        assert int(va.allocatedBytes3D) - int(vb.allocatedBytes3D) == 2 * memory_cells
        # The learned boundary reads FP32 memories only.
        net = seis3d.BoundaryNet(8, seed=1)
        with pytest.raises(seis3d.InvalidArgument, match="FP32 CPML memories"):
            seis3d.attach_boundary(b, net, gain=1.0)
        net.release()
    finally:
        a.release()
        b.release()


def test_bf16_batch_equals_solo(solver_lib, cuda_device):
    steps = 120
    shot_list = [models3d.small_shot(nx=40, ny=32, nz=36, steps=steps, seed=7),
                 models3d.small_shot(nx=33, ny=41, nz=44, steps=steps, seed=9, free_surface=False,
                                     kind=capi.SOURCE_FORCE)]

    def prepared(shot):
        s = seis3d.Session(shot.context, storage=capi.STORAGE_BF16_CPML)
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        s.gather_begin(1, steps)
        return s

    solo = []
    for shot in shot_list:
        s = prepared(shot)
        s.run_steps(shot.source, 0, steps)
        solo.append((s.gather_fetch(), [s.field(k) for k in range(9)]))
        s.release()
    sessions = [prepared(shot) for shot in shot_list]
    batch = seis3d.Batch(sessions, shots_per_launch=2, z_chunk=16)
    batch.run_steps([shot.source for shot in shot_list], 0, steps)
    batch.synchronize()
    batch.release()
    for (gather, fields), s in zip(solo, sessions):
        assert np.array_equal(s.gather_fetch(), gather)
        for k in range(9):
            assert np.array_equal(s.field(k), fields[k]), capi.FIELDS[k]
        s.release()


def test_bf16_mode_without_cpml_equals_fp32(solver_lib, cuda_device):
    """Slip walls have no CPML memories, so the storage mode changes nothing: bit-identical."""
    shot = models3d.small_shot(steps=60, free_surface=False)
    c = shot.context.copy()
    c.reflecting3D = 1
    c = seis3d.validate_context3D(c)
    out = []
    for storage in (capi.STORAGE_FP32, capi.STORAGE_BF16_CPML):
        s = seis3d.Session(c, storage=storage)
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        s.gather_begin(1, shot.steps)
        s.run_steps(shot.source, 0, shot.steps)
        out.append((s.gather_fetch(), [s.field(k) for k in range(9)]))
        s.release()
    (g0, f0), (g1, f1) = out
    assert np.abs(g0).max() > 0
    assert np.array_equal(g0.view(np.uint32), g1.view(np.uint32))
    for k in range(9):
        assert np.array_equal(f0[k].view(np.uint32), f1[k].view(np.uint32)), capi.FIELDS[k]
