"""What 16-bit storage would cost, measured before building it.

The CPU oracle emulates kernels that keep the wavefields and/or materials in FP16 or BF16
(per-field power-of-two scale, FP32 arithmetic, CPML memories in FP32) and the receiver
traces are compared with the FP64 run of the same scheme.  The bar for a faster storage mode
is 1e-3 relative L2 trace error.  Rounding every stored value to 11 (FP16) or 8 (BF16) bits
adds an error of about 2^-12 or 2^-9 per store, which random-walks over the steps: full 16-bit
wavefield storage misses the bar, so the solver keeps FP32 storage."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import models3d

STEPS = 400


def traces(shot, precision, storage=0, mask=7):
    lib = oracle.oracle_library()
    lib.oracle3d_set_storage(storage, mask)
    try:
        o = oracle.CpuOracle(shot.context, precision)
        o.upload_model(shot.vp, shot.vs, shot.rho)
        g = o.run_gather(shot.source, 0, STEPS, shot.receivers, 2)
        o.close()
    finally:
        lib.oracle3d_set_storage(0, 7)
    return g


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_sixteen_bit_storage_error_against_fp64(solver_lib):
    shot = models3d.small_shot(nx=32, ny=28, nz=30, steps=STEPS)
    ref = traces(shot, 64)
    errors = {
        "fp32": rel(traces(shot, 32), ref),
        "fp16 all": rel(traces(shot, 32, 1, 7), ref),
        "bf16 all": rel(traces(shot, 32, 2, 7), ref),
        "fp16 stresses": rel(traces(shot, 32, 1, 2), ref),
        "fp16 materials": rel(traces(shot, 32, 1, 4), ref),
    }
    print({k: f"{v:.2e}" for k, v in errors.items()})
    assert errors["fp32"] < 1e-5
    assert errors["fp16 all"] > 1e-3          # misses the bar
    assert errors["bf16 all"] > 1e-2
    assert errors["fp16 stresses"] > 5e-4     # half the traffic saving, still close to the bar
    assert errors["fp16 materials"] < 1e-3    # within the bar, but only 6 of 84 B per cell


def test_sixteen_bit_cpml_memories(solver_lib):
    """CPML memories kept in 16 bits, the FP32 update used in full and only the stored memory
    rounded (it would halve the 48 B per slab cell of memory traffic).  BF16 moves the traces by
    a few 1e-4 relative: within the 1e-3 bar, far outside the 1e-5 FP32 parity bar, so the
    memories stay FP32.  FP16 without a scale loses the small memories outright."""
    lib = oracle.oracle_library()
    shot = models3d.small_shot(nx=32, ny=28, nz=30, steps=STEPS)
    plain = traces(shot, 32)
    out = {}
    for name, mode in (("bf16", 2), ("fp16", 1)):
        lib.oracle3d_set_psi_storage(mode)
        try:
            out[name] = rel(traces(shot, 32), plain)
        finally:
            lib.oracle3d_set_psi_storage(0)
    print({k: f"{v:.2e}" for k, v in out.items()})
    assert 1e-5 < out["bf16"] < 1e-3
    assert out["fp16"] > 1e-3


def test_memory_rounding_does_not_depend_on_threads(solver_lib):
    """The 16-bit memory emulation reads no state that the parallel updates write: one thread
    and all threads give the same traces bit for bit."""
    lib = oracle.oracle_library()
    shot = models3d.small_shot(nx=32, ny=28, nz=30, steps=150)
    out = []
    lib.oracle3d_set_psi_storage(2)
    try:
        for threads in (1, 0):
            lib.oracle3d_set_threads(threads)
            o = oracle.CpuOracle(shot.context, 32)
            o.upload_model(shot.vp, shot.vs, shot.rho)
            out.append(o.run_gather(shot.source, 0, 150, shot.receivers, 2))
            o.close()
    finally:
        lib.oracle3d_set_psi_storage(0)
        lib.oracle3d_set_threads(0)
    assert np.array_equal(out[0], out[1])
