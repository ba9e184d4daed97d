"""Generate the host-side golden vectors of the reference solver.

Runs the reference's own validateContext3D / estimateMemory3D / makeCoefficients3D
(cuda/Cuda_Seis3D.cu:45-64, :433-483, :504-516), compiled unmodified from the reference
tree into oracle/_ref/libref3d.so, on a fixed list of contexts and writes:

  ref3d_host.json          validation outcome + derived fields, memory budgets
  ref3d_coefficients.npz   CPML coefficient tables (float32) per context and axis

    python tests/golden/make_cpu_golden.py        (needs oracle/_ref/libref3d.so)
"""
import json
import os
import sys
from ctypes import POINTER, byref, c_float

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from cmakepro_cuda_seissim_v2_b200 import capi, seis3d  # noqa: E402

# (label, overrides) -- the first block are the reference test's own KAT sizes
# (tests/Seis3DBoundaryRegression.cpp:70-82); the rest cover the derivation branches.
CASES = [
    ("kat_600x200x200", dict(nx3D=600, ny3D=200, nz3D=200)),
    ("kat_300x300x400", dict(nx3D=300, ny3D=300, nz3D=400)),
    ("kat_reject_400x400x300", dict(nx3D=400, ny3D=400, nz3D=300)),
    ("kat_reject_intmax", dict(nx3D=2147483647, ny3D=2147483647, nz3D=2147483647)),
    ("kat_reject_negative", dict(nx3D=-1, ny3D=96, nz3D=96)),
    ("budget_96", dict(nx3D=96, ny3D=96, nz3D=96)),
    ("budget_160", dict(nx3D=160, ny3D=160, nz3D=160)),
    ("budget_300", dict(nx3D=300, ny3D=300, nz3D=300)),
    ("budget_300x300x400", dict(nx3D=300, ny3D=300, nz3D=400)),
    ("default", dict()),
    ("six_face_p20", dict(freeSurface3D=0, pml3D=20)),
    ("reflecting", dict(reflecting3D=1)),
    ("manual_500us", dict(manualTimeStep3D=1, requestedDtMs3D=0.5)),
    ("manual_fraction", dict(manualTimeStep3D=1, requestedDtMs3D=0.5004)),
    ("manual_above_cfl", dict(manualTimeStep3D=1, requestedDtMs3D=5.0)),
    ("pml_7", dict(pml3D=7)),
    ("pml_41", dict(pml3D=41)),
    ("cfl_high", dict(cfl3D=0.95)),
    ("bad_material", dict(vs3D=3000.0)),
    ("bad_geometry", dict(interfaceDepth3D=0.95)),
    ("uniform", dict(modelKind3D=capi.MODEL_UNIFORM)),
    ("imported", dict(modelKind3D=capi.MODEL_IMPORTED, maxVp3D=4500.0)),
    ("small_fs_p8", dict(nx3D=32, ny3D=24, nz3D=28, pml3D=8)),
    ("small_6face_p12_f50", dict(nx3D=32, ny3D=24, nz3D=28, pml3D=12, freeSurface3D=0, frequency3D=50.0)),
    ("cfg2", dict(nx3D=300, ny3D=50, nz3D=300, pml3D=20, modelKind3D=capi.MODEL_IMPORTED, maxVp3D=4500.0,
                  frequency3D=15.0, manualTimeStep3D=1, requestedDtMs3D=0.5)),
]
COEFFICIENT_CASES = ["default", "six_face_p20", "small_fs_p8", "small_6face_p12_f50", "cfg2"]


def main():
    ref = oracle.reference_library()
    if ref is None:
        raise SystemExit("oracle/_ref/libref3d.so is missing: run `make -C oracle` with the reference tree")
    host = {}
    tables = {}
    for label, overrides in CASES:
        c = seis3d.default_context(**overrides)
        status = ref.ref3d_validate(byref(c))
        entry = {"input": overrides, "status": status}
        if status == 0:
            entry["derived"] = {k: c.as_dict()[k] for k in ("gx3D", "gy3D", "gz3D", "ox3D", "oy3D", "oz3D",
                                                            "cells3D", "freeSurface3D")}
            entry["dt_bits"] = int(np.float32(c.dt3D).view(np.uint32))
            entry["safe_dt_bits"] = int(np.float32(c.safeDt3D).view(np.uint32))
            entry["maxVp3D"] = float(c.maxVp3D)
            b = capi.MemoryBudget()
            c2 = seis3d.default_context(**overrides)
            ref.ref3d_estimate_memory(byref(c2), byref(b))
            entry["budget"] = [b.fieldBytes3D, b.cpmlBytes3D, b.viewBytes3D, b.totalBytes3D]
            if label in COEFFICIENT_CASES and not c.reflecting3D:
                for axis in range(3):
                    n = (c.gx3D, c.gy3D, c.gz3D)[axis]
                    out = np.zeros(n * 6, dtype=np.float32)
                    ref.ref3d_make_coefficients(byref(c), axis, out.ctypes.data_as(POINTER(c_float)))
                    tables[f"{label}_axis{axis}"] = out
        host[label] = entry
    with open(os.path.join(HERE, "ref3d_host.json"), "w") as f:
        json.dump(host, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "ref3d_coefficients.npz"), **tables)
    print("wrote", len(host), "contexts and", len(tables), "coefficient tables")


if __name__ == "__main__":
    main()
