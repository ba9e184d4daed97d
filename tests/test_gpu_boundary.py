"""The learned thin boundary's kernels against their CPU restatement (oracle/boundary_net.py).

* gradients: one forward and backward pass of the tensor-core training kernel on given rows
  equals the restatement's gradient of the weighted squared error (same BF16 rounding
  points, FP32 vs FP64 accumulation);
* inference: one step of a thin-CPML session with a network attached equals the same step
  without it plus the restatement's corrections on the owned band cells;
* collection: the rows recorded from a thin and a wide session are the restatement's inputs
  and targets of the same columns, and the thin interior afterwards holds the wide one's.
"""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d
from oracle import boundary_net as ref

pytestmark = pytest.mark.gpu


def random_parameters(rng, scale=1.0):
    p = np.zeros(capi.BOUNDARY_PARAMETERS, dtype=np.float32)
    p[ref.W1:ref.W2] = rng.normal(0, np.sqrt(2 / 240), ref.W2 - ref.W1)
    p[ref.W2:ref.W3] = rng.normal(0, np.sqrt(2 / 64), ref.W3 - ref.W2)
    w3 = rng.normal(0, 0.2 * scale, (ref.OUT_PAD, ref.HIDDEN))
    w3[ref.OUT:] = 0.0
    p[ref.W3:ref.MATRICES] = w3.ravel()
    p[ref.B1:ref.B3] = rng.normal(0, 0.05, ref.B3 - ref.B1)
    b3 = rng.normal(0, 0.05 * scale, ref.OUT_PAD)
    b3[ref.OUT:] = 0.0
    p[ref.B3:] = b3
    return p


def thin_shot(steps, free_surface=True, pml=6):
    """A small layered shot on a thin CPML, source near the x- and z+ faces."""
    nx, ny, nz = 40, 32, 36
    vp = models3d.layered_model(nx, ny, nz, [2000, 2600, 3200])
    vp = vp * (1.0 + 0.05 * models3d.splitmix64_uniform(nx * ny * nz, 3).reshape(nz, ny, nx))
    vp, vs, rho = models3d.elastic_from_vp(vp)
    c = seis3d.default_context(nx3D=nx, ny3D=ny, nz3D=nz, spacing3D=10.0, pml3D=pml, freeSurface3D=int(free_surface),
                               reflecting3D=0, modelKind3D=capi.MODEL_IMPORTED, maxVp3D=float(vp.max()),
                               frequency3D=25.0)
    seis3d.validate_thin_context3D(c)
    src = seis3d.default_source(x3D=8, y3D=16, z3D=26, kind3D=capi.SOURCE_EXPLOSION, amplitude3D=1.0e8)
    return c, src, vp, vs, rho, steps


def test_training_gradients_match_cpu_restatement(solver_lib, cuda_device):
    rng = np.random.default_rng(5)
    net = seis3d.BoundaryNet(6, seed=3)
    params = random_parameters(rng)
    net.set_parameters(2, params, 0.7)
    rows = 200                                   # not a multiple of the kernel's 64-row tiles
    x = rng.normal(0, 1, (rows, ref.IN)).astype(np.float32)
    x[:, ref.SCHEME:ref.SCHEME + 5] = [0.3, 0.17, 0.4, 0.01, 1.0]
    x[:, ref.SCHEME + 5:] = 0.0
    x = ref.bf16(x)                              # the dataset stores BF16 inputs
    t = rng.normal(0, 0.5, (rows, ref.OUT)).astype(np.float32)
    w = rng.uniform(0.1, 1.0, rows).astype(np.float32) / (rows * ref.OUT)
    grad, loss = net.gradients(2, x, t, w)
    want, want_loss = ref.gradients(params, x, t, w, 0.7)
    assert loss == pytest.approx(want_loss, rel=2e-3)
    blocks = {"W1": (ref.W1, ref.W2), "W2": (ref.W2, ref.W3), "W3": (ref.W3, ref.MATRICES), "b1": (ref.B1, ref.B2),
              "b2": (ref.B2, ref.B3), "b3": (ref.B3, ref.PARAMETERS)}
    for name, (a, b) in blocks.items():
        g, e = grad[a:b].astype(np.float64), want[a:b]
        err = np.linalg.norm(g - e) / np.linalg.norm(e)
        assert err < 2e-2, (name, err)
    assert np.all(grad[ref.W3 + ref.OUT * ref.HIDDEN:ref.MATRICES] == 0)
    assert np.all(grad[ref.B3 + ref.OUT:] == 0)
    net.release()


def materials(session):
    return [session.field(9), session.field(10), session.field(11)]


def memories(session):
    """Host copies of the session's three CPML memory arrays (flat) and the row pitch."""
    from cuda.bindings import runtime as rt
    v = session.views()
    c = session.context
    p, pitch = c.pml3D, int(v.pitch)
    counts = [6 * c.gz3D * c.gy3D * 2 * p, 6 * c.gz3D * 2 * p * pitch,
              6 * (1 if c.freeSurface3D else 2) * p * c.gy3D * pitch]
    out = []
    for a in range(3):
        host = np.zeros(counts[a], dtype=np.float32)
        err, = rt.cudaMemcpy(host.ctypes.data, v.cpml3D[a], host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(host)
    return out, pitch


@pytest.mark.parametrize("free_surface", [True, False])
def test_correction_step_matches_cpu_restatement(free_surface, solver_lib, cuda_device):
    c, src, vp, vs, rho, steps = thin_shot(40, free_surface)
    rng = np.random.default_rng(11)
    net = seis3d.BoundaryNet(6, seed=1)
    params, scales = {}, {}
    for face in ref.faces(c):
        params[face] = random_parameters(rng, 0.5)
        scales[face] = 1e-3 * (1 + face)
        net.set_parameters(face, params[face], scales[face])
    plain = seis3d.Session(c, thin_cpml=True)
    learned = seis3d.Session(c, thin_cpml=True)
    for s in (plain, learned):
        s.upload_model(vp, vs, rho)
        s.run_steps(src, 0, steps)
    seis3d.attach_boundary(learned, net, gain=0.8)
    plain.run_step(src, steps)
    learned.run_step(src, steps)
    before = [plain.field(k).astype(np.float64) for k in range(9)]
    after = [learned.field(k).astype(np.float64) for k in range(9)]
    psi, pitch = memories(plain)
    want = ref.corrections(c, before, materials(plain), psi, pitch, params, scales, gain=0.8)
    z0 = 4 if free_surface else 0                # ghost planes above a free surface are re-imaged
    if free_surface:
        want[5][4] = -before[5][4]               # the re-imaging keeps szz = 0 on the surface plane
    total = max(np.abs(w).max() for w in want)
    assert total > 0
    for k in range(9):
        got = (after[k] - before[k])[z0:]
        err = np.abs(got - want[k][z0:]).max()
        assert err <= 2e-2 * total + 1e-6 * np.abs(before[k]).max(), (capi.FIELDS[k], err, total)
    # The network changes nothing outside the owned band cells.
    mask = np.zeros_like(before[0], dtype=bool)
    for w in want:
        mask |= w != 0
    for k in range(9):
        assert np.array_equal(after[k][z0:][~mask[z0:]], before[k][z0:][~mask[z0:]]), capi.FIELDS[k]
    seis3d.attach_boundary(learned, None)
    for s in (plain, learned):
        s.release()
    net.release()


def test_collected_rows_match_cpu_restatement(solver_lib, cuda_device):
    c, src, vp, vs, rho, steps = thin_shot(40, True)
    wide_c = c.copy()
    wide_c.pml3D = 16
    seis3d.validate_thin_context3D(wide_c)
    thin = seis3d.Session(c, thin_cpml=True)
    wide = seis3d.Session(wide_c)
    for s in (thin, wide):
        s.upload_model(vp, vs, rho)
        s.run_steps(src, 0, steps)
    thin_fields = [thin.field(k).astype(np.float64) for k in range(9)]
    wide_fields = [wide.field(k).astype(np.float64) for k in range(9)]
    mats = materials(thin)
    psi, pitch = memories(thin)
    data = seis3d.BoundaryDataset(20000)
    data.begin_model()
    data.collect(thin, wide, fraction=1.0, seed=9)
    rows = data.rows()
    faces = ref.faces(c)
    assert rows[4] == 0 and all(rows[f] > 0 for f in faces)
    face = 0                                     # the face nearest the source
    axis, side, nu, nw, ends = faces[face]
    x, y, s = data.read(face, 0, rows[face])
    # Index the restatement's columns by their (rounded) input rows to match the unordered rows.
    expect = {}
    ow = [c.ox3D, c.oy3D, c.oz3D]
    wo = [wide_c.ox3D, wide_c.oy3D, wide_c.oz3D]
    for w in range(nw):
        for u in range(nu):
            x_in, amp, imp = ref.column_inputs(c, thin_fields, mats, face, u, w, psi, pitch)
            if amp <= 0:
                continue
            target = np.zeros(36)
            for k in range(9):
                for d in range(4):
                    p = ref.cell(c, face, u, w, d)
                    q = [p[a] - ow[a] + wo[a] for a in range(3)]
                    diff = wide_fields[k][q[2], q[1], q[0]] - thin_fields[k][p[2], p[1], p[0]]
                    target[4 * k + d] = diff * (1.0 if k < 3 else 1.0 / imp) / amp
            expect[float(amp)] = (x_in, target)
    # Columns with a measurable amplitude (the weakest underflow differently in FP32 and FP64).
    thr = 1e-6 * max(expect)
    strong = [r for r in range(rows[face]) if s[r] > thr]
    keys = np.array(sorted(a for a in expect if a > thr))
    assert abs(len(strong) - len(keys)) <= 2 and len(keys) > 100
    for r in strong:
        i = int(np.argmin(np.abs(keys - s[r])))
        assert abs(keys[i] - s[r]) <= 1e-5 * keys[i]
        x_in, target = expect[keys[i]]
        assert np.allclose(x[r], ref.bf16(x_in.astype(np.float32)), rtol=1e-2, atol=1e-2)
        assert np.allclose(y[r], target, rtol=1e-3, atol=1e-4 * np.abs(target).max() + 1e-12)
    # Teacher forcing: the thin interior now equals the wide interior.
    for k in range(9):
        t = thin.field(k)[c.oz3D:c.oz3D + c.nz3D, c.oy3D:c.oy3D + c.ny3D, c.ox3D:c.ox3D + c.nx3D]
        v = wide.field(k)[wide_c.oz3D:wide_c.oz3D + c.nz3D, wide_c.oy3D:wide_c.oy3D + c.ny3D,
                          wide_c.ox3D:wide_c.ox3D + c.nx3D]
        assert np.array_equal(t, v), capi.FIELDS[k]
    data.release()
    thin.release()
    wide.release()
