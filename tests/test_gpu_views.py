"""Display views of the 3-D solver (seis3d_extract_views = extractViews3D,
cuda/Cuda_Seis3D.cu:334-418,627-646) against the reference's own extraction on the same shot,
and the slice values against a numpy restatement of sampleScalar3D on the copied fields."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import models3d, seis3d

pytestmark = pytest.mark.gpu


def run_both(steps=40):
    shot = models3d.small_shot(steps=steps)
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.run_steps(shot.source, 0, steps)
    ref = None
    if oracle.reference_library() is not None:
        # The extraction is compared on identical inputs: the reference session gets this
        # solver's final fields (its materials come from the same upload path, bit for bit).
        ref = oracle.ReferenceSolver(shot.context)
        ref.upload_model(shot.vp, shot.vs, shot.rho)
        for k in range(9):
            ref.set_field(k, s.field(k))
        for k in (9, 10, 11):
            assert np.array_equal(ref.field(k), s.field(k))
    return shot, s, ref


def extract(s, layout, slices, component, material, volume, boundary):
    import torch
    count = layout.totalSamples3D if volume else layout.volumeOffset3D
    out = torch.full((2 * count,), -7.0, dtype=torch.float32, device="cuda")
    stats = s.extract_views(out.data_ptr(), layout, slices, component, material, volume, boundary)
    return out.cpu().numpy(), stats


def test_views_match_reference_and_numpy(solver_lib, cuda_device):
    shot, s, ref = run_both()
    c = s.context
    layout = seis3d.make_view_layout3D(c)
    slices = (c.nx3D // 2 + 1, c.ny3D // 3, c.nz3D // 2)
    for component, material, volume, boundary in [(0, 5, True, False), (1, 6, True, True), (2, 7, False, False),
                                                   (3, 5, True, False), (4, 7, True, True)]:
        ours, stats = extract(s, layout, slices, component, material, volume, boundary)
        assert np.all(np.isfinite(ours)) and np.abs(ours[0::2]).max() > 0
        if ref is not None:
            theirs, rstats = ref.extract_views(ours.size // 2, slices, component, material, volume, boundary)
            assert np.array_equal(ours, theirs), (component, np.abs(ours - theirs).max())
            assert stats == rstats
    # XZ slice of vz and the vp material by hand from the copied fields.
    ours, stats = extract(s, layout, slices, 0, 5, False, False)
    vz, lam, mu, inv = s.field(2), s.field(10), s.field(11), s.field(9)
    nx, nz = layout.domainSize3D[0], layout.domainSize3D[2]
    ox, oz = layout.domainOrigin3D[0], layout.domainOrigin3D[2]
    xs = np.arange(nx) + ox + c.ox3D
    zs = np.arange(nz) + oz + c.oz3D
    y = slices[1] + c.oy3D
    expect = (np.float32(0.5) * (vz[zs][:, y, xs] + vz[zs - 1][:, y, xs])).astype(np.float32)
    got = ours[0: 2 * nx * nz: 2].reshape(nz, nx)
    assert np.array_equal(got, expect)
    vp = np.sqrt((lam[zs][:, y, xs] + np.float32(2) * mu[zs][:, y, xs]) * inv[zs][:, y, xs]).astype(np.float32)
    assert np.allclose(ours[1: 2 * nx * nz: 2].reshape(nz, nx), vp, rtol=2e-7, atol=0)
    inside = (slice(-oz, -oz + c.nz3D), slice(-ox, -ox + c.nx3D))
    assert stats["maximum"] >= np.abs(got[inside]).max()
    assert stats["material_range"][0] <= vp[inside].min() and stats["material_range"][1] >= vp[inside].max()


def test_view_parameter_and_buffer_checks(solver_lib, cuda_device):
    import torch
    shot, s, _ = run_both(steps=2)
    c = s.context
    layout = seis3d.make_view_layout3D(c)
    good = torch.zeros(2 * layout.totalSamples3D, dtype=torch.float32, device="cuda")
    for slices, comp, mat in [((c.nx3D, 0, 0), 0, 5), ((0, 0, 0), 8, 5), ((0, 0, 0), 0, 4), ((0, -1, 0), 0, 5)]:
        with pytest.raises(seis3d.InvalidArgument):
            s.extract_views(good.data_ptr(), layout, slices, comp, mat, True)
    # An allocation of exactly the slices' size (torch's caching allocator would hand out a
    # piece of a larger segment, which the range check rightly accepts).
    from cuda.bindings import runtime as rt
    err, small = rt.cudaMalloc(2 * layout.volumeOffset3D * 4)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        with pytest.raises(seis3d.InvalidArgument):
            s.extract_views(int(small), layout, (1, 1, 1), 0, 5, True)     # the volume does not fit
        s.extract_views(int(small), layout, (1, 1, 1), 0, 5, False)         # the slices do
    finally:
        rt.cudaFree(small)
    host = np.zeros(2 * layout.totalSamples3D, np.float32)
    with pytest.raises(seis3d.InvalidArgument):
        s.extract_views(host.ctypes.data, layout, (1, 1, 1), 0, 5, True)    # not device memory
    bad = seis3d.make_view_layout3D(c)
    bad.volumeX3D += 1
    with pytest.raises(seis3d.InvalidArgument):
        s.extract_views(good.data_ptr(), bad, (1, 1, 1), 0, 5, True)
