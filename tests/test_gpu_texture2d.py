"""2-D wavefield texture (seis2d_wavefield_texture = generateWavefieldTextureOnGpu,
CUDA_Kernels/Cuda_Check.cu:700-790,1136-1141) on the B200: bit-identical to the reference's own
kernel on the same fields (both built with --use_fast_math), and within one 8-bit step of a
numpy restatement with IEEE arithmetic (the approximate division and square root of fast math
can move a truncated byte by one)."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi2d, seis2d
from seis2d_cases import add_pml, make_context

pytestmark = pytest.mark.gpu

BALANCE = {0: 1.0, 1: 1.0, 2: 1.0, 3: 2.0, 4: 3.0, 5: 8.0, 6: 8.0}


def component_values(f, flag, comp):
    """The value of generateColorMapKernel before scaling, float32 [NZ][NX]."""
    split = flag in (1, 3)
    vx = f["vx_1"] + f["vx_2"] if split else f["vx"]
    vz = f["vz_1"] + f["vz_2"] if split else f["vz"]
    left = lambda a: np.concatenate([a[:, :1], a[:, :-1]], axis=1)   # noqa: E731  (column j-1, clamped)
    up = lambda a: np.concatenate([a[:1], a[:-1]], axis=0)           # noqa: E731  (row i-1, clamped)
    k = np.float32(1000)
    if comp == 0:
        return np.sqrt(vx * vx + vz * vz)
    if comp == 1:
        return vx
    if comp == 2:
        return vz
    if comp == 3:
        stress = (f["sxx_1"] + f["sxx_2"] + f["szz_1"] + f["szz_2"]) if split else f["sigmaxx"] + f["sigmazz"]
        l2m = f["lambda2mu"]
        return np.where(l2m > 1000, stress / l2m, stress) * k
    if comp == 4:
        shear = f["sxz_1"] + f["sxz_2"] if split else f["sigmaxz"]
        mu = f["mu"]
        return np.where(mu > 1000, shear / mu, shear) * k
    if comp == 5:
        return (vx - left(vx)) + (vz - up(vz))
    if comp == 6:
        return (vz - left(vz)) - (vx - up(vx))
    return np.zeros_like(vx)


def texture_numpy(f, flag, scale, comp):
    val = component_values(f, flag, comp).astype(np.float32)
    norm = np.clip(val * np.float32(scale) * np.float32(BALANCE.get(comp, 1.0)), -1, 1).astype(np.float32)
    out = np.full(val.shape + (4,), 255, np.uint8)
    pos = norm > 0
    fade_pos = (np.float32(255) * (np.float32(1) - norm)).astype(np.uint8)
    fade_neg = (np.float32(255) * (np.float32(1) + norm)).astype(np.uint8)
    out[..., 1] = np.where(pos, fade_pos, fade_neg)
    out[..., 2] = np.where(pos, fade_pos, 255)
    out[..., 0] = np.where(pos, 255, fade_neg)
    return out


def fields_of(gpu):
    out = {}
    for name in capi2d.FIELDS:
        try:
            out[name] = seis2d.copyField(gpu, name)
        except seis2d.InvalidArgument:
            pass
    return out


@pytest.mark.parametrize("scheme,up", [(1, False), (2, False), (3, True)])
def test_texture_matches_reference_and_numpy(scheme, up, solver2d_lib, cuda_device):
    import torch
    ctx = add_pml(make_context(scheme, up))
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    seis2d.runGpuSimulationSteps(gpu, 0, 250, ctx)
    f = fields_of(gpu)
    ref = None
    if oracle.reference2d_library() is not None:
        ref = oracle.ReferenceSolver2D(ctx)
        for name, values in f.items():
            try:
                ref.set_field(capi2d.FIELD[name], values)
            except RuntimeError:
                pass          # a buffer the reference does not allocate for this scheme
    n = ctx.NX * ctx.NZ
    ours_buf = torch.zeros(4 * n, dtype=torch.uint8, device="cuda")
    ref_buf = torch.zeros(4 * n, dtype=torch.uint8, device="cuda")
    try:
        for comp in range(8):
            peak = float(np.abs(component_values(f, scheme, comp)).max()) * BALANCE.get(comp, 1.0)
            for scale in (0.7 / max(peak, 1e-30), 4.0 / max(peak, 1e-30)):
                torch.cuda.synchronize()
                seis2d.generateWavefieldTextureOnGpu(gpu, ours_buf.data_ptr(), scale, comp)
                seis2d.synchronize(gpu)
                ours = ours_buf.cpu().numpy().reshape(ctx.NZ, ctx.NX, 4)
                want = texture_numpy(f, scheme, scale, comp)
                diff = np.abs(ours.astype(int) - want.astype(int))
                assert diff.max() <= 1 and (diff == 0).mean() >= 0.999, (comp, diff.max(), (diff == 0).mean())
                if comp < 7:
                    assert len(np.unique(ours[..., 1])) > 16          # a picture, not a flat colour
                else:
                    assert np.all(ours == 255)                        # unknown component: white
                if ref is not None:
                    ref.texture(ref_buf.data_ptr(), scale, comp)
                    assert np.array_equal(ours, ref_buf.cpu().numpy().reshape(ctx.NZ, ctx.NX, 4)), comp
    finally:
        if ref is not None:
            ref.close()
        seis2d.releaseGpuSimulation(gpu)


def test_texture_argument_checks(solver2d_lib, cuda_device):
    from cuda.bindings import runtime as rt
    ctx = make_context(1)
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    n = ctx.NX * ctx.NZ
    err, small = rt.cudaMalloc(4 * n - 4)
    assert err == rt.cudaError_t.cudaSuccess
    err, exact = rt.cudaMalloc(4 * n + 4)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        seis2d.generateWavefieldTextureOnGpu(gpu, int(exact), 1.0, 0)
        seis2d.synchronize(gpu)
        with pytest.raises(seis2d.InvalidArgument):          # one pixel short
            seis2d.generateWavefieldTextureOnGpu(gpu, int(small), 1.0, 0)
        with pytest.raises(seis2d.InvalidArgument):          # misaligned
            seis2d.generateWavefieldTextureOnGpu(gpu, int(exact) + 2, 1.0, 0)
        host = np.zeros(4 * n, np.uint8)
        with pytest.raises(seis2d.InvalidArgument):          # host memory
            seis2d.generateWavefieldTextureOnGpu(gpu, host.ctypes.data, 1.0, 0)
    finally:
        rt.cudaFree(small)
        rt.cudaFree(exact)
        seis2d.releaseGpuSimulation(gpu)
    with pytest.raises(seis2d.LogicError):                    # released session
        seis2d.generateWavefieldTextureOnGpu(gpu, 0, 1.0, 0)
