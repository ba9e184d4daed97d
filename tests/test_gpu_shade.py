"""Display shading kernels (seis3d_shade_slices / seis3d_render_volume: the reference's
shaders/seis3d_slice.frag and shaders/seis3d_volume.frag as CUDA) against the CPU shader
oracle (oracle/seis3d_shade_oracle.cpp) on views extracted from a running shot.

Tolerances: the slice pass is per sample with no data-dependent control flow beyond the
shader's own selects, so FP32 colours agree to 2e-6 and RGBA8 to one step.  The volume pass
marches 192..1024 samples per ray with an early exit at 98 % opacity and a step count from
ceil(); FP32 contraction differences between the GPU and the CPU oracle can move a ray across
those thresholds, so at most 0.5 % of pixels may differ by more than 1e-3 and none by more
than 0.05."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

SLICE_TOL = 2e-6
VOLUME_TOL, VOLUME_OUTLIERS, VOLUME_MAX = 1e-3, 0.005, 0.05


@pytest.fixture(scope="module")
def shot_views():
    import torch
    shot = models3d.small_shot(steps=60)
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.run_steps(shot.source, 0, 60)
    c = s.context
    layout = seis3d.make_view_layout3D(c)
    slices = (c.nx3D // 2, c.ny3D // 2, shot.source.z3D)
    extracted = {}
    for component, boundary in ((0, False), (3, True)):
        buf = torch.zeros(2 * layout.totalSamples3D, dtype=torch.float32, device="cuda")
        stats = s.extract_views(buf.data_ptr(), layout, slices, component, 5, True, boundary)
        extracted[component] = (buf, stats)
    yield s, layout, extracted
    s.release()


def uniforms(s, layout, stats, component, **display):
    d = seis3d.default_display(component3D=component, scale3D=stats["velocity_maximum"],
                               materialRange3D=list(stats["material_range"]), **display)
    return seis3d.make_display_uniforms(s.context, layout, d)


def shade_slices(s, layout, buf, t, scale, gain, fmt):
    import torch
    n = layout.volumeOffset3D
    out = torch.zeros(n * (16 if fmt == capi.PIXELS_RGBA32F else 4), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()          # the buffer is ready before the session stream writes it
    s.shade_slices(layout, buf.data_ptr(), t, scale, gain, fmt, out.data_ptr())
    s.synchronize()                   # the kernel ran on the session stream
    host = out.cpu().numpy()
    return host.view(np.float32).reshape(n, 4) if fmt == capi.PIXELS_RGBA32F else host.reshape(n, 4)


def render(s, layout, buf, t, u, w, h, fmt):
    import torch
    out = torch.zeros(w * h * (16 if fmt == capi.PIXELS_RGBA32F else 4), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    s.render_volume(layout, buf.data_ptr(), t, u, w, h, fmt, out.data_ptr())
    s.synchronize()
    host = out.cpu().numpy()
    return host.view(np.float32).reshape(h, w, 4) if fmt == capi.PIXELS_RGBA32F else host.reshape(h, w, 4)


STYLES = [  # (display overrides, component)
    (dict(), 0),
    (dict(modelStyle3D=0, waveStyle3D=7, gain3D=2.5), 0),
    (dict(modelStyle3D=2, displayMode3D=1, waveGamma3D=0.5), 0),
    (dict(modelStyle3D=3, displayMode3D=2), 0),
    (dict(modelStyle3D=4, waveStyle3D=13, showBoundary3D=1), 3),
    (dict(modelStyle3D=3, waveStyle3D=4, showBoundary3D=1, volumeSizeCompensation3D=0, pan3D=[0.1, -0.05],
          yaw3D=-1.2, pitch3D=0.9, distance3D=2.4), 3),
]


@pytest.mark.parametrize("case", range(len(STYLES)))
def test_slices_match_oracle(shot_views, case, cuda_device):
    s, layout, extracted = shot_views
    display, component = STYLES[case]
    buf, stats = extracted[component]
    t, u, _, _ = uniforms(s, layout, stats, component, **display)
    views = buf.cpu().numpy().reshape(-1, 2)[:layout.volumeOffset3D]
    want = oracle.shade_slices(views, t, u.scale3D, u.gain3D)
    got = shade_slices(s, layout, buf, t, u.scale3D, u.gain3D, capi.PIXELS_RGBA32F)
    assert np.abs(got - want).max() <= SLICE_TOL
    got8 = shade_slices(s, layout, buf, t, u.scale3D, u.gain3D, capi.PIXELS_RGBA8)
    diff = np.abs(got8.astype(int) - oracle.to_rgba8(want).astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999
    # Something is actually drawn: the wave is visible on the slices.
    assert np.ptp(want[:, :3]) > 0.1


@pytest.mark.parametrize("case", range(len(STYLES)))
def test_volume_matches_oracle(shot_views, case, cuda_device):
    s, layout, extracted = shot_views
    display, component = STYLES[case]
    buf, stats = extracted[component]
    t, u, _, _ = uniforms(s, layout, stats, component, volumeRequestedWidth3D=192, volumeRequestedHeight3D=144,
                          **display)
    w, h = 192, 144
    texels = buf.cpu().numpy().reshape(-1, 2)[layout.volumeOffset3D:].reshape(
        layout.volumeZ3D, layout.volumeY3D, layout.volumeX3D, 2)
    want = oracle.render_volume(texels, t, u, w, h)
    got = render(s, layout, buf, t, u, w, h, capi.PIXELS_RGBA32F)
    err = np.abs(got - want).max(axis=-1)
    assert err.max() <= VOLUME_MAX, err.max()
    assert (err > VOLUME_TOL).mean() <= VOLUME_OUTLIERS, (err > VOLUME_TOL).mean()
    got8 = render(s, layout, buf, t, u, w, h, capi.PIXELS_RGBA8)
    diff = np.abs(got8.astype(int) - oracle.to_rgba8(want).astype(int)).max(axis=-1)
    assert diff.max() <= round(VOLUME_MAX * 255) and (diff <= 1).mean() >= 1 - VOLUME_OUTLIERS
    assert np.ptp(want[..., :3]) > 0.05
    # The same launch twice gives the same pixels.
    assert np.array_equal(got, render(s, layout, buf, t, u, w, h, capi.PIXELS_RGBA32F))


def test_shading_argument_checks(shot_views, cuda_device):
    from cuda.bindings import runtime as rt
    s, layout, extracted = shot_views
    buf, stats = extracted[0]
    t, u, _, _ = uniforms(s, layout, stats, 0)
    n = layout.volumeOffset3D
    # Exact allocations (torch's caching allocator hands out pieces of larger segments, which
    # the range check rightly accepts).
    err, out = rt.cudaMalloc(4 * n)
    assert err == rt.cudaError_t.cudaSuccess
    err, views = rt.cudaMalloc(8 * n)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        out, views = int(out), int(views)
        s.shade_slices(layout, views, t, 1.0, 1.0, capi.PIXELS_RGBA8, out)        # slices only: fits
        with pytest.raises(seis3d.InvalidArgument):      # unknown pixel format
            s.shade_slices(layout, views, t, 1.0, 1.0, 7, out)
        with pytest.raises(seis3d.InvalidArgument):      # RGBA32F needs 16 bytes per pixel
            s.shade_slices(layout, views, t, 1.0, 1.0, capi.PIXELS_RGBA32F, out)
        with pytest.raises(seis3d.InvalidArgument):      # misaligned output
            s.shade_slices(layout, views, t, 1.0, 1.0, capi.PIXELS_RGBA8, out + 2)
        with pytest.raises(seis3d.InvalidArgument):      # the views hold no volume
            s.render_volume(layout, views, t, u, 8, 8, capi.PIXELS_RGBA8, out)
        for w, h in ((0, 10), (10, 0), (capi.MAX_VOLUME_OUTPUT + 1, 4)):
            with pytest.raises(seis3d.InvalidArgument):
                s.render_volume(layout, buf.data_ptr(), t, u, w, h, capi.PIXELS_RGBA8, out)
        host = np.zeros(4 * n, np.uint8)
        with pytest.raises(seis3d.InvalidArgument):      # host memory is not a device buffer
            s.shade_slices(layout, views, t, 1.0, 1.0, capi.PIXELS_RGBA8, host.ctypes.data)
        other = seis3d.make_view_layout3D(seis3d.validate_context3D(seis3d.default_context(nx3D=40, ny3D=40,
                                                                                          nz3D=40)))
        with pytest.raises(seis3d.InvalidArgument):      # a layout of another grid
            s.shade_slices(other, views, t, 1.0, 1.0, capi.PIXELS_RGBA8, out)
        s.synchronize()
    finally:
        rt.cudaFree(out)
        rt.cudaFree(views)
