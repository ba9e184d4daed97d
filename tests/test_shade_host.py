"""Display shading on the host (no GPU): the palette table and display defaults against the
reference's own headers (tests/golden/display_reference.json, made by
tests/golden/make_display_golden.py), the uniform derivation of Renderer3D
(src/Seis3D/Renderer3D.cpp:148-160, 224-267) restated here in float32, and known answers of
the CPU shader oracle (oracle/seis3d_shade_oracle.cpp)."""
import json
import math
import os

import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, seis3d

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "display_reference.json")))
F = np.float32


def test_palettes_match_reference_table():
    for style, stops in enumerate(GOLDEN["palettes"]):
        np.testing.assert_array_equal(seis3d.wave_palette(style), np.array(stops, np.float32))
    # Styles outside 0..13 clamp (WavePalettes.h:27).
    np.testing.assert_array_equal(seis3d.wave_palette(-3), seis3d.wave_palette(0))
    np.testing.assert_array_equal(seis3d.wave_palette(99), seis3d.wave_palette(13))


def test_display_defaults_match_reference_state():
    d = seis3d.default_display()
    for name, value in GOLDEN["state_defaults"].items():
        got = getattr(d, name)
        if isinstance(value, list):
            np.testing.assert_array_equal(np.array(got[:], np.float32), np.array(value, np.float32), err_msg=name)
        else:
            assert F(got) == F(value), name
    assert capi.MAX_VOLUME_OUTPUT == GOLDEN["limits"]["maxVolumeOutput3D"]
    assert capi.MAX_VOLUME_AXIS == GOLDEN["limits"]["maxVolumeAxis3D"]


def restated_uniforms(c, layout, d):
    """Renderer3D's arithmetic, in float32 and in its order."""
    width = min(max(d.volumeRequestedWidth3D, 1), 1536)
    height = min(max(d.volumeRequestedHeight3D, 1), 1536)
    physical = [c.nx3D, c.ny3D, c.nz3D]
    visible, low, high = [], [], []
    for a in range(3):
        n, offset = F(layout.domainSize3D[a]), F(-layout.domainOrigin3D[a])
        visible.append(n if d.showBoundary3D else F(physical[a]))
        low.append(offset / n)
        high.append((offset + F(physical[a])) / n)
    extent = max(visible)
    rng = d.materialRange3D if d.materialRangeAuto3D else d.manualMaterialRange3D
    scale = F(d.scale3D) if math.isfinite(d.scale3D) and F(d.scale3D) > F(1e-12) else F(1e-12)
    return {
        "width": width, "height": height, "aspect3D": F(width) / F(height),
        "domainLow3D": [F(0) if d.showBoundary3D else v for v in low],
        "domainHigh3D": [F(1) if d.showBoundary3D else v for v in high],
        "physicalLow3D": low, "physicalHigh3D": high,
        "extent3D": [visible[0] / extent, visible[2] / extent, visible[1] / extent],
        "opticalScale3D": max(F(1), extent / F(96)) if d.volumeSizeCompensation3D else F(1),
        "scale3D": max(scale, F(1e-12)),
        "materialRange3D": [F(rng[0]), max(F(rng[0]), F(rng[1]))],
        "unsignedWave3D": int(d.component3D == 3),
    }


CONTEXTS = {
    "free-surface": dict(nx3D=300, ny3D=50, nz3D=300, freeSurface3D=1, pml3D=20),
    "six-face": dict(nx3D=120, ny3D=90, nz3D=200, freeSurface3D=0, pml3D=12),
    "reflecting": dict(nx3D=64, ny3D=64, nz3D=48, freeSurface3D=0, reflecting3D=1, pml3D=10),
}
DISPLAYS = {
    "defaults": dict(),
    "boundary": dict(showBoundary3D=1, scale3D=3.5e-7, component3D=3),
    "manual-range": dict(materialRangeAuto3D=0, manualMaterialRange3D=[4000.0, 1800.0], volumeSizeCompensation3D=0),
    "clamped-target": dict(volumeRequestedWidth3D=0, volumeRequestedHeight3D=4000, scale3D=float("nan")),
}


@pytest.mark.parametrize("ctx", list(CONTEXTS))
@pytest.mark.parametrize("disp", list(DISPLAYS))
def test_display_uniforms_match_renderer(ctx, disp):
    c = seis3d.validate_context3D(seis3d.default_context(**CONTEXTS[ctx]))
    layout = seis3d.make_view_layout3D(c)
    d = seis3d.default_display(**DISPLAYS[disp])
    t, u, w, h = seis3d.make_display_uniforms(c, layout, d)
    want = restated_uniforms(c, layout, d)
    assert (w, h) == (want["width"], want["height"])
    for key in ("domainLow3D", "domainHigh3D", "physicalLow3D", "physicalHigh3D", "extent3D"):
        np.testing.assert_array_equal(np.array(getattr(u, key)[:], np.float32), np.array(want[key], np.float32), key)
    for key in ("aspect3D", "opticalScale3D", "scale3D"):
        assert F(getattr(u, key)) == want[key], key
    np.testing.assert_array_equal(np.array(t.materialRange3D[:], np.float32), np.array(want["materialRange3D"]))
    assert t.unsignedWave3D == want["unsignedWave3D"]
    np.testing.assert_array_equal(np.array(t.palette3D[:], np.float32).reshape(5, 3), seis3d.wave_palette(d.waveStyle3D))
    assert (u.yaw3D, u.pitch3D, u.distance3D) == (d.yaw3D, d.pitch3D, d.distance3D)
    assert (u.opacity3D, u.threshold3D, u.gain3D) == (d.volumeOpacity3D, d.volumeThreshold3D, d.gain3D)


def test_display_uniforms_reject_foreign_layout():
    a = seis3d.validate_context3D(seis3d.default_context(**CONTEXTS["six-face"]))
    b = seis3d.validate_context3D(seis3d.default_context(**CONTEXTS["reflecting"]))
    with pytest.raises(seis3d.InvalidArgument):
        seis3d.make_display_uniforms(a, seis3d.make_view_layout3D(b), seis3d.default_display())


# ---- known answers of the shader oracle -------------------------------------------------

def transfer(**overrides):
    c = seis3d.validate_context3D(seis3d.default_context(**CONTEXTS["six-face"]))
    t, u, _, _ = seis3d.make_display_uniforms(c, seis3d.make_view_layout3D(c), seis3d.default_display())
    for k, v in overrides.items():
        field = getattr(t, k)
        if hasattr(field, "__len__"):
            for i, x in enumerate(v):
                field[i] = x
        else:
            setattr(t, k, v)
    return t, u


def lerp(a, b, f):
    return np.asarray(a, np.float64) * (1 - f) + np.asarray(b, np.float64) * f


def test_slice_known_answers():
    t, _ = transfer(modelStyle3D=2, materialRange3D=[1000.0, 3000.0])
    brightness, opacity = t.materialBrightness3D, t.waveOpacity3D
    pal = np.array(t.palette3D[:], np.float64).reshape(5, 3)
    views = np.array([[0.0, 1000.0],      # no wave, lowest material: grey .12 x brightness
                      [0.0, 3000.0],      # highest material: grey .85 x brightness
                      [1e-9, 2000.0],     # below the wave threshold: material only
                      [5.0, 2000.0],      # clamped to +1: full visibility, last palette stop
                      [-5.0, 2000.0]], np.float32)  # -1: first stop
    out = oracle.shade_slices(views, t, scale=1.0, gain=1.0).astype(np.float64)
    grey = lambda g: np.array([g, g, g]) * brightness  # noqa: E731
    np.testing.assert_allclose(out[0, :3], grey(.12), atol=1e-6)
    np.testing.assert_allclose(out[1, :3], grey(.85), atol=1e-6)
    np.testing.assert_allclose(out[2, :3], grey(lerp(.12, .85, .5)), atol=1e-6)
    np.testing.assert_allclose(out[3, :3], lerp(grey(lerp(.12, .85, .5)), pal[4], opacity), atol=1e-6)
    np.testing.assert_allclose(out[4, :3], lerp(grey(lerp(.12, .85, .5)), pal[0], opacity), atol=1e-6)
    assert np.all(out[:, 3] == 1)
    # Display mode 2 shows the material alone; mode 1 shows the wave over the plain background.
    t2, _ = transfer(modelStyle3D=2, materialRange3D=[1000.0, 3000.0], displayMode3D=2)
    np.testing.assert_allclose(oracle.shade_slices(views[3:4], t2, 1.0, 1.0)[0, :3], [lerp(.12, .85, .5)] * 3, atol=1e-6)
    t1, _ = transfer(displayMode3D=1)
    np.testing.assert_allclose(oracle.shade_slices(views[0:1], t1, 1.0, 1.0)[0, :3], [0.028, 0.045, 0.052], atol=1e-7)
    # A homogeneous model (zero range) maps to the middle of the style (transfer.glsl:20-21).
    t3, _ = transfer(modelStyle3D=0, materialRange3D=[2500.0, 2500.0], displayMode3D=2)
    np.testing.assert_allclose(oracle.shade_slices(views[0:1], t3, 1.0, 1.0)[0, :3],
                               lerp([.09, .13, .17], [.43, .53, .6], 0.5), atol=1e-6)


def test_volume_rays_that_miss_show_background():
    t, u = transfer()
    u.pan3D[0], u.pan3D[1] = 40.0, 40.0
    tex = np.zeros((4, 5, 6, 2), np.float32)
    img = oracle.render_volume(tex, t, u, 24, 16)
    np.testing.assert_array_equal(img[..., :3], np.broadcast_to(np.float32([0.025, 0.041, 0.05]), (16, 24, 3)))


def test_volume_uniform_material_follows_beer_lambert():
    """A one-pixel target looks straight at the box centre; with no wave and one material the
    composite is tint (1 - e^{-mL}) + background e^{-mL}, m = 3 x modelOpacity, L = chord."""
    t, u = transfer(modelStyle3D=2, materialRange3D=[1000.0, 3000.0])
    tex = np.zeros((6, 7, 8, 2), np.float32)
    tex[..., 1] = 1500.0
    img = oracle.render_volume(tex, t, u, 1, 1).astype(np.float64)[0, 0, :3]
    yaw, pitch, dist = u.yaw3D, u.pitch3D, u.distance3D
    forward = np.array([math.cos(pitch) * math.sin(yaw), math.sin(pitch), math.cos(pitch) * math.cos(yaw)])
    direction = -forward
    origin = dist * forward
    extent = np.array(u.extent3D[:], np.float64)
    t1, t2 = (-0.5 * extent - origin) / direction, (0.5 * extent - origin) / direction
    chord = np.min(np.maximum(t1, t2)) - max(np.max(np.minimum(t1, t2)), 0.0)
    transmittance = math.exp(-3 * t.modelOpacity3D * chord)
    tint = np.full(3, lerp(.12, .85, 0.25))
    want = tint * (1 - transmittance) + np.array([0.025, 0.041, 0.05]) * transmittance
    np.testing.assert_allclose(img, want, atol=2e-5)


def test_rgba8_rounding():
    x = np.array([[-1.0, 0.0, 0.5 / 255, 1.5 / 255], [0.5, 254.5 / 255, 1.0, 7.0]], np.float32)
    assert oracle.to_rgba8(x).tolist() == [[0, 0, 0, 2], [128, 254, 255, 255]]
