"""3-D file formats on the CPU: .s3dm models (src/Seis3D/ModelIo3D.cpp:20-102) and SEG-Y rev1
gathers + geometry CSV (src/Seis3D/Acquisition3D.cpp:40-185), written by the library and read
back here by an independent parser that restates the reference's byte layout."""
import csv
import os
import struct

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, files3d, models3d, seis3d


def small_model(nx=20, ny=18, nz=16, free_surface=True):
    rng = np.random.default_rng(3)
    vp = (2000 + 1500 * rng.random((nz, ny, nx))).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = (np.float32(310) * vp ** np.float32(0.25)).astype(np.float32)
    c = models3d.imported_context(nx, ny, nz, 10.0, 8, free_surface, float(vp.max()), 15.0)
    return c, vp, vs, rho


# ---- .s3dm --------------------------------------------------------------------------------

def test_model_file_layout_and_round_trip(tmp_path, solver_lib):
    c, vp, vs, rho = small_model()
    path = tmp_path / "m.s3dm"
    files3d.write_model(path, c, vp, vs, rho)
    raw = path.read_bytes()
    assert raw[:8] == b"S3DMOD1\x00"
    version, nx, ny, nz, pml, boundary, spacing_bits = struct.unpack("<7I", raw[8:36])
    assert (version, nx, ny, nz, pml, boundary) == (1, c.nx3D, c.ny3D, c.nz3D, c.pml3D, 1)
    assert struct.unpack("<f", struct.pack("<I", spacing_bits))[0] == np.float32(c.spacing3D)
    assert len(raw) == 36 + nx * ny * nz * 3 * 4
    payload = np.frombuffer(raw[36:], dtype="<f4").reshape(nz, ny, nx, 3)
    assert np.array_equal(payload[..., 0], vp) and np.array_equal(payload[..., 2], rho)
    base = seis3d.default_context(frequency3D=15.0)
    back = files3d.inspect_model(path, base)
    assert (back.nx3D, back.ny3D, back.nz3D, back.pml3D) == (nx, ny, nz, pml)
    assert back.freeSurface3D == 1 and back.reflecting3D == 0 and back.modelKind3D == capi.MODEL_IMPORTED
    assert back.maxVp3D == np.float32(vp.max()) and back.gx3D == c.gx3D
    rvp, rvs, rrho = files3d.read_model(path, back)
    assert np.array_equal(rvp, vp) and np.array_equal(rvs, vs) and np.array_equal(rrho, rho)
    with pytest.raises(seis3d.InvalidArgument):  # never overwrite
        files3d.write_model(path, c, vp, vs, rho)
    assert not os.path.exists(str(path) + ".part")


def test_reflecting_model_uses_version_2(tmp_path, solver_lib):
    c, vp, vs, rho = small_model(free_surface=False)
    c.reflecting3D = 1
    c.freeSurface3D = 0
    files3d.write_model(tmp_path / "r.s3dm", c, vp, vs, rho)
    raw = (tmp_path / "r.s3dm").read_bytes()
    assert struct.unpack("<I", raw[8:12])[0] == 2 and struct.unpack("<I", raw[28:32])[0] == 2
    back = files3d.inspect_model(tmp_path / "r.s3dm", seis3d.default_context())
    assert back.reflecting3D == 1 and back.freeSurface3D == 0


def test_model_file_rejections(tmp_path, solver_lib):
    c, vp, vs, rho = small_model()
    good = tmp_path / "g.s3dm"
    files3d.write_model(good, c, vp, vs, rho)
    raw = good.read_bytes()
    base = seis3d.default_context()
    cases = {
        "magic": b"S3DMOD2\x00" + raw[8:],
        "version": raw[:8] + struct.pack("<I", 3) + raw[12:],
        "boundary": raw[:8] + struct.pack("<I", 1) + raw[12:28] + struct.pack("<I", 2) + raw[32:],
        "truncated": raw[:-4],
        "header": raw[:20],
    }
    bad_cell = bytearray(raw)
    bad_cell[36 + 4:36 + 8] = struct.pack("<f", 1e6)          # vs >= vp
    cases["material"] = bytes(bad_cell)
    for name, data in cases.items():
        p = tmp_path / f"{name}.s3dm"
        p.write_bytes(data)
        with pytest.raises(seis3d.SolverError):
            files3d.inspect_model(p, base)
    with pytest.raises(seis3d.SolverError):
        files3d.inspect_model(tmp_path / "missing.s3dm", base)
    tiny = raw[:12] + struct.pack("<III", 4, 4, 4) + raw[24:36]  # below the 16-node minimum
    (tmp_path / "tiny.s3dm").write_bytes(tiny + b"\0" * (4 * 4 * 4 * 12))
    with pytest.raises(seis3d.InvalidArgument):
        files3d.inspect_model(tmp_path / "tiny.s3dm", base)


# ---- SEG-Y ----------------------------------------------------------------------------------

def be16(b, o, signed=False):
    return struct.unpack(">h" if signed else ">H", b[o:o + 2])[0]


def be32(b, o):
    return struct.unpack(">i", b[o:o + 4])[0]


def make_gather(stride=2, samples=40, shot=7, world=(1000.0, 2000.0)):
    c = seis3d.validate_context3D(seis3d.default_context())
    src = seis3d.default_source(x3D=40, y3D=20, z3D=10, amplitude3D=2.5e8)
    q = files3d.default_survey()
    q.worldOrigin3D[0], q.worldOrigin3D[1] = world
    receivers = [(2 + 6 * i, 1 + 23 * j, 0) for j in range(3) for i in range(50)]
    g = files3d.Gather(c, src, receivers, stride, samples, shot_id=shot, survey=q)
    rng = np.random.default_rng(11)
    data = rng.standard_normal((samples, len(receivers), 3)).astype(np.float32) * np.float32(1e-3)
    g.set_samples(data)
    return c, src, q, receivers, g, data


def test_freeze_gather_metadata(solver_lib):
    c, src, q, receivers, g, _ = make_gather()
    assert g.sample_interval_us == round(float(c.dt3D) * 1e6) * 2
    assert g.first_sample_time == pytest.approx((2 - 0.5) * float(c.dt3D), rel=0, abs=0)
    assert g.coordinate_scalar == -1000
    # Large northings drop the scalar to keep integers in range (Acquisition3D.cpp:220-225).
    _, _, _, _, g2, _ = make_gather(world=(1.0e6, 3.0e6))
    assert g2.coordinate_scalar == -100
    # CMP bins: one-based, inline indexed by y, crossline by x (cmpBin3D).
    h = float(c.spacing3D)
    for r in receivers[:5] + receivers[-3:]:
        mx, my = 0.5 * (src.x3D + r[0]) * h, 0.5 * (src.y3D + r[1]) * h
        assert g.cmp_bin(r) == (int(np.floor(my / 25.0)) + 1, int(np.floor(mx / 25.0)) + 1)
    for stride, samples in ((0, 10), (2, 0), (2, 40000)):
        with pytest.raises(seis3d.SolverError):
            make_gather(stride=stride, samples=samples)


def test_segy_files_match_the_reference_layout(tmp_path, solver_lib):
    c, src, q, receivers, g, data = make_gather()
    g.export(tmp_path, "shotA")
    names = sorted(os.listdir(tmp_path))
    assert names == ["shotA_0007_geometry.csv", "shotA_0007_vx.sgy", "shotA_0007_vy.sgy", "shotA_0007_vz.sgy"]
    nr, ns = len(receivers), data.shape[0]
    h = float(c.spacing3D)
    sx, sy = 1000.0 + src.x3D * h, 2000.0 + src.y3D * h
    for component, suffix in enumerate(("vx", "vy", "vz")):
        b = (tmp_path / f"shotA_0007_{suffix}.sgy").read_bytes()
        assert len(b) == 3600 + nr * (240 + 4 * ns)
        text = b[:3200].decode("ascii")
        assert text[:4] == "C01 " and text[80:84] == "C02 " and text[3120:3124] == "C40 "
        assert text[4:68] == "SEIS3D ISOTROPIC ELASTIC COMMON-SHOT GATHER / SEG-Y REV1 / ASCII"
        assert text[84:96] == f"COMPONENT {suffix.upper()}"
        assert "XY SCALAR -1000" in text[160:240]
        assert f"FIRST VELOCITY SAMPLE TIME (S): {g.first_sample_time:f}" in text[400:480]
        bh = b[3200:3600]
        assert be32(bh, 0) == 1 and be32(bh, 4) == 1
        assert be16(bh, 12) == nr and be16(bh, 16) == g.sample_interval_us and be16(bh, 20) == ns
        assert be16(bh, 24) == 5 and be16(bh, 28) == 5 and be16(bh, 54) == 1
        assert be16(bh, 300) == 0x0100 and be16(bh, 302) == 1
        time_factor = 10000
        while time_factor > 1 and round(g.first_sample_time * 1000 * time_factor) > 32767:
            time_factor //= 10
        for r in (0, 1, 77, nr - 1):
            off = 3600 + r * (240 + 4 * ns)
            t = b[off:off + 240]
            gx, gy = 1000.0 + receivers[r][0] * h, 2000.0 + receivers[r][1] * h
            assert [be32(t, o) for o in (0, 4, 8, 12, 16, 20, 24)] == [r + 1, r + 1, 7, r + 1, 7, 7, r + 1]
            assert be16(t, 28) == (14, 13, 12)[component]
            assert be32(t, 36) == round(np.hypot(gx - sx, gy - sy))
            assert be32(t, 40) == round(-receivers[r][2] * h * 1000) and be32(t, 48) == round(src.z3D * h * 1000)
            assert be16(t, 68, True) == -1000 and be16(t, 70, True) == -1000
            assert [be32(t, o) for o in (72, 76, 80, 84)] == [round(v * 1000) for v in (sx, sy, gx, gy)]
            assert be16(t, 108) == round(g.first_sample_time * 1000 * time_factor)
            assert be16(t, 114) == ns and be16(t, 116) == g.sample_interval_us
            assert be32(t, 180) == round(0.5 * (sx + gx) * 1000) and be32(t, 184) == round(0.5 * (sy + gy) * 1000)
            assert (be32(t, 188), be32(t, 192)) == g.cmp_bin(receivers[r]) and be32(t, 196) == 7
            assert be16(t, 202) == 6 and be16(t, 210) == 6 and be16(t, 212) == r + 1
            assert be16(t, 214, True) == -time_factor
            trace = np.frombuffer(b[off + 240:off + 240 + 4 * ns], dtype=">f4")
            assert np.array_equal(trace, data[:, r, component])
    rows = list(csv.reader(open(tmp_path / "shotA_0007_geometry.csv")))
    assert rows[0][:3] == ["shot", "receiver", "sx_m"] and len(rows) == nr + 1
    assert rows[1][:2] == ["7", "1"] and float(rows[1][2]) == sx and float(rows[5][5]) == 1000.0 + receivers[4][0] * h
    assert int(rows[1][12]) == ns
    with pytest.raises(seis3d.SolverError):  # no overwrite of an existing shot
        g.export(tmp_path, "shotA")
    with pytest.raises(seis3d.SolverError):
        g.export(tmp_path, "bad/prefix")


def test_segy_refuses_non_finite_samples(tmp_path, solver_lib):
    _, _, _, _, g, data = make_gather()
    data = data.copy()
    data[3, 5, 1] = np.nan
    g.set_samples(data)
    with pytest.raises(seis3d.SolverError):
        g.write_segy(tmp_path / "x.sgy", 1)
    assert not os.path.exists(tmp_path / "x.sgy") and not os.path.exists(str(tmp_path / "x.sgy") + ".part")
    g.write_segy(tmp_path / "z.sgy", 2)   # the other components are fine
