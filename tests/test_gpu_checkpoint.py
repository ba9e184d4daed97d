"""Shot restart (seis3d_save/load_checkpoint, seis3d_write/read_checkpoint): a run restored from
a checkpoint continues bit-identically, across the pitched and unpitched row layouts and
through a file, with FP32 or BF16 CPML memories; checkpoints of another grid or storage mode,
truncated data and a restore under an active gather are refused without touching the
session."""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

FIRST, REST = 40, 30


def session(shot, compact=False, storage=capi.STORAGE_FP32):
    s = seis3d.Session(shot.context, compact_rows=compact, storage=storage)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    return s


def finish(s, shot):
    s.gather_begin(1, REST)
    s.run_steps(shot.source, FIRST, REST)
    g = s.gather_fetch()
    f = [s.field(k) for k in range(9)]
    return g, f


def test_restart_is_bit_identical(tmp_path, cuda_device):
    # gx = 44 + 2*8 + 8 = 68: pitched rows of 96 floats, unpitched rows of 68.
    shot = models3d.small_shot(nx=44, ny=30, nz=34, steps=FIRST + REST)
    a = session(shot)
    a.run_steps(shot.source, 0, FIRST)
    data = a.save_checkpoint()
    path = tmp_path / "shot.s3dstate"
    a.write_checkpoint(path)
    assert path.read_bytes() == data and not (tmp_path / "shot.s3dstate.part").exists()
    want_g, want_f = finish(a, shot)
    a.release()
    for restore in ("bytes", "file"):
        for compact in (False, True):
            b = session(shot, compact)
            if restore == "bytes":
                b.load_checkpoint(data)
            else:
                b.read_checkpoint(path)
            g, f = finish(b, shot)
            b.release()
            assert np.array_equal(g, want_g), (restore, compact)
            for k in range(9):
                assert np.array_equal(f[k], want_f[k]), (restore, compact, k)


def test_checkpoint_refusals(tmp_path, cuda_device):
    shot = models3d.small_shot(nx=40, ny=32, nz=36, steps=10)
    a = session(shot)
    a.run_steps(shot.source, 0, 10)
    data = a.save_checkpoint()
    before = [a.field(k) for k in range(9)]
    other = session(models3d.small_shot(nx=40, ny=32, nz=38, steps=10))
    with pytest.raises(seis3d.InvalidArgument):
        other.load_checkpoint(data)
    with pytest.raises(seis3d.InvalidArgument):
        a.load_checkpoint(data[:-4])
    with pytest.raises(seis3d.InvalidArgument):
        a.load_checkpoint(b"XXXXXXXX" + data[8:])
    (tmp_path / "short").write_bytes(data[: len(data) // 2])
    with pytest.raises(seis3d.InvalidArgument):
        a.read_checkpoint(tmp_path / "short")
    a.gather_begin(1, 4)
    with pytest.raises(seis3d.LogicError):
        a.load_checkpoint(data)
    a.gather_end()
    for k in range(9):
        assert np.array_equal(a.field(k), before[k])
    a.release()
    other.release()


def test_bf16_memory_checkpoint(cuda_device):
    """A session with BF16 CPML memories checkpoints its 2-byte memories (half the bytes of the
    FP32 memories), restarts bit-identically, and its checkpoints do not restore into an FP32
    session (nor the other way round)."""
    shot = models3d.small_shot(nx=44, ny=30, nz=34, steps=FIRST + REST)
    a = session(shot, storage=capi.STORAGE_BF16_CPML)
    a.run_steps(shot.source, 0, FIRST)
    data = a.save_checkpoint()
    want_g, want_f = finish(a, shot)
    a.release()
    plain = session(shot)
    plain.run_steps(shot.source, 0, FIRST)
    plain_data = plain.save_checkpoint()
    c = shot.context
    p = c.pml3D
    memories = 6 * (c.gz3D * c.gy3D * 2 * p + c.gz3D * 2 * p * c.gx3D + (1 if c.freeSurface3D else 2) * p * c.gy3D * c.gx3D)
    assert len(plain_data) - len(data) == 2 * memories       # unpitched rows, 4 vs 2 bytes
    with pytest.raises(seis3d.InvalidArgument, match="storage mode"):
        plain.load_checkpoint(data)
    plain.release()
    for compact in (False, True):
        b = session(shot, compact, storage=capi.STORAGE_BF16_CPML)
        with pytest.raises(seis3d.InvalidArgument, match="storage mode"):
            b.load_checkpoint(plain_data)
        b.load_checkpoint(data)
        g, f = finish(b, shot)
        b.release()
        assert np.array_equal(g, want_g), compact
        for k in range(9):
            assert np.array_equal(f[k], want_f[k]), (compact, k)
