"""Batched shots (seis3d_batch_*): shots of different grids stepped together in one graph
replay must give, shot by shot, exactly the fields and device gathers of solo
seis3d_run_steps runs (same launches, only their interleaving on the device differs), with
the tuner on or off, for any shots-per-launch and z chunk; and the batch checks its inputs."""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

STEPS = 150


def shots():
    return [models3d.small_shot(nx=40, ny=32, nz=36, steps=STEPS, seed=7),
            models3d.small_shot(nx=56, ny=24, nz=30, steps=STEPS, seed=8, layers=(1800, 2500), source=(20, 12, 9)),
            models3d.small_shot(nx=33, ny=41, nz=44, steps=STEPS, seed=9, free_surface=False,
                                kind=capi.SOURCE_FORCE)]


def prepared(shot):
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(1, STEPS)
    return s


def finish(s):
    g = s.gather_fetch()
    fields = [s.field(k) for k in range(9)]
    s.release()
    return g, fields


@pytest.fixture(scope="module")
def solo():
    out = []
    for shot in shots():
        s = prepared(shot)
        s.run_steps(shot.source, 0, STEPS)
        out.append(finish(s))
    return out


@pytest.mark.parametrize("options", [dict(tune=True), dict(shots_per_launch=1, z_chunk=16),
                                     dict(shots_per_launch=2, z_chunk=48)])
def test_batch_equals_solo_runs(solo, options, cuda_device):
    shot_list = shots()
    sessions = [prepared(shot) for shot in shot_list]
    batch = seis3d.Batch(sessions, **options)
    before = [s.views().kernelLaunches for s in sessions]
    # Two calls: the second continues the clock of the first.
    batch.run_steps([shot.source for shot in shot_list], 0, 100)
    batch.run_steps([shot.source for shot in shot_list], 100, STEPS - 100)
    batch.synchronize()
    info = batch.info()
    assert info["shots"] == 3
    if options.get("tune"):
        assert info["tuned"] and info["candidates"] == 10 and info["tuned_ms_per_step"] > 0
        assert info["z_chunk"] in (0, 16, 24, 32, 48) and info["shots_per_launch"] in (1, 3)
    else:
        assert not info["tuned"]
        assert info["z_chunk"] == options["z_chunk"] and info["shots_per_launch"] == options["shots_per_launch"]
    launched = [s.views().kernelLaunches - b for s, b in zip(sessions, before)]
    assert info["kernel_launches"] == sum(launched) and min(launched) >= 3 * STEPS
    batch.release()
    for (gather, fields), s in zip(solo, sessions):
        g, f = finish(s)
        assert np.array_equal(g, gather)
        for k in range(9):
            assert np.array_equal(f[k], fields[k]), k


def test_batch_argument_checks(cuda_device):
    shot_list = shots()[:2]
    sessions = [prepared(shot) for shot in shot_list]
    with pytest.raises(seis3d.InvalidArgument):
        seis3d.Batch([sessions[0], sessions[0]])
    with pytest.raises(seis3d.InvalidArgument):
        seis3d.Batch([])
    with pytest.raises(seis3d.InvalidArgument):
        seis3d.Batch(sessions, shots_per_launch=-1)
    batch = seis3d.Batch(sessions)
    bad = seis3d.default_source(x3D=0, y3D=1, z3D=5)
    with pytest.raises(seis3d.InvalidArgument):
        batch.run_steps([shot_list[0].source, bad], 0, 4)
    with pytest.raises(seis3d.InvalidArgument):
        batch.run_steps([shot_list[0].source], 0, 4)
    batch.run_steps([shot.source for shot in shot_list], 0, 4)
    batch.synchronize()
    sessions[1].release()
    with pytest.raises(seis3d.LogicError):
        batch.run_steps([shot.source for shot in shot_list], 4, 4)
    batch.release()
    sessions[0].release()


def test_tuned_session_equals_default(solo, cuda_device):
    """A session whose z chunk was tuned at initialisation computes the default session's bits."""
    shot = shots()[0]
    s = seis3d.Session(shot.context, tune=True)
    setting, planes = s.z_chunk()
    assert setting in (0, 16, 20, 24, 28, 32, 40) and planes > 0
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(1, STEPS)
    s.run_steps(shot.source, 0, STEPS)
    gather, fields = solo[0]
    g, f = finish(s)
    assert np.array_equal(g, gather)
    for k in range(9):
        assert np.array_equal(f[k], fields[k]), k
