"""Survey driver: the reference's shot-sequence, receiver-mesh and gather rules
(src/Seis3D/Acquisition3D.cpp:21-37,188-243) and the sharding of a survey's shots over ranks,
checked on the CPU with two gloo ranks (the oracle stands in for each rank's GPU)."""
import multiprocessing as mp
import os
import pickle
import socket

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import seis3d, survey
from survey_worker import (costs_for, oracle_group_runner, oracle_runner, tiny_setup, tiny_window_survey,
                           window_worker, worker)


def test_sequence_positions_and_spread_checks(solver_lib):
    c, q = tiny_setup()
    cells = [survey.sequence_shot(q, c, i) for i in range(survey.shot_count(q))]
    assert cells == [(4, 4, 4), (8, 4, 4), (12, 4, 4), (4, 9, 4), (8, 9, 4), (12, 9, 4)]
    with pytest.raises(ValueError):
        survey.sequence_shot(survey.Survey3D(shot_count=(4, 1), shot_spacing=(4, 1), shot_origin=(4, 4, 4)), c, 0)
    with pytest.raises(ValueError):
        survey.sequence_shot(survey.Survey3D(shot_count=(1, 1), shot_origin=(4, 4, 1)), c, 0)


def test_receiver_mesh_rules(solver_lib):
    c, q = tiny_setup()
    mesh = survey.receiver_mesh(q, c)
    assert mesh[:5] == [(1, 2, 0), (4, 2, 0), (7, 2, 0), (10, 2, 0), (1, 7, 0)] and len(mesh) == 8
    big = seis3d.validate_context3D(seis3d.default_context(nx3D=400, ny3D=300, nz3D=50, pml3D=8))
    with pytest.raises(ValueError):
        survey.receiver_mesh(survey.Survey3D(receiver_count=(301, 1), receiver_spacing=(1, 1)), big)
    with pytest.raises(ValueError):
        survey.receiver_mesh(survey.Survey3D(receiver_count=(20, 16), receiver_spacing=(1, 1)), big)
    with pytest.raises(ValueError):
        survey.receiver_mesh(survey.Survey3D(receiver_count=(4, 1), receiver_spacing=(6, 1), receiver_origin=(0, 0, 0)), c)


def test_gather_checks(solver_lib):
    c = seis3d.validate_context3D(seis3d.default_context())
    src = seis3d.default_source(x3D=10, y3D=10, z3D=10)
    survey.check_gather(c, src, 2, 1000, 150)
    for stride, samples in ((0, 10), (10001, 10), (1, 0), (1, 32768)):
        with pytest.raises(ValueError):
            survey.check_gather(c, src, stride, samples, 150)
    with pytest.raises(ValueError):  # interval above 32767 us
        survey.check_gather(c, src, int(32768 / (c.dt3D * 1e6)) + 1, 10, 150)
    with pytest.raises(ValueError):
        survey.check_gather(c, seis3d.default_source(x3D=10, y3D=10, z3D=1), 2, 10, 150)


def test_partition_is_balanced_and_deterministic():
    costs = [5, 1, 1, 3, 2, 2, 4]
    plan = survey.partition_shots(costs, 3)
    assert sorted(i for p in plan for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in plan]
    assert max(loads) - min(loads) <= max(costs)
    assert plan == survey.partition_shots(costs, 3)
    assert survey.partition_shots(costs, 1) == [list(range(len(costs)))]
    assert survey.partition_shots([1, 1], 4)[2:] == [[], []]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_process(tmp_path, solver_lib):
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    with open(os.path.join(tmp_path, "rank0.pkl"), "rb") as f:
        merged = pickle.load(f)
    with open(os.path.join(tmp_path, "rank1.pkl"), "rb") as f:
        assert pickle.load(f) is None

    c, q = tiny_setup()
    receivers = survey.receiver_mesh(q, c)
    single = survey.run_survey(q, c, oracle_runner(c, receivers), costs=costs_for(q, c))
    plan = survey.partition_shots(costs_for(q, c), 2)
    assert [r.index for r in merged] == list(range(survey.shot_count(q)))
    for r, s in zip(merged, single):
        assert r.source == s.source
        assert r.rank == (0 if r.index in plan[0] else 1)
        assert r.gather.shape == (6, len(receivers), 3) and np.abs(r.gather).max() > 0
        assert np.array_equal(r.gather, s.gather)
    assert {r.rank for r in merged} == {0, 1}


@pytest.mark.gpu
def test_gpu_runner_matches_oracle(solver_lib, cuda_device):
    # The product runner (one session per rank, model uploaded once, reset per shot) against
    # the oracle on the same uploaded model, shot by shot, within the FP32 trace tolerance of
    # the parity tests.
    import oracle
    c, q = tiny_setup()
    c = c.copy()
    c.modelKind3D = 3  # imported model
    c = seis3d.validate_context3D(c)
    receivers = survey.receiver_mesh(q, c)
    z = np.arange(c.nz3D, dtype=np.float32)[:, None, None]
    vp = np.broadcast_to(np.where(z < 7, 2400.0, 3300.0), (c.nz3D, c.ny3D, c.nx3D)).astype(np.float32)
    vs = (vp / np.float32(np.sqrt(3.0))).astype(np.float32)
    rho = (np.float32(310.0) * vp ** np.float32(0.25)).astype(np.float32)

    def oracle_run(index, cell):
        o = oracle.CpuOracle(c, 32)
        o.upload_model(vp, vs, rho)
        g = o.run_gather(seis3d.default_source(x3D=cell[0], y3D=cell[1], z3D=cell[2]), 0, 12, receivers, 2)
        o.close()
        return g.astype(np.float32)

    run = survey.gpu_runner(c, vp, vs, rho, seis3d.default_source(), 12, 2, receivers)
    results = survey.run_survey(q, c, run)
    expected = survey.run_survey(q, c, oracle_run)
    for r, e in zip(results, expected):
        assert r.gather.shape == e.gather.shape
        err = np.linalg.norm(r.gather - e.gather) / np.linalg.norm(e.gather)
        assert err < 1e-5, (r.index, err)
    run.session.release()


def test_windowed_survey_two_gloo_ranks_match_one_process(tmp_path, solver_lib):
    """Windowed shots (cropped windows of one model) sharded over two gloo ranks and run in
    groups of two: rank 0 ends with every shot, in survey order, bit-equal to one process."""
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=window_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    with open(os.path.join(tmp_path, "window_rank0.pkl"), "rb") as f:
        merged = pickle.load(f)
    with open(os.path.join(tmp_path, "window_rank1.pkl"), "rb") as f:
        assert pickle.load(f) is None
    q = tiny_window_survey()
    single = survey.run_window_survey(q, oracle_group_runner(q), batch=3)
    costs = [float(q.active_cells(s)) * q.steps for s in q.shots]
    plan = survey.partition_shots(costs, 2)
    assert [r.index for r in merged] == list(range(len(q.shots))) == [r.index for r in single]
    for r, s in zip(merged, single):
        assert r.rank == (0 if r.index in plan[0] else 1)
        assert r.extra["origin"] == q.shots[r.index].origin
        assert r.gather.shape == (q.steps // 2, len(q.receivers(q.shots[r.index])), 3)
        assert np.abs(r.gather).max() > 0
        assert np.array_equal(r.gather, s.gather)
    assert {r.rank for r in merged} == {0, 1}


@pytest.mark.gpu
def test_gpu_window_runner_matches_solo_sessions(solver_lib, cuda_device):
    """The batched group runner gives, shot by shot, the gathers of solo sessions."""
    q = tiny_window_survey()
    results = survey.run_window_survey(q, survey.gpu_window_runner(q), batch=4)
    for r in results:
        shot = q.shots[r.index]
        s = seis3d.Session(q.context(shot))
        s.upload_volumes(*q.window(shot))
        s.set_receivers(q.receivers(shot))
        s.gather_begin(2, q.steps // 2)
        s.run_steps(q.source(shot), 0, q.steps)
        solo = s.gather_fetch()
        s.release()
        assert np.array_equal(r.gather, solo), r.index
