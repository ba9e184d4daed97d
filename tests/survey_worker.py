"""Worker of the two-rank survey test: one gloo rank on the CPU that runs its share of a small
survey with the CPU oracle standing in for the GPU runner (test infrastructure only)."""
import datetime
import os
import pickle

import numpy as np


def tiny_setup():
    from cmakepro_cuda_seissim_v2_b200 import seis3d, survey

    c = seis3d.validate_context3D(seis3d.default_context(nx3D=16, ny3D=16, nz3D=16, pml3D=8, freeSurface3D=1))
    q = survey.Survey3D(receiver_count=(4, 2), receiver_spacing=(3, 5), receiver_origin=(1, 2, 0),
                        shot_count=(3, 2), shot_spacing=(4, 5), shot_origin=(4, 4, 4))
    return c, q


def oracle_runner(context, receivers, steps=12, stride=2):
    import oracle
    from cmakepro_cuda_seissim_v2_b200 import seis3d

    def run(index, cell):
        o = oracle.CpuOracle(context, 32, threads=1)
        o.generate()
        src = seis3d.default_source(x3D=cell[0], y3D=cell[1], z3D=cell[2])
        g = o.run_gather(src, 0, steps, receivers, stride)
        o.close()
        return g.astype(np.float32)

    return run


def costs_for(q, context):
    # Uneven costs so the plan is not a plain round robin.
    from cmakepro_cuda_seissim_v2_b200 import survey
    return [1.0 + (i % 3) for i in range(survey.shot_count(q))]


def worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from cmakepro_cuda_seissim_v2_b200 import survey

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c, q = tiny_setup()
        receivers = survey.receiver_mesh(q, c)
        results = survey.run_survey(q, c, oracle_runner(c, receivers), costs=costs_for(q, c), rank=rank,
                                    world=world, dist=dist)
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump(results, f)
    finally:
        dist.destroy_process_group()


def tiny_window_survey():
    from cmakepro_cuda_seissim_v2_b200 import models3d

    return models3d.window_survey(shots=6, steps=12, nx=48, ny=32, nz=40, window_range=(20, 30), pml=8,
                                  source_depth=4)


def oracle_group_runner(survey, stride=2):
    """Group runner with the CPU oracle standing in for the GPU batch: each shot of the group
    on its window, one after another."""
    import oracle

    def run(group):
        out = []
        for i in group:
            shot = survey.shots[i]
            o = oracle.CpuOracle(survey.context(shot), 32, threads=1)
            o.upload_model(*survey.window(shot))
            g = o.run_gather(survey.source(shot), 0, survey.steps, survey.receivers(shot), stride)
            o.close()
            out.append(g.astype(np.float32))
        return out

    return run


def window_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from cmakepro_cuda_seissim_v2_b200 import survey

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        q = tiny_window_survey()
        results = survey.run_window_survey(q, oracle_group_runner(q), batch=2, rank=rank, world=world, dist=dist)
        with open(os.path.join(out_dir, f"window_rank{rank}.pkl"), "wb") as f:
            pickle.dump(results, f)
    finally:
        dist.destroy_process_group()
