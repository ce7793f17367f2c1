"""The multi-rank path of bench.py on CPU: two ranks on the gloo backend
(127.0.0.1) stand in for the GPUs of a node.  Each rank runs its own
independent replica (no data-path collective); the whole-job figures are the
slowest rank's time and the units of all ranks, and only rank 0 reports."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: times (10 + r, 3 r) ms, 1000 (r + 1) units
        times, units = bench.job_totals(dist, "cpu", [10.0 + rank, 3.0 * rank], 1000 * (rank + 1))
        with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
            json.dump([times, units], f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_totals_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        times, units = json.load(open(tmp_path / ("rank%d.json" % r)))
        assert times == [11.0, 3.0]  # the slowest rank's time, per entry
        assert units == 3000.0       # 1000 + 2000: the units of both replicas


def test_job_totals_single_rank_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert bench.job_totals(None, "cpu", [4.5, 2.0], 77) == ([4.5, 2.0], 77.0)


@pytest.mark.parametrize("config", ["3", "4"])
def test_reference_arm_runs_on_rank_zero_only(config):
    # under torchrun every rank starts bench.py --impl reference; ranks other
    # than 0 exit at once, without work and without output
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="29999")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--config", config, "--steps", "2", "--warmup", "1"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_replicas_differ_by_rank():
    # each rank simulates its own seeded scene (weak scaling): the scenes
    # differ, so their particle counts may too, which is why units are summed
    from agimp import scenes
    a, b = scenes.make_config(3, seed=0, scale=0.3), scenes.make_config(3, seed=1, scale=0.3)
    assert a.n > 1000 and b.n > 1000
    assert a.x.shape != b.x.shape or not (a.x == b.x).all()
