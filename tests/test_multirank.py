"""The multi-rank path of bench.py on CPU: two gloo ranks (world size 2).

Every rank runs its own campaign: the same shapes, disjoint seeds, no
collective on the data path; the ranks meet only to take the slowest rank's
time, and the job's rate counts every rank's histories over that time.
"""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = bench.workload("campaign", rank)
        # each rank's time differs; every rank must see the largest
        slowest = bench.max_over_ranks(10.0 + rank, dist, "cpu")
        # a second collective in the same order on every rank
        again = bench.max_over_ranks(-float(rank), dist, "cpu")
        out.put((rank, list(cfg["seeds"]), [tuple(d) for d in cfg["dims"]], slowest, again))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_own_disjoint_campaigns_and_agree_on_the_slowest_time():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, seeds0, dims0, slow0, again0), (r1, seeds1, dims1, slow1, again1) = res
    assert dims0 == dims1 and len(dims0) == 64
    assert not set(seeds0) & set(seeds1)
    assert slow0 == slow1 == 11.0
    assert again0 == again1 == 0.0


def test_job_rate_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(2, 64, 20, 1000.0) == pytest.approx(2 * 64 * 20)
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_the_reference_arm_runs_on_rank_0_only():
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_the_cpu_arms_schedule_the_whole_campaign_longest_first():
    sys.path.insert(0, ROOT)
    import bench
    # longest-first list scheduling: 3, 3 | 2 -> 5, 3 | 2 -> 5, 5 | 2 -> 7, 5
    assert bench.lpt_makespan([2, 3, 2, 3, 2], 2) == 7
    assert bench.lpt_makespan([1.0] * 8, 16) == 1.0
    assert bench.lpt_makespan([4.0, 1.0, 1.0, 1.0, 1.0], 2) == 4.0
    from cellweave_b200 import synthetic
    cfg = synthetic.campaign(per_size=3, sizes=(32, 48))
    v, detail, sample = bench.cpu_sample(cfg, 2)
    per = detail["seconds_per_mcs"]
    assert set(per) == {"32x32x1", "48x48x1"} and detail["sampled_histories"] == 6
    costs = [per["32x32x1"]] * 3 + [per["48x48x1"]] * 3
    assert v == pytest.approx(6 / bench.lpt_makespan(costs, 2), rel=0.02)  # the detail is rounded
    assert detail["makespan_s"] >= detail["serial_s"] / 2 - 1e-3
