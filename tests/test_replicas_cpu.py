"""The multi-rank path of bench.py on CPU: two gloo ranks run the replica
bookkeeping (exoplasim_b200/replicas.py) that bench.py uses under torchrun,
and bench.py's reference arm prints on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from exoplasim_b200 import replicas as RP
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = {"rank_world": RP.rank_world()}
        RP.barrier()
        out["max"] = RP.max_over_ranks(10.0 * (rank + 1))          # each rank's timed ms
        out["rate"] = RP.job_rate(8 * (rank + 1), out["max"])      # units over the slowest rank
        out["shard"] = list(RP.shard(11, rank, world))
        out["seed"] = RP.unit_seed(3, rank, 5)
        RP.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert res[r]["rank_world"] == (r, world)
        assert res[r]["max"] == 20.0                      # both ranks see the slowest
        assert res[r]["rate"] == pytest.approx((8 + 16) / 0.020)
    assert res[0]["shard"] + res[1]["shard"] == list(range(11))
    assert len(res[0]["shard"]) == 6 and len(res[1]["shard"]) == 5
    assert res[0]["seed"] != res[1]["seed"]


def test_single_process_is_a_no_op():
    from exoplasim_b200 import replicas as RP
    assert RP.rank_world() == (0, 1)
    RP.barrier()
    assert RP.max_over_ranks(3.5) == 3.5 and RP.job_rate(10, 500.0) == 20.0
    assert list(RP.shard(3, 2, 4)) == [2] and list(RP.shard(3, 3, 4)) == [] and list(RP.shard(5, 0, 1)) == list(range(5))
    with pytest.raises(ValueError):
        RP.shard(4, 2, 2)


def _bench_reference(rank):
    env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2")
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                           "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600,
                          cwd=ROOT)


def test_bench_reference_arm_prints_on_rank_zero_only():
    r1 = _bench_reference(1)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = _bench_reference(0)
    assert r0.returncode == 0, r0.stderr
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    for k in ("metric", "unit", "steps", "warmup", "ms_per_step", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    # both arms print one metric string and state the batch alike, so their lines compare
    import bench
    assert line["metric"] == bench.METRIC and line["unit"] == "round-trips/s"
    assert line["config"]["workload"] == bench.WORKLOAD and line["config"]["batch"] == bench.BATCH
