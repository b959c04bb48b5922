"""The multi-GPU path of the benchmark on CPU: world size 2 over gloo (no GPU).

`bench.py --gpus N` runs one independent replica per rank; the process group carries only
the barriers and the max-over-ranks timing.  These tests run that logic with two gloo
processes, and the reference arm's rule that only rank 0 works and prints under torchrun.
"""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _, pg = bench.dist_setup(None, backend="gloo")
    try:
        bench.barrier_sync(pg)
        ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(pg, ms)
        bench.barrier_sync(pg)
        q.put((r, w, ms_max, bench.replica_rate(w, 64, 4, ms_max)))
    finally:
        pg.destroy_process_group()


def test_two_rank_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, ms_max, rate in got:
        assert w == 2 and ms_max == 15.0  # both ranks see the slowest rank's time
        assert rate == pytest.approx(2 * 64 ** 3 * 4 / 0.015 / 1e9)


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_runs_on_rank0_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                        "--steps", "4", "--warmup", "2"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr
    if rank == 0:
        sys.path.insert(0, ROOT)
        import bench
        line = json.loads(r.stdout.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
        # the driver's K and W, the same workload as the GPU arm, and a value consistent with
        # the timed samples (each one RK3 stage: N^3 / 3 grid-point * steps)
        assert line["steps"] == 4 and line["warmup"] == 2
        assert line["config"] == bench.workload_config(16, "fp32", 2)
        assert line["value"] == pytest.approx(16 ** 3 / 3 / (line["ms_per_step"] / 1e3) / 1e9, rel=1e-9)
        assert line["fp64_stage"]["value"] > 0
    else:
        assert r.stdout.strip() == ""
