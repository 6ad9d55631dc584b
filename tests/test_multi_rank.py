"""The N>1 plumbing of bench.py on CPU: world_size-2 process groups over
gloo.  The frame path does not shard (each GPU runs an independent replica
of the workload), so the only cross-rank steps are the reductions of the
timed results: the slowest rank's time for the device-timed and end-to-end
rates, the sum of per-rank rates for the serving workload."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", init_method="env://",
                            timeout=datetime.timedelta(seconds=60))
    try:
        w, r, loc = bench._dist()
        ms = [120.0, 150.0][rank]  # rank 1 is the slow one
        total_ms = bench.reduce_over_ranks(ms, "max")
        e2e_s = bench.reduce_over_ranks([0.40, 0.35][rank], "max")
        serve = bench.reduce_over_ranks([1000.0, 1250.5][rank], "sum")
        value = bench.job_rate(2_000_000, 10, w, total_ms * 1e-3)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
            json.dump(dict(world=w, rank=r, local=loc, total_ms=total_ms, e2e_s=e2e_s,
                           serve=serve, value=value), fh)
    finally:
        dist.destroy_process_group()


def test_reductions_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, g in enumerate(got):
        assert (g["world"], g["rank"], g["local"]) == (2, r, r)
        assert g["total_ms"] == 150.0          # slowest rank's device time
        assert g["e2e_s"] == 0.40              # slowest rank's end-to-end time
        assert g["serve"] == 2250.5            # serving: rates add up
        # 2 replicas x 10 steps x 2M rays in 150 ms
        assert g["value"] == pytest.approx(2 * 10 * 2_000_000 / 0.150 / 1e6)


def test_reduction_without_a_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(3.5, "max") == 3.5
    assert bench.reduce_over_ranks(3.5, "sum") == 3.5
    assert bench.job_rate(1_000_000, 4, 1, 2.0) == 2.0


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the reference arm; rank 1 exits 0
    without output and without touching the reference library."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1",
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
