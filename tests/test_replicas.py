"""The multi-GPU path of bench.py on CPU: one replica per rank (the solve
does not shard), the job's step time is the slowest rank's, and the
reference arm runs on rank 0 only.  world_size 2 over gloo on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 10 + 5 r ms for its replica
        got = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        with open(tmp_path / f"rank{r}.json") as f:
            assert json.load(f)["max"] == 15.0


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs and prints the reference line."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_prints_the_benchmark_metric():
    """Rank 0 of the reference arm runs the reference PLASMA (oracle/_ref) and
    prints the same metric string as the GPU arm, on the same workload."""
    import bench
    from oracle import ref
    if not (os.path.exists(ref.LIB_PATH) or ref.available()):
        pytest.skip("reference library not built here")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--n", "512", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["info"] == 0 and line["iter"] >= 0
    assert line["value"] > 0
