"""The N > 1 path of bench.py on CPU: replicas only, so the one exchange is
the max over ranks of each timed interval (gloo stands in for NCCL), and
the reference arm under torchrun prints one line from rank 0 while the other
ranks exit without work."""
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


def _rank_main(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(values[rank], dist)
        rate = bench.whole_job_rate(1000, world, 10, ms)
        with open(os.path.join(out, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "rate": rate}, f)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_timing_is_the_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp
    values = [12.5, 40.0]
    mp.spawn(_rank_main, args=(2, _free_port(), values, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        got = json.load(open(tmp_path / f"rank{r}.json"))
        assert got["ms"] == 40.0
        assert got["rate"] == pytest.approx(1000 * 2 * 10 / 0.040)


def test_without_a_process_group_the_value_stands():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, None) == 3.25


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--particles", "4096",
           "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
