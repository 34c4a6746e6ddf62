"""The multi-process path of bench.py, on CPU with world size 2 over gloo.

The implicit path does not shard: `bench.py --gpus N` runs N independent
replicas. Its only collectives are the barrier around the timed region and
the max over ranks of the device time. Under torchrun, the reference arm
runs on rank 0 alone and the other ranks exit 0 without work. CPU only.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank: int, port: int, outdir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2", LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    ws, r, _ = bench.dist_setup()
    assert (ws, r) == (2, rank)
    bench.dist_barrier(ws)
    m = bench.dist_max(10.0 * (rank + 1), ws)
    bench.dist_barrier(ws)
    Path(outdir, f"rank{rank}").write_text(repr(m))
    dist.destroy_process_group()


def test_max_over_ranks_over_gloo(tmp_path):
    mp.start_processes(_replica, args=(_free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    assert [float(Path(tmp_path, f"rank{r}").read_text()) for r in range(2)] == [20.0, 20.0]


def test_reference_arm_prints_one_line_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--cpu-n", "6"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
