"""The multi-GPU form of the benchmark is replicas only (no data-path
collective): each rank renders its own frame and only the timing is reduced.
These run the reduction and the reference arm's multi-rank launch as two
`gloo` ranks on the CPU."""
import os
import pathlib
import socket
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slowest = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
    thr = bench.replica_throughput(1_000_000, 3, world, slowest)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, slowest, thr))


def test_max_over_ranks_and_replica_throughput_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [20.0, 20.0]          # max over ranks
    assert out[0][2] == pytest.approx(1e6 * 3 * 2 / 0.020 / 1e6)  # both replicas' rays over the slowest time


def test_reference_arm_under_torchrun_two_ranks():
    """Rank 0 alone times the reference CPU path and prints one line; rank 1 exits 0."""
    import oracle as O
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--scene", "box", "--spp", "1", "--bounces", "0",
           "--cpu-row-step", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    import json
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
