"""The multi-rank path of bench.py on CPU (gloo, world size 2): the process
group set-up, the barrier and the max-over-ranks timing that the replica
benchmark uses, and the reference arm launched exactly as the driver launches
it (torch.distributed.run, one JSON line from rank 0, the other rank exits 0
without work).  The path does not shard: ranks are independent replicas."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    # every rank reports its own "time"; all must see the maximum
    got = bench.allmax(w, 1.5 + rank)
    import torch.distributed as dist

    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump({"allmax": got}, f)


def test_dist_helpers_world_size_2(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    for r in range(2):
        with open(tmp_path / ("rank%d.json" % r)) as f:
            assert json.load(f)["allmax"] == pytest.approx(2.5)


def test_reference_arm_under_torchrun_world_size_2():
    from oracle import pyoracle

    if not pyoracle.reference_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--size", "32", "--steps", "3", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
