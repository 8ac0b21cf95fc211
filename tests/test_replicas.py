"""The multi-process (one rank per GPU) path of the bench and the library on
CPU: gloo ranks, world size 2 (no GPU). The path has no data-path
collective; what crosses ranks is a barrier and the maximum of the ranks'
times, and the reference arm runs on rank 0 alone."""
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


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from illuminaprt_b200 import replicas
    replicas.init("gloo", timeout_s=60)
    assert replicas.rank_info() == (world, rank, rank)
    replicas.barrier()
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    slowest = replicas.max_over_ranks(ms)
    rate = replicas.aggregate_rate(1000, world, slowest / 1e3)
    out.put((rank, slowest, rate))
    replicas.finish()


def test_max_over_ranks_and_aggregate_rate_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [20.0, 20.0]  # both ranks see the slowest time
    assert res[0][2] == pytest.approx(2 * 1000 / 0.020)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libilref.so")),
                    reason="reference engine library not built")
def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    env = dict(os.environ, PYTHONPATH=ROOT)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--ref-seconds", "2"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"
