"""Multi-rank path of bench.py on the CPU: world size 2 over gloo.

bench.py runs one independent case per rank (replicas, no data-path
collective); its only collectives are the barriers around the timed regions
and the max over ranks of each region's time, so that the whole-job value
is set by the slowest replica.  These tests run that host-side logic with two
gloo ranks on 127.0.0.1, and the reference arm under torch.distributed.run,
where rank 0 alone times the CPU restatement and prints the one JSON line.
"""

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
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out.put((rank, [bench.max_over_ranks(v) for v in values[rank]]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_takes_the_slowest_replica():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    values = [[3.5, 10.0, 0.25], [7.0, 2.0, 0.5]]  # per rank: region times
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [max(a, b) for a, b in zip(*values)]
    assert got[0] == expect and got[1] == expect


def test_max_over_ranks_without_a_process_group_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(4.25) == 4.25


def test_reference_arm_prints_one_line_from_rank_zero():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="4")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-substeps", "2"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "port"


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
