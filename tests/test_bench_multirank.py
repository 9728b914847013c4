"""The multi-process paths of bench.py on CPU: the max-over-ranks timing reduction with two gloo
ranks, and the reference arm launched as two ranks (rank 0 runs and prints one JSON line, rank 1
exits without work)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out_q.put((rank, bench.max_over_ranks(1.5 + rank, dist, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}


def test_reference_arm_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--rings", "2",
           "--layers", "6"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 1 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["parallelism"] == "replicas x2" and "BiCGSTAB pressure" in d["solver"]


def test_reference_arm_maps_no_product_library():
    """The reference arm builds its mesh with the oracle's mesher: the process never maps the
    product's libcfsa.so, and it runs the same warm-up as the GPU arm."""
    code = (
        "import sys, json, io, contextlib; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
        "'--warmup', '5', '--rings', '2', '--layers', '6', '--reference-single-core-steps', '1']; "
        "sys.path.insert(0, '.'); import bench; buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf): bench.main()\n"
        "maps = open('/proc/self/maps').read(); d = json.loads(buf.getvalue())\n"
        "print(json.dumps({'libcfsa': 'libcfsa' in maps, 'oracle': 'liboracle_ns' in maps, "
        "'cfsa_module': 'cfsa_b200' in sys.modules, 'warmup': d['warmup'], "
        "'single': d['cpu_baseline']['single_core']['cores']}))"
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       cwd=str(ROOT), env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d == {"libcfsa": False, "oracle": True, "cfsa_module": False, "warmup": 5, "single": 1}
