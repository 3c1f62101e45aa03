"""Multi-process path on the CPU: two ranks over gloo (world size 2, rendezvous on 127.0.0.1).

Covers the replica plumbing the benchmark uses at N > 1 (process-group setup from the torchrun
environment, the barrier, the maximum over ranks, the whole-job figure) and a full two-rank launch
of `bench.py --impl reference` under torch.distributed.run, which must print exactly one line
(rank 0) while rank 1 exits cleanly.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    from tcscf_b200 import replicas

    r, w, local = replicas.env_ranks()
    backend = replicas.init(w, local, timeout_s=60, backend="gloo")
    try:
        replicas.barrier(w)
        # each rank times a different total; every rank must see the slowest one
        total_ms = 100.0 + 25.0 * r
        mx = replicas.max_over_ranks(total_ms, w)
        out.put((r, w, backend, mx, replicas.whole_job_seconds_per_build(mx, 4, w)))
    finally:
        replicas.finalize(w)


def test_max_over_ranks_gloo_world2():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for r, (rank, w, backend, mx, s) in enumerate(got):
        assert (rank, w, backend) == (r, world, "gloo")
        assert mx == 125.0                       # the slower rank's total
        assert s == pytest.approx(125.0 / 1e3 / (4 * world))


def test_single_process_is_identity():
    from tcscf_b200 import replicas

    assert replicas.init(1, 0) is None
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.whole_job_seconds_per_build(200.0, 4, 1) == pytest.approx(0.05)
    replicas.barrier(1)
    replicas.finalize(1)


def test_bench_reference_arm_two_ranks():
    """`bench.py --impl reference` launched as the N = 2 job is launched: rank 0 alone times the
    CPU reference and prints one JSON line; rank 1 does no work and exits 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--workload", "he",
           "--steps", "1", "--warmup", "0", "--ref-seconds", "0.2"]
    env = dict(os.environ, OMP_NUM_THREADS="2", CUDA_VISIBLE_DEVICES="")
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["unit"] == "s/iter"
    assert line["higher_is_better"] is False and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
