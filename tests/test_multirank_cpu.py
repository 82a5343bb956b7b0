"""The multi-rank path of bench.py on CPU with world size 2 (gloo): the
max-over-ranks device time, the whole-job value, and the reference arm
printing one line from rank 0 only under torchrun."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, ms, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    got = bench.max_over_ranks(ms[rank], device="cpu")
    out[rank] = (got, bench.whole_job_mlups(2, 1000, 10, got))
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        ms = [3.0, 7.5]
        port = free_port()
        procs = [ctx.Process(target=_rank, args=(r, port, ms, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            got, value = out[r]
            assert got == 7.5
            assert value == pytest.approx(2 * 1000 * 10 / 7.5e-3 / 1e6)


def test_reference_arm_prints_once_under_torchrun():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("port", "reference")
