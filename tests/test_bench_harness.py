"""The multi-rank harness of bench.py on CPU with gloo, world size 2: the
replica timing reduces to the slowest rank, and the reference arm under
torchrun prints one line from rank 0 while the other rank exits cleanly."""
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
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    v = bench.max_over_ranks(1.5 + rank, world, "cpu")
    out.put((rank, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(2))
    assert got == [(0, 2.5), (1, 2.5)]


def test_reference_arm_under_torchrun_world2():
    port = _free_port()
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--grid", "128", "--num-freq", "4", "--no-ref-gpu"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_roofline_numerator_of_the_headline():
    """The algorithmic bytes of one E pass at 256^3 FP32 (the roofline's
    numerator): 9 values per cell plus the psi read and write of the six
    CPML slabs, from the host-side plan (no GPU)."""
    sys.path.insert(0, ROOT)
    import bench
    import fdtd_b200 as F
    p = bench.workload_params(F, F.FDTD_FP32)
    d = F.plan(p)
    assert (d.nx, d.ny, d.nz) == (256, 256, 256)
    cells = 256 ** 3
    e = bench.pass_bytes(d, p, 4, "e")
    h = bench.pass_bytes(d, p, 4, "h")
    assert e == cells * 9 * 4 + 3 * (2 * 2 * 13 * 256 * 256 * 2 * 4)
    assert h == cells * 9 * 4 + 3 * (2 * 2 * 12 * 256 * 256 * 2 * 4)
    assert e == 685768704
