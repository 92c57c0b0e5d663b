"""The benchmark's multi-rank path on CPU: two gloo ranks for the
max-over-ranks timing, and a two-rank torchrun launch of the reference arm
(rank 0 alone runs and prints; the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (r + 1) s for the kernel and (10 - r) s end to end
        got = bench.max_over_ranks([rank + 1.0, 10.0 - rank], "cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: [2.0, 10.0], 1: [2.0, 10.0]}


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["unit"] == "GB/s" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def test_shard_bounds_balance_rows_within_one_system():
    import numpy as np
    from ginkgo_b200.batch import shard_bounds
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        sizes = rng.integers(32, 1025, size=500)
        offs = np.concatenate([[0], np.cumsum(sizes)])
        b = shard_bounds(offs, world)
        assert b[0] == 0 and b[-1] == len(sizes) and np.all(np.diff(b) >= 0)
        rows = np.diff(offs[b])
        assert abs(rows - offs[-1] / world).max() <= sizes.max()
    # more ranks than systems: the extra ranks own none
    b = shard_bounds([0, 10, 30], 4)
    assert b[0] == 0 and b[-1] == 2 and np.all(np.diff(b) >= 0)


def _sharded_main(rank, world, port, out):
    import datetime
    import types

    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from ginkgo_b200 import batch as B
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        host = types.SimpleNamespace(device=torch.device("cpu"))
        A, systems = B.convection_diffusion_batch(host, 9, lo=4, hi=30, seed=3)
        rng = np.random.default_rng(1)
        b = torch.from_numpy(rng.standard_normal(A.total_rows))
        x = torch.zeros_like(b)

        def dense_solve(A_loc, b_loc, x_loc):
            # host stand-in for the device solve: a dense solve per system
            xs, its = [], []
            for s, (rp, ci, v) in enumerate(A_loc.to_csr_list()):
                n = len(rp) - 1
                M = np.zeros((n, n))
                for r in range(n):
                    M[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
                o = int(A_loc.host_row_offsets[s])
                xs.append(np.linalg.solve(M, b_loc[o:o + n].numpy()))
                its.append(n)
            xl = torch.from_numpy(np.concatenate(xs)) if xs else x_loc
            return xl, torch.tensor(its, dtype=torch.int32), torch.zeros(len(its))

        xs, its, res = B.solve_sharded(A, b, x, host, local_solve=dense_solve)
        out.put((rank, xs.numpy().tolist(), its.tolist(), res.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batch_solve_sharded_over_gloo_ranks(world):
    import numpy as np
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sharded_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r, (x, it, rn)) for r, x, it, rn in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the serial answer: every system solved on one process
    import types

    import torch
    from ginkgo_b200 import batch as B
    host = types.SimpleNamespace(device=torch.device("cpu"))
    A, systems = B.convection_diffusion_batch(host, 9, lo=4, hi=30, seed=3)
    b = np.random.default_rng(1).standard_normal(A.total_rows)
    exp = []
    for s, (rp, ci, v) in enumerate(systems):
        n = len(rp) - 1
        M = np.zeros((n, n))
        for r in range(n):
            M[r, ci[rp[r]:rp[r + 1]]] = v[rp[r]:rp[r + 1]]
        o = int(A.host_row_offsets[s])
        exp.append(np.linalg.solve(M, b[o:o + n]))
    exp = np.concatenate(exp)
    for r in range(world):
        x, it, rn = res[r]
        np.testing.assert_allclose(x, exp, rtol=1e-12, atol=1e-12)
        assert it == [len(rp) - 1 for rp, _, _ in systems]
        assert len(rn) == len(systems)
