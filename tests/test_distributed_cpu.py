"""Multi-process checks of the N > 1 path on the CPU (gloo, world size 2).

bench.py runs one rank per GPU; ranks solve independent workloads (weak scaling, no data-path
collective), meet at barriers around the timed region and reduce their timings with a MAX.
These tests run the same helpers on gloo ranks, and the reference arm under torchrun, where
only rank 0 works and prints."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        bench.barrier(ws)
        t = bench.max_over_ranks(1.5 + rank, ws)
        w = bench.make_workload("uniform_potential", seed_offset=rank)
        out.put((rank, t, float(w["xs"][0])))
        bench.barrier(ws)
    finally:
        dist.destroy_process_group()


def test_gloo_barrier_and_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    assert all(t == 2.5 for _, t, _ in res)          # the max over ranks, on every rank
    assert res[0][2] != res[1][2]                     # each rank solves its own inputs


class _OracleContext:
    """A stand-in with the library context's host entry points, computed by the CPU oracle."""

    def force_mrag_host(self, theta, xs, ys, vs, x0s, y0s, hs):
        import oracle as O
        return O.force_mrag(theta, xs, ys, vs, x0s, y0s, hs)

    def potential_host(self, theta, xs, ys, vs, xt, yt):
        import oracle as O
        return O.potential(theta, xs, ys, vs, xt, yt)


def _shard_rank_main(rank, ws, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path[:0] = [os.path.join(ROOT, "2d-treecodes_b200"), os.path.join(ROOT, "oracle")]
    import sharding
    import workloads as W
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        w = W.lamb_oseen_force(n=4000, blocks_per_side=3, h=1.0 / 96)
        part = sharding.solve_shard(_OracleContext(), w["theta"], w["xs"], w["ys"], w["vs"],
                                    w["x0s"], w["y0s"], w["hs"], rank, ws)
        parts = [None] * ws
        dist.all_gather_object(parts, part)
        if rank == 0:
            xo, yo = sharding.assemble(parts, len(w["x0s"]))
            rx, ry = _OracleContext().force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"],
                                                      w["x0s"], w["y0s"], w["hs"])
            out.put((np.array_equal(xo, rx) and np.array_equal(yo, ry), [len(p[0]) for p in parts]))
    finally:
        dist.destroy_process_group()


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_force_exact64.so")),
                    reason="oracle not built")
def test_sharded_force_solve_on_two_gloo_ranks():
    """One problem split by blocks over two ranks (tree replicated, no exchange while
    evaluating): the gathered shards equal the unsplit solve bit for bit."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    equal, sizes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert equal and sorted(sizes) == [4, 5]


def test_block_shards_partition_in_morton_order():
    sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))
    import sharding
    import workloads as W
    x0, y0, _ = W.mrag_grid(8, 1.0 / 256)
    order = sharding.block_order(x0, y0)
    # Morton order of an 8 x 8 grid: the first four blocks are the lower-left 2 x 2 square
    assert sorted(order[:4].tolist()) == [0, 1, 8, 9]
    for ws in (1, 2, 3, 7, 64, 65):
        shards = [sharding.block_shard(x0, y0, r, ws) for r in range(ws)]
        allidx = np.concatenate(shards)
        assert sorted(allidx.tolist()) == list(range(64))
        assert np.array_equal(allidx, order)             # contiguous runs of the order
        assert max(map(len, shards)) - min(map(len, shards)) <= 1
    with pytest.raises(ValueError):
        sharding.block_shard(x0, y0, 2, 2)


def test_reference_arm_under_torchrun():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_potential_big.so")):
        pytest.skip("the compiled reference (oracle/_ref) is not built")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", "bench.py", "--impl",
           "reference", "--gpus", "2", "--workload", "uniform_potential", "--steps", "1",
           "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"


def _potential_shard_rank_main(rank, ws, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path[:0] = [os.path.join(ROOT, "2d-treecodes_b200"), os.path.join(ROOT, "oracle")]
    import sharding
    import workloads as W
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        w = W.gaussian_mixture_potential(n=20000, seed=7)
        part = sharding.solve_potential_shard(_OracleContext(), w["theta"], w["xs"], w["ys"],
                                              w["vs"], w["xt"], w["yt"], rank, ws)
        parts = [None] * ws
        dist.all_gather_object(parts, part)
        if rank == 0:
            got = sharding.assemble_potential(parts, len(w["xt"]))
            ref = _OracleContext().potential_host(w["theta"], w["xs"], w["ys"], w["vs"],
                                                  w["xt"], w["yt"])
            out.put((np.array_equal(got, ref), [len(p[0]) for p in parts]))
    finally:
        dist.destroy_process_group()


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_potential_exact64.so")),
                    reason="oracle not built")
def test_sharded_potential_solve_on_two_gloo_ranks():
    """One potential problem split by targets over two ranks in Morton order (tree replicated,
    no exchange while evaluating): the gathered shards equal the unsplit solve bit for bit."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_potential_shard_rank_main, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    equal, sizes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert equal and sorted(sizes) == [10000, 10000]


def test_target_shards_partition_in_morton_order():
    sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))
    import sharding
    r = np.random.default_rng(3)
    xt, yt = r.random(1001), r.random(1001)
    order = sharding.morton_order(xt, yt)
    for ws in (1, 2, 5, 1001, 1002):
        shards = [sharding.target_shard(xt, yt, k, ws) for k in range(ws)]
        allidx = np.concatenate(shards)
        assert np.array_equal(allidx, order)
        assert max(map(len, shards)) - min(map(len, shards)) <= 1
    with pytest.raises(ValueError):
        sharding.target_shard(xt, yt, -1, 2)
    with pytest.raises(ValueError):
        sharding.assemble_potential([(np.array([0, 1]), np.zeros(2))], 3)
