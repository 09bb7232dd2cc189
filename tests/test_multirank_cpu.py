"""Multi-rank host logic on CPU (gloo, world size 2): sharding covers every
row / mesh exactly once, and the reported time is the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import dolfin_b200 as d2
        from dolfin_b200 import shard
        mesh = d2.UnitCubeMesh(3, 3, 3)
        V = d2.FunctionSpace(mesh, "Lagrange", 2)
        plan = V.pattern().plan()
        cuts = shard.row_partition(plan["inc_ptr"], world)
        mine = np.arange(cuts[rank], cuts[rank + 1])
        got = [None] * world
        dist.all_gather_object(got, mine.tolist())
        t = shard.max_over_ranks(1.0 + rank)
        weights = [5, 3, 8, 1, 7, 2]
        assign = shard.lpt_assign(weights, world)
        q.put((rank, got, t, assign, V.dim()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_row_partition_and_max_reduction_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, t, assign, n in res:
        rows = sorted(sum(got, []))
        assert rows == list(range(n))          # every node row owned exactly once
        assert t == 2.0                        # max over ranks
        assert sorted(sum(assign, [])) == list(range(6))
    # both ranks computed the same partition (deterministic)
    assert res[0][1] == res[1][1] and res[0][3] == res[1][3]


def test_lpt_balance():
    from dolfin_b200.shard import lpt_assign
    rng = np.random.default_rng(0)
    w = rng.integers(1, 1000, size=512)
    parts = lpt_assign(w, 8)
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= w.max()


def _block_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import dolfin_b200 as d2
        from dolfin_b200 import shard
        mesh = d2.UnitCubeMesh(3, 3, 3)
        V = d2.VectorFunctionSpace(mesh, "Lagrange", 2)
        P = V.pattern()
        cuts = shard.row_partition(P.plan()["inc_ptr"], world)
        P.set_row_block(int(cuts[rank]), int(cuts[rank + 1]))
        nrows, nnz = P.row_block_info()
        rp, cols = P.row_block_csr_host()
        dofs = shard.row_block_dofs(V.dim() // 3, 3, int(cuts[rank]), int(cuts[rank + 1]))
        got = [None] * world
        dist.all_gather_object(got, (dofs.tolist(), rp.tolist(), cols.tolist(), nrows, nnz))
        P.set_row_range(0, V.dim() // 3)
        frp, fcols = P.csr_host()
        q.put((rank, got, frp.tolist(), fcols.tolist()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_row_blocks_partition_the_csr_two_ranks():
    """Each rank's row block (its own CSR rows, rowptr from 0, global
    columns) is exactly the whole pattern's rows of its dofs; together the
    blocks hold every row once."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_block_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rank, got, frp, fcols = res[0]
    frp, fcols = np.array(frp), np.array(fcols)
    all_dofs = []
    for dofs, rp, cols, nrows, nnz in got:
        rp, cols = np.array(rp), np.array(cols)
        assert len(dofs) == nrows and rp[-1] == nnz == len(cols) and rp[0] == 0
        for i, d in enumerate(dofs):
            assert np.array_equal(cols[rp[i]:rp[i + 1]], fcols[frp[d]:frp[d + 1]])
        all_dofs += dofs
    assert sorted(all_dofs) == list(range(len(frp) - 1))
