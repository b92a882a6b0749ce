"""Row sharding (spgemm_b200.shard): partition balance, and the 2-rank gloo
path on CPU with the oracle standing in for the per-rank GPU product."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from spgemm_b200 import shard
from spgemm_b200 import workloads as W


def oracle_product(A, B):
    import oracle
    a = A.to_csc()
    r = oracle.spgemm(A.rows, B.cols, a.colptr, a.rowidx, a.val, B.rowptr, B.col, B.val,
                      mode=1, threads=1)
    return W.Csr(A.rows, B.cols, r["rowptr"].astype(np.int32), r["col"], r["val"].astype(np.float32))


def test_partition_balances_work():
    A = W.rmat(12, 16, 0)
    p = shard.row_products(A, A)
    for parts in (1, 2, 3, 8):
        ranges = shard.partition_rows(p, parts)
        assert ranges[0][0] == 0 and ranges[-1][1] == A.rows
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        loads = [p[r0:r1].sum() + (r1 - r0) for r0, r1 in ranges]
        assert max(loads) <= (p.sum() + A.rows) / parts + p.max() + 1


def test_row_slice_and_concat_roundtrip():
    A = W.er(500, 6.0, 2)
    parts = [shard.row_slice(A, a, b) for a, b in shard.partition_rows(np.ones(A.rows), 3)]
    back = shard.concat_rows(parts)
    assert np.array_equal(back.rowptr, A.rowptr) and np.array_equal(back.col, A.col)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = W.rmat(11, 12, 4, values="sym")
        C, (r0, r1) = shard.shard_multiply(A, A, rank, world, oracle_product)
        q.put((rank, r0, r1, C.rowptr, C.col, C.val))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shard_gather():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    A = W.rmat(11, 12, 4, values="sym")
    full = oracle_product(A, A)
    ranges = sorted((g[1], g[2]) for g in got)
    assert ranges[0][0] == 0 and ranges[-1][1] == A.rows and ranges[0][1] == ranges[1][0]
    for _, _, _, rp, col, val in got:  # every rank holds the whole gathered C
        assert np.array_equal(rp, full.rowptr) and np.array_equal(col, full.col)
        assert np.array_equal(val, full.val)
