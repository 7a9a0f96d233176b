"""Row-partitioned eigsh over gloo ranks on CPU.

Each rank holds a slab of rows of a sector operator; the slab action here is
the oracle's assembled rows (scipy) standing in for the GPU slab kernel, so
the partition, the all-gather layout, the all-reduced Gram-Schmidt and the
thick restart are what is under test. Two ranks must give the oracle's
eigenvalues within 1e-10 relative with every residual verified, agree with
the one-rank run, and a rank that fails mid-solve must end the other rank's
solve with an error rather than a hang.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from qmbed_b200.distributed import RowPartition, distributed_eigsh

SITES, UP, MOMENTUM, PARITY, DELTA = 16, 8, 0, 1, 0.8


def test_partition_covers_rows_in_gather_order():
    for dim, world in [(10, 3), (7, 7), (5, 8), (1000, 4), (13, 1)]:
        part = RowPartition(dim, world)
        ranges = [part.range(r) for r in range(world)]
        assert sum(rows for _, rows in ranges) == dim
        covered = np.concatenate([np.arange(r0, r0 + rows) for r0, rows in ranges])
        assert np.array_equal(covered, np.arange(dim))
        # slab r lands at r * block in the gathered buffer: its rows keep their index
        for r, (r0, rows) in enumerate(ranges):
            assert rows == 0 or r0 == r * part.block
    with pytest.raises(ValueError):
        RowPartition(0, 2)


def _problem():
    from oracle import oracle
    basis = oracle.Basis(SITES, up=UP, momentum=MOMENTUM, parity=PARITY)
    op = oracle.Operator.build(basis, oracle.heisenberg_terms(SITES, delta=DELTA))
    matrix = op.to_scipy().real.tocsr()
    start = oracle.deterministic_start(op.dim, 3).real
    return op, matrix, start


def _slab_apply(matrix, part, rank, fail_after=None):
    import torch
    row0, rows = part.range(rank)
    block = matrix[row0:row0 + rows]
    calls = [0]

    def apply(x_full, y_slab):
        calls[0] += 1
        if fail_after is not None and calls[0] > fail_after:
            raise RuntimeError("planted slab failure")
        x = x_full[: part.dim].numpy()
        y_slab.copy_(torch.from_numpy(block @ x))
    return apply


def _tiny():
    """A 4 x 4 symmetric matrix: with three ranks the last slab is empty."""
    import scipy.sparse as sp
    a = np.random.default_rng(5).normal(size=(4, 4))
    return sp.csr_matrix(a + a.T), np.ones(4)


def _solve(rank, world, fail_rank=None, case="sector"):
    if case == "tiny":
        matrix, start = _tiny()
        eigenpairs, krylov = 1, 3
    else:
        _, matrix, start = _problem()
        eigenpairs, krylov = 4, 24
    part = RowPartition(matrix.shape[0], world)
    row0, rows = part.range(rank)
    apply = _slab_apply(matrix, part, rank, fail_after=3 if rank == fail_rank else None)
    return distributed_eigsh(apply, part, eigenpairs, krylov_dimension=krylov, tolerance=1e-10,
                             start=start[row0:row0 + rows], restart_keep=0 if case == "tiny" else 8)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, fail_rank, queue, case="sector"):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    try:
        r = _solve(rank, world, fail_rank, case)
        queue.put((rank, "ok", r.eigenvalues.tolist(), r.residuals.tolist(), r.converged, r.applications))
    except Exception as exc:  # the planted failure, or the collective that ends because of it
        queue.put((rank, "error", f"{type(exc).__name__}: {exc}", None, None, None))
    finally:
        if fail_rank is None:
            dist.destroy_process_group()


def _run(world, fail_rank=None, case="sector"):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, fail_rank, queue, case)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(queue.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
            raise AssertionError("a rank did not exit")
    return out


def test_two_ranks_match_the_oracle_and_one_rank():
    op, _, _ = _problem()
    expected = op.eigsh(4, tolerance=1e-12, seed=1).eigenvalues
    single = _solve(0, 1)
    assert single.converged
    out = _run(2)
    assert [o[0] for o in out] == [0, 1]
    for rank, status, values, residuals, converged, applications in out:
        assert status == "ok" and converged
        values = np.array(values)
        assert np.max(np.abs(values - expected) / np.abs(expected)) <= 1e-10
        assert np.all(np.array(residuals) <= 1e-10 * np.maximum(np.abs(values), 1.0))
        assert np.max(np.abs(values - single.eigenvalues) / np.abs(expected)) <= 1e-12
        assert applications == out[0][5]  # every rank applies its slab the same number of times


def test_three_ranks_with_a_short_last_slab():
    """Three ranks on a dimension that does not divide by three: the last slab
    is shorter, and the gathered layout still puts every row in place."""
    op, _, _ = _problem()
    part = RowPartition(op.dim, 3)
    assert part.range(2)[1] < part.block
    expected = op.eigsh(4, tolerance=1e-12, seed=1).eigenvalues
    out = _run(3)
    for rank, status, values, residuals, converged, applications in out:
        assert status == "ok" and converged
        assert np.max(np.abs(np.array(values) - expected) / np.abs(expected)) <= 1e-10


def test_failed_rank_ends_the_other_ranks_solve():
    out = _run(2, fail_rank=1)
    assert out[1][1] == "error" and "planted slab failure" in out[1][2]
    assert out[0][1] == "error"  # the next collective fails instead of waiting forever


def test_rank_with_an_empty_slab():
    """Four rows over three ranks: blocks of two, so rank 2 owns no rows but
    still takes part in every gather and reduction."""
    part = RowPartition(4, 3)
    assert part.range(2) == (4, 0)
    matrix, _ = _tiny()
    expected = np.linalg.eigvalsh(matrix.toarray())[0]
    out = _run(3, case="tiny")
    for rank, status, values, residuals, converged, applications in out:
        assert status == "ok" and converged, (rank, status, values)
        assert abs(values[0] - expected) <= 1e-10 * max(abs(expected), 1.0)
        assert applications == out[0][5]


def test_partition_property():
    """For any dimension and rank count: slabs are disjoint, cover every row in
    order, and slab r starts at r * block in the gathered buffer."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=300, deadline=None)
    @given(st.integers(1, 10**9), st.integers(1, 4096))
    def check(dim, world):
        part = RowPartition(dim, world)
        assert (part.block - 1) * world < dim <= part.block * world  # block = ceil(dim / world)
        end = 0
        for r in range(world):
            r0, rows = part.range(r)
            assert rows >= 0 and r0 + rows <= dim
            if rows:
                assert r0 == end == r * part.block
                end = r0 + rows
        assert end == dim

    check()
