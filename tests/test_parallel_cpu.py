"""Sharding of independent solves over two gloo ranks on CPU.

Each rank solves its share of small sector eigenproblems with the CPU oracle
(standing in for the GPU solver), and every rank must end with all results,
identical to the serial run. A unit that raises on one rank must surface as an
error on both ranks after the same collective, without hanging.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp

from qmbed_b200.parallel import ShardError, lpt_partition, run_sharded


def test_lpt_partition_is_balanced_and_complete():
    weights = [400024, 400023, 400023, 200012, 100, 7, 7, 3]
    parts = lpt_partition(weights, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(weights)))
    loads = [sum(weights[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(weights)
    assert parts == lpt_partition(weights, 3)  # deterministic
    assert lpt_partition([], 2) == [[], []]


def _units():
    # (sites, momentum) sectors of the Heisenberg chain at half filling
    return [(10, k) for k in range(10)] + [(12, k) for k in (0, 3, 6)]


def _solve(unit):
    from oracle import oracle
    sites, k = unit
    if sites < 0:
        raise ValueError("planted failure")
    op = oracle.Operator.build(oracle.Basis(sites, up=sites // 2, momentum=k), oracle.heisenberg_terms(sites))
    return [float(v) for v in op.eigsh(2, tolerance=1e-10, seed=1).eigenvalues]


def _weights(units):
    from math import comb
    return [comb(max(s, 1), max(s, 1) // 2) / max(s, 1) for s, _ in units]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, phases, queue):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        for name, units in phases:  # every rank runs the same phases in the same order
            try:
                queue.put((name, rank, "ok", run_sharded(units, _weights(units), _solve)))
            except ShardError as exc:
                queue.put((name, rank, "error", str(exc)))
    finally:
        dist.destroy_process_group()


def _run(phases, world=2):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, phases, queue)) for r in range(world)]
    for p in procs:
        p.start()
    out = [queue.get(timeout=300) for _ in range(world * len(phases))]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


def test_two_ranks_match_serial_and_report_failures_everywhere():
    units = _units()
    serial = run_sharded(units, _weights(units), _solve)  # no process group: serial
    failing = units[:4] + [(-1, 0)]
    out = _run([("full", units), ("failing", failing)])
    full = [o for o in out if o[0] == "full"]
    assert [r for _, r, _, _ in full] == [0, 1]
    for _, _, status, results in full:
        assert status == "ok"
        assert results == serial
    bad = [o for o in out if o[0] == "failing"]
    assert len(bad) == 2
    assert all(status == "error" and "planted failure" in text for _, _, status, text in bad)
