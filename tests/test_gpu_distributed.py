"""Slab form of the matrix-free action and the row-partitioned eigsh on one GPU.

The rows of a slab must equal the same rows of the full action bit for bit
(the slab kernel runs the same per-row arithmetic), for the nearest-neighbour
hop kernel and the general tile kernel, in FP64 and FP32. The row-partitioned
thick-restart Lanczos driven by the GPU slab kernel must give the oracle's
eigenvalues within 1e-10 relative, with every residual verified in FP64.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model", ["heisenberg", "j1j2"])
@pytest.mark.parametrize("precision", [64, 32])
def test_row_slabs_equal_the_full_action(model, precision):
    import torch
    from qmbed_b200 import engine
    from qmbed_b200.distributed import RowPartition, gpu_slab
    sites = 20
    terms = engine.heisenberg_terms(sites, delta=0.9) if model == "heisenberg" else \
        engine.heisenberg_terms(sites, j2=0.3, delta=0.9)
    op = engine.GpuOperator(engine.GpuBasis(sites, up=10, momentum=0, parity=1), terms, storage="matrix_free")
    assert op.lookup_info()["lookup"] == ("table_hop" if model == "heisenberg" else "table")
    n = op.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    x = torch.randn(n, dtype=dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(4))
    full = torch.empty_like(x)
    op.apply_device(x, full, precision=precision)
    part = RowPartition(n, 3)
    xg = torch.zeros(part.world * part.block, dtype=dtype, device="cuda")
    xg[:n] = x
    for rank in range(3):
        row0, rows = part.range(rank)
        y = torch.full((rows,), float("nan"), dtype=dtype, device="cuda")
        gpu_slab(op, part, rank, precision=precision)(xg, y)
        torch.cuda.synchronize()
        assert torch.equal(y, full[row0:row0 + rows]), rank


def test_row_slab_rejects_stored_rows_and_bad_ranges():
    import ctypes
    import torch
    from qmbed_b200 import engine
    from qmbed_b200._lib import QmbedError, check, lib
    basis = engine.GpuBasis(14, up=7, momentum=0, parity=1)
    packed = engine.GpuOperator(basis, engine.heisenberg_terms(14), storage="packed")
    free = engine.GpuOperator(basis, engine.heisenberg_terms(14), storage="matrix_free")
    x = torch.zeros(packed.dim, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    with pytest.raises(QmbedError):
        check(lib().qmbed_gpu_operator_apply_rows_device(packed.handle, 64, 0, packed.dim, p(x), p(y), None))
    with pytest.raises(QmbedError):
        check(lib().qmbed_gpu_operator_apply_rows_device(free.handle, 64, 5, free.dim, p(x), p(y), None))


def test_row_partitioned_eigsh_matches_oracle():
    import torch
    from oracle import oracle
    from qmbed_b200 import engine
    from qmbed_b200.distributed import RowPartition, distributed_eigsh, gpu_slab
    sites, delta = 20, 1.2
    terms = engine.heisenberg_terms(sites, delta=delta)
    op = engine.GpuOperator(engine.GpuBasis(sites, up=10, momentum=0, parity=1), terms, storage="matrix_free")
    ref = oracle.Operator.build(oracle.Basis(sites, up=10, momentum=0, parity=1),
                                oracle.heisenberg_terms(sites, delta=delta))
    expected = ref.eigsh(4, tolerance=1e-12, seed=1).eigenvalues
    part = RowPartition(op.dim, 1)
    start = torch.as_tensor(engine.deterministic_start(op.dim, 0), device="cuda")
    r = distributed_eigsh(gpu_slab(op, part, 0), part, 4, krylov_dimension=40, tolerance=1e-10, start=start,
                          restart_keep=12, device="cuda")
    assert r.converged
    assert np.max(np.abs(r.eigenvalues - expected) / np.abs(expected)) <= 1e-10
    assert np.all(r.residuals <= 1e-10 * np.maximum(np.abs(r.eigenvalues), 1.0))
