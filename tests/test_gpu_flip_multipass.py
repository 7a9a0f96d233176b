"""Multi-pass flip-chain action (TMA-staged boxes) against the one-pass kernel and the oracle.

Vectors beyond 256 MB take the multi-pass action by default; QMBED_FLIP_PASSES
forces either form, so small chains exercise both. The multi-pass action must
equal the oracle's assembled action (FP64 1e-13 relative) and the one-pass
kernel (FP32 / complex64 2e-6), in real and complex vectors, through the fused
Chebyshev step, and in the Chebyshev propagator itself (complex128 states
within 1e-12 of each other, complex64 within 1e-5).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _operator(sites, seed=1, periodic=False):
    from qmbed_b200 import engine
    fields = np.random.default_rng(seed).uniform(-2.0, 2.0, sites)
    terms = engine.tfim_terms(sites, j=1.0, g=0.9, fields=fields, periodic=periodic)
    op = engine.GpuOperator(engine.GpuBasis(sites, normalization="pauli"), terms, storage="matrix_free")
    return op, terms


def _apply(op, x, precision, cplx, passes, monkeypatch):
    import torch
    monkeypatch.setenv("QMBED_FLIP_PASSES", passes)
    y = torch.full_like(x, float("nan"))
    op.apply_device(x, y, precision=precision, complex_vectors=cplx)
    torch.cuda.synchronize()
    return y


# sites: 14 (one group pass of 2-3 bits), 17 (one of 5-6), 22 (two group passes for complex128)
@pytest.mark.parametrize("sites", [14, 17, 22])
@pytest.mark.parametrize("precision,cplx", [(64, True), (64, False), (32, True), (32, False)])
def test_multipass_equals_one_pass(sites, precision, cplx, monkeypatch):
    import torch
    op, _ = _operator(sites, seed=sites, periodic=sites % 2 == 1)
    n = op.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    x = torch.randn(2 * n if cplx else n, dtype=dtype, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(sites))
    one = _apply(op, x, precision, cplx, "single", monkeypatch)
    multi = _apply(op, x, precision, cplx, "multi", monkeypatch)
    tol = 1e-13 if precision == 64 else 2e-6
    err = float(torch.linalg.vector_norm((multi - one).double()))
    assert err <= tol * float(torch.linalg.vector_norm(one.double())), err


@pytest.mark.parametrize("sites", [14, 16])
def test_multipass_matches_oracle(oracle, sites, monkeypatch):
    import torch
    op, terms = _operator(sites, seed=3)
    o = oracle.Operator.build(oracle.Basis(sites, normalization="pauli"), terms, check_particles=False)
    rng = np.random.default_rng(sites)
    x = rng.normal(size=op.dim) + 1j * rng.normal(size=op.dim)
    xd = torch.tensor(np.stack([x.real, x.imag], -1).reshape(-1), dtype=torch.float64, device="cuda")
    y = _apply(op, xd, 64, True, "multi", monkeypatch).cpu().numpy().reshape(-1, 2) @ np.array([1, 1j])
    expected = o.apply(x)
    assert np.linalg.norm(y - expected) <= 1e-13 * np.linalg.norm(expected)


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-5)])
def test_chebyshev_propagation_multipass_equals_one_pass(precision, tol, monkeypatch):
    op, _ = _operator(18, seed=7)
    psi0 = np.zeros(op.dim, np.complex128)
    psi0[-1] = 1.0
    times = [0.5, 1.0]
    monkeypatch.setenv("QMBED_FLIP_PASSES", "single")
    one, _ = op.chebyshev_evolve(psi0, times, precision=precision)
    monkeypatch.setenv("QMBED_FLIP_PASSES", "multi")
    multi, info = op.chebyshev_evolve(psi0, times, precision=precision)
    assert info["applications"] > 0
    assert np.max(np.linalg.norm(multi - one, axis=1)) <= tol


def test_unaligned_vectors_take_the_one_pass_kernel(monkeypatch):
    """Views that do not start on a 32-byte boundary cannot be the source of
    TMA boxes; the action falls back to the one-pass kernel."""
    import torch
    op, _ = _operator(16, seed=2)
    n = op.dim
    storage = torch.randn(2 * n + 2, dtype=torch.float32, device="cuda",
                          generator=torch.Generator(device="cuda").manual_seed(9))
    x = storage[2:]  # one complex64 element (8 bytes) past the allocation
    assert x.data_ptr() % 32 != 0
    ref = _apply(op, x.clone(), 32, True, "single", monkeypatch)
    got = _apply(op, x, 32, True, "multi", monkeypatch)
    assert float(torch.linalg.vector_norm(got - ref)) <= 2e-6 * float(torch.linalg.vector_norm(ref))


def test_stage_wait_times_out_instead_of_hanging():
    """The passes' wait on a box copy is bounded: a barrier armed for bytes that
    never arrive gives up and reports it, and the context stays usable."""
    import ctypes
    from qmbed_b200._lib import check, lib
    status = ctypes.c_int(-1)
    check(lib().qmbed_gpu_flip_wait_selftest(0, ctypes.byref(status)))
    assert status.value == 1
    op, _ = _operator(12, seed=4)
    assert op.apply(np.ones(op.dim)).shape == (op.dim,)
