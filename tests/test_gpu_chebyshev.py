"""Structured flip-chain action and the Chebyshev propagator against the oracle.

The flip-chain kernels serve full-space chains whose terms are z products or a
single x (transverse-field Ising chains with longitudinal fields). Their action
must equal the oracle's assembled action (FP64: 1e-13 relative) and the
generic on-the-fly expansion on sizes that exercise both tiled passes. The
Chebyshev states must match the FP64 oracle's exponential action within 1e-9
(complex128 working vectors) or 1e-5 (complex64).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _fields(sites, seed, width=2.0):
    return np.random.default_rng(seed).uniform(-width, width, sites)


def _tfim(engine, sites, g=1.0, seed=0, periodic=False):
    return engine.tfim_terms(sites, j=1.0, g=g, fields=_fields(sites, seed), periodic=periodic)


@pytest.mark.parametrize("sites,normalization,periodic", [
    (10, "pauli", False), (11, "pauli", True), (12, "angular_momentum", False),
    (16, "pauli", False),   # complex128 tiles of 12 bits: the top bits flip through global partner reads
    (18, "pauli", True),
    (20, "angular_momentum", True),  # 7-8 high bits through global partner reads
])
def test_flip_chain_action_matches_oracle(engine, oracle, sites, normalization, periodic):
    terms = _tfim(engine, sites, g=0.8, seed=sites, periodic=periodic)
    g = engine.GpuOperator(engine.GpuBasis(sites, normalization=normalization), terms, storage="matrix_free")
    o = oracle.Operator.build(oracle.Basis(sites, normalization=normalization), terms)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(g.dim)
    z = x + 1j * rng.standard_normal(g.dim)
    for v in (x, z):
        ref = o.apply(v)
        got = g.apply(v)
        assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)


@pytest.mark.parametrize("precision,complex_vectors", [(32, False), (64, True)])
def test_flip_chain_large_matches_generic_expansion(engine, precision, complex_vectors):
    import torch
    sites = 26  # 12 to 14 bits flip through global partner reads at this size
    g = engine.GpuOperator(engine.GpuBasis(sites, normalization="pauli"), _tfim(engine, sites, seed=5),
                           storage="matrix_free")
    n = g.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(2 * n if complex_vectors else n, dtype=dtype, device="cuda", generator=gen)
    fast, generic = torch.empty_like(x), torch.empty_like(x)
    g.apply_device(x, fast, precision=precision, complex_vectors=complex_vectors)
    g.apply_device(x, generic, precision=precision, complex_vectors=complex_vectors, force_matrix_free=True)
    torch.cuda.synchronize()
    tol = 1e-13 if precision == 64 else 2e-6
    assert float(torch.linalg.norm(fast - generic) / torch.linalg.norm(generic)) <= tol


@pytest.mark.parametrize("precision,tol", [(64, 1e-9), (32, 1e-5)])
def test_chebyshev_matches_oracle_evolution(engine, oracle, precision, tol):
    sites = 12
    terms = _tfim(engine, sites, seed=3)
    g = engine.GpuOperator(engine.GpuBasis(sites, normalization="pauli"), terms, storage="matrix_free")
    o = oracle.Operator.build(oracle.Basis(sites, normalization="pauli"), terms)
    psi0 = np.zeros(g.dim, complex)
    psi0[-1] = 1.0  # all spins up
    times = [0.0, 0.1, 0.35, 1.0, 2.5]
    states, info = g.chebyshev_evolve(psi0, times, precision=precision)
    ref, _ = o.evolve(psi0, times, krylov_dimension=40, tolerance=1e-12)
    errors = [float(np.linalg.norm(a - b)) for a, b in zip(states, ref)]
    assert max(errors) <= tol, errors
    assert info["intervals"] == 4 and info["applications"] > 0
    assert info["max_norm_drift"] <= (1e-9 if precision == 64 else 1e-5)
    # a tighter interval from the exact extremes gives the same states with fewer terms
    from qmbed_b200.learned import lanczos_extremes
    lo, hi, r_lo, r_hi = lanczos_extremes(g, 300)
    assert r_lo < 1e-6 and r_hi < 1e-6
    tight, tinfo = g.chebyshev_evolve(psi0, times, e_min=lo - 1e-3, e_max=hi + 1e-3, precision=precision)
    assert max(float(np.linalg.norm(a - b)) for a, b in zip(tight, ref)) <= tol
    assert tinfo["applications"] < info["applications"]


def test_chebyshev_time_reversal_at_twenty_sites(engine):
    sites = 20
    g = engine.GpuOperator(engine.GpuBasis(sites, normalization="pauli"), _tfim(engine, sites, seed=9),
                           storage="matrix_free")
    psi0 = np.zeros(g.dim, complex)
    psi0[-1] = 1.0
    forward, _ = g.chebyshev_evolve(psi0, [0.5, 1.0])
    back, _ = g.chebyshev_evolve(forward[-1], [-1.0])
    assert np.linalg.norm(back[0] - psi0) <= 1e-9
    assert abs(np.linalg.norm(forward[-1]) - 1.0) <= 1e-9
    # only the last state kept: the same state
    last, _ = g.chebyshev_evolve(psi0, [0.5, 1.0], final_only=True)
    assert last.shape == (1, g.dim) and np.array_equal(last[0], forward[-1])


def test_chebyshev_rejects_other_operators(engine, oracle):
    from qmbed_b200 import QmbedError
    g = engine.GpuOperator(engine.GpuBasis(10, up=5, momentum=0), oracle.heisenberg_terms(10))
    with pytest.raises(QmbedError) as e:
        g.chebyshev_evolve(np.ones(g.dim, complex), [1.0])
    assert e.value.code == 11
    t = engine.GpuOperator(engine.GpuBasis(8, normalization="pauli"), _tfim(engine, 8), storage="matrix_free")
    with pytest.raises(QmbedError) as e:
        t.chebyshev_evolve(np.ones(t.dim, complex), [1.0], e_min=1.0, e_max=-1.0)
    assert e.value.code == 8
