"""Cross-sector actions and spectral functions on the GPU against the oracle.

Reference behaviour: apply_sector_shift (src/operator/mod.rs:2305-2351) and
spectral_function (src/dynamics/mod.rs:964-1021) with the Lanczos spectral
measure (src/solve/mod.rs:2886-2907); anchors of
tests/general_tensor_wide_basis.rs:164-217 and tests/visible_contract.rs:
1128-1143. Shifted vectors agree with the oracle within 1e-13 (atomic
accumulation reorders sums), spectra within 1e-10 of their maximum on the
dense path and 1e-8 on the Lanczos path.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


@pytest.fixture(scope="module")
def sp():
    import qmbed_b200.spectrum as module
    return module


def _momentum_terms(symbol, sites, q):
    return [(symbol, [(np.exp(-2j * np.pi * q * j / sites), (j,)) for j in range(sites)])]


@pytest.mark.parametrize("sites,up_s,up_t,k_s,k_t,symbol,q", [
    (4, 0, 1, 0, 1, "+", 1),        # tests/general_tensor_wide_basis.rs:164-217
    (8, 4, 4, 1, 4, "z", 3),
    (10, 4, 5, 2, 5, "+", 3),
    (9, 4, 4, 0, 2, "z", 2),
    (20, 10, 11, 0, 3, "+", 3),
    (21, 10, 10, 4, 11, "z", 7),
])
def test_sector_shift_matches_oracle(engine, sp, oracle, sites, up_s, up_t, k_s, k_t, symbol, q):
    terms = _momentum_terms(symbol, sites, q)
    g = sp.SectorShift(engine.GpuBasis(sites, up=up_s, momentum=k_s), engine.GpuBasis(sites, up=up_t, momentum=k_t),
                       terms)
    ob_s = oracle.Basis(sites, up=up_s, momentum=k_s)
    ob_t = oracle.Basis(sites, up=up_t, momentum=k_t)
    rng = np.random.default_rng(sites)
    x = rng.standard_normal(len(ob_s)) + 1j * rng.standard_normal(len(ob_s))
    y = g.apply(x)
    ref = oracle.sector_shift(ob_s, ob_t, terms, x)
    assert np.max(np.abs(ref)) > 0.1
    np.testing.assert_allclose(y, ref, atol=1e-13 * max(1.0, np.max(np.abs(ref))))
    if sites == 4:
        assert y.shape == (1,) and abs(y[0] / x[0]) > 1.0


@pytest.mark.parametrize("case", ["full", "colex", "parity"])
def test_sector_shift_without_momentum(engine, sp, oracle, case):
    if case == "full":
        sites, src, tgt, terms = 10, {}, {}, [("x", [(0.3, (2,))]), ("zz", [(1.0, (0, 1))])]
    elif case == "colex":
        sites, src, tgt, terms = 12, {"up": 5}, {"up": 6}, [("+", [(1.0 + 0.5j, (j,)) for j in range(12)])]
    else:
        sites, src, tgt = 12, {"up": 6, "momentum": 0, "parity": 1}, {"up": 6, "momentum": 0, "parity": -1}
        terms = [("z", [((1.0 if j < sites // 2 else -1.0), (j,)) for j in range(sites)])]
    g = sp.SectorShift(engine.GpuBasis(sites, **src), engine.GpuBasis(sites, **tgt), terms)
    ob_s, ob_t = oracle.Basis(sites, **src), oracle.Basis(sites, **tgt)
    x = np.random.default_rng(3).standard_normal(len(ob_s)).astype(complex)
    ref = oracle.sector_shift(ob_s, ob_t, terms, x)
    assert np.max(np.abs(ref)) > 0.1
    np.testing.assert_allclose(g.apply(x), ref, atol=1e-13 * max(1.0, np.max(np.abs(ref))))


def test_spectrum_single_pole_anchor(engine, sp):
    """tests/visible_contract.rs:1128-1143: H = [1], probe = [1] gives 2/pi at omega = 1, eta = 0.5."""
    basis = engine.GpuBasis(1, up=1)
    h = engine.GpuOperator(basis, [("I", [(1.0, (0,))])])
    probe = sp.SectorShift(basis, basis, [("I", [(1.0, (0,))])])
    out = sp.spectral_function(h, probe, np.ones(1), [1.0], 0.0, 0.5, krylov_dimension=8, tolerance=1e-12)
    assert abs(out[0] - 2.0 / np.pi) <= 1e-12


@pytest.mark.parametrize("sites,storage", [(10, "packed"), (14, "packed"), (20, "matrix_free")])
def test_spectral_function_matches_oracle(engine, sp, oracle, sites, storage):
    """S(q = pi, omega) of the k = 0 ground state: dense path (D <= 128) at L=10,
    Lanczos measure at L=14 and L=20."""
    half = sites // 2
    ob, ot = oracle.Basis(sites, up=half, momentum=0), oracle.Basis(sites, up=half, momentum=half % sites)
    oh = oracle.Operator.build(ob, oracle.heisenberg_terms(sites))
    oht = oracle.Operator.build(ot, oracle.heisenberg_terms(sites))
    ground = oh.eigsh(1, tolerance=1e-12, seed=1, eigenvectors=True)
    probe_terms = [("z", [((-1.0) ** j, (j,)) for j in range(sites)])]
    gb, gt = engine.GpuBasis(sites, up=half, momentum=0), engine.GpuBasis(sites, up=half, momentum=half % sites)
    gh = engine.GpuOperator(gt, engine.heisenberg_terms(sites), storage=storage)
    probe = sp.SectorShift(gb, gt, probe_terms)
    freqs = np.linspace(0.0, 4.0, 41)
    e0, eta, krylov = ground.eigenvalues[0], 0.2, 120
    out = sp.spectral_function(gh, probe, ground.eigenvectors[0], freqs, e0, eta, krylov_dimension=krylov)
    created = oracle.sector_shift(ob, ot, probe_terms, ground.eigenvectors[0])
    ref = oht.spectral_function(created, freqs, e0, eta, krylov_dimension=krylov)
    tol = 1e-10 if len(ot) <= 128 else 1e-8
    np.testing.assert_allclose(out, ref, atol=tol * np.max(ref))
    assert np.max(ref) > 1e-3 and np.all(out >= -1e-12)


def test_spectrum_errors(engine, sp):
    from qmbed_b200 import QmbedError
    basis = engine.GpuBasis(8, up=4)
    other = engine.GpuBasis(8, up=5)
    h = engine.GpuOperator(basis, engine.heisenberg_terms(8))
    probe = sp.SectorShift(basis, basis, [("z", [(1.0, (0,))])])
    x = np.ones(len(basis))
    for freqs, eta, krylov in (([], 0.1, 8), ([1.0], 0.0, 8), ([np.nan], 0.1, 8), ([1.0], 0.1, 0)):
        with pytest.raises(QmbedError) as e:
            sp.spectral_function(h, probe, x, freqs, 0.0, eta, krylov_dimension=krylov)
        assert e.value.code == 8
    with pytest.raises(QmbedError) as e:
        sp.spectral_function(h, probe, np.ones(3), [1.0], 0.0, 0.1)
    assert e.value.code == 9
    wrong = sp.SectorShift(basis, other, [("+", [(1.0, (0,))])])
    with pytest.raises(QmbedError) as e:
        sp.spectral_function(h, wrong, x, [1.0], 0.0, 0.1)
    assert e.value.code == 9
    with pytest.raises(QmbedError) as e:
        wrong.apply(np.ones(3))
    assert e.value.code == 9
