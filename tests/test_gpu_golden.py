"""GPU results against the committed oracle fixtures (tests/golden/oracle_fixtures.npz).

Sector states and orbit sizes bit-exact; H.v within 1e-13 of the fixture's
norm (FP64); eigenvalues within 1e-10 relative; thermal Lanczos estimates
within 1e-10; the cross-sector shift within 1e-13 of the fixture's norm.
"""

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "oracle_fixtures.npz"


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _close(got, ref, tol):
    assert np.linalg.norm(np.asarray(got) - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.parametrize("storage", ["packed", "matrix_free"])
def test_real_sector(fx, engine, storage):
    basis = engine.GpuBasis(16, up=8, momentum=0, parity=1)
    lo, _, orbit = basis.states()
    np.testing.assert_array_equal(lo, fx["real_sector_states"])
    np.testing.assert_array_equal(orbit, fx["real_sector_orbits"])
    op = engine.GpuOperator(basis, engine.heisenberg_terms(16, delta=0.85), storage=storage)
    _close(op.apply(fx["real_sector_x"]), fx["real_sector_hx"], 1e-13)
    for mode in ("fp64", "mixed", "filtered"):
        r = op.eigsh(4, tolerance=1e-10, seed=3, mode=mode)
        np.testing.assert_allclose(r.eigenvalues, fx["real_sector_eigenvalues"], rtol=1e-10)


def test_complex_sector(fx, engine):
    basis = engine.GpuBasis(15, up=7, momentum=3)
    lo, _, orbit = basis.states()
    np.testing.assert_array_equal(lo, fx["complex_sector_states"])
    np.testing.assert_array_equal(orbit, fx["complex_sector_orbits"])
    op = engine.GpuOperator(basis, engine.heisenberg_terms(15, delta=1.1))
    _close(op.apply(fx["complex_sector_x"]), fx["complex_sector_hx"], 1e-13)
    r = op.eigsh(3, tolerance=1e-10, seed=5)
    np.testing.assert_allclose(r.eigenvalues, fx["complex_sector_eigenvalues"], rtol=1e-10)


def test_xxz_twenty_sites(fx, engine):
    op = engine.GpuOperator(engine.GpuBasis(20, up=10, momentum=0, parity=1),
                            engine.heisenberg_terms(20, delta=1.3518), storage="matrix_free")
    for mode in ("fp64", "filtered"):
        r = op.eigsh(6, tolerance=1e-10, seed=20, mode=mode)
        np.testing.assert_allclose(r.eigenvalues, fx["xxz20_eigenvalues"], rtol=1e-10)


def test_flip_chain(fx, engine):
    op = engine.GpuOperator(engine.GpuBasis(12, normalization="pauli"),
                            engine.tfim_terms(12, g=0.9, fields=fx["tfim12_fields"]), storage="matrix_free")
    _close(op.apply(fx["tfim12_x"]), fx["tfim12_hx"], 1e-13)


def test_thermal_lanczos(fx, engine):
    from qmbed_b200 import lanczos
    op = engine.GpuOperator(engine.GpuBasis(14, up=7, momentum=0, parity=1), engine.heisenberg_terms(14))
    v = engine.deterministic_start(op.dim, 7)
    lz, e, m = lanczos.thermal_iteration(op, v, fx["ftlm14_betas"], 40)
    assert m == int(fx["ftlm14_krylov"][0])
    np.testing.assert_allclose(lz, fx["ftlm14_log_partition"], atol=1e-10)
    np.testing.assert_allclose(e, fx["ftlm14_energy"], atol=1e-10)


def test_sector_shift(fx, engine):
    from qmbed_b200 import spectrum
    terms = [("-", [(np.exp(-2j * np.pi * 3 * j / 12), (j,)) for j in range(12)])]
    shift = spectrum.SectorShift(engine.GpuBasis(12, up=6, momentum=1), engine.GpuBasis(12, up=5, momentum=4), terms)
    _close(shift.apply(fx["shift12_x"]), fx["shift12_y"], 1e-13)
