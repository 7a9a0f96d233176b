"""Learned eigsh hint: a network trained on the batched scan's own outputs.

The chain-spectrum network is trained on the GPU (the library's MLP kernels)
on what the batched scan solver returns for every momentum sector and scan
point of J1-J2 / XXZ chains at 12-20 sites: the lowest eigenvalue, the
largest Ritz value and the gap. Its prediction for a held-out 28-site XXZ
sector becomes an eigsh hint. The filtered solver must accept the interval
after its short Lanczos check and spend fewer operator applications on
bounds than without the network; the plain thick restart takes the
predicted restart size and needs fewer operator applications. Eigenvalues must agree with the un-hinted solves within 1e-10
relative, every residual verified. A hint that contradicts the check is
rejected and the solver falls back to its own bounds.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SITES, DELTA = 28, 1.3518


@pytest.fixture(scope="module")
def trained():
    from qmbed_b200 import learned
    x, y, info = learned.scan_training_set(sizes=(12, 14, 16, 18, 20), points=16, seed=0)
    model = learned.ChainSpectrum()
    loss = model.fit(x, y, epochs=300, seed=1)
    return model, x, y, info, loss


@pytest.fixture(scope="module")
def xxz28():
    from qmbed_b200 import engine
    basis = engine.GpuBasis(SITES, up=SITES // 2, momentum=0, parity=1)
    return engine.GpuOperator(basis, engine.heisenberg_terms(SITES, delta=DELTA), storage="packed")


def test_training_set_comes_from_the_scan(trained):
    model, x, y, info, loss = trained
    assert info["solves"] == (12 + 14 + 16 + 18 + 20) * 16 == len(x)
    assert np.all(y[:, 1] > y[:, 0])  # E_max above E0
    assert np.all(y[:, 2] >= -1e-9)   # gaps are not negative
    assert loss < 1e-2


def test_prediction_brackets_the_spectrum_at_28_sites(trained, xxz28):
    from qmbed_b200 import learned
    model = trained[0]
    hint = model.hint(SITES, 0.0, DELTA, 0, eigenpairs=6)
    ext = learned.lanczos_extremes(xxz28, 300, seed=0)
    assert hint["lower"] <= ext[0] and ext[1] <= hint["upper"]
    # the interval is tight: within 10% of the spectral width of the true extremes
    width = ext[1] - ext[0]
    assert ext[0] - hint["lower"] <= 0.1 * width and hint["upper"] - ext[1] <= 0.1 * width


def test_learned_hint_cuts_bound_applications_with_identical_eigenvalues(trained, xxz28):
    model = trained[0]
    hint = model.hint(SITES, 0.0, DELTA, 0, eigenpairs=6)
    base = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="filtered")
    hinted = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="filtered", hint=hint)
    assert hinted.hint_used and not base.hint_used
    assert hinted.bound_applications < base.bound_applications
    assert np.max(np.abs(hinted.eigenvalues - base.eigenvalues) / np.abs(base.eigenvalues)) <= 1e-10
    assert np.all(hinted.residuals <= 1e-10 * np.maximum(np.abs(hinted.eigenvalues), 1.0))


def test_learned_restart_size_cuts_thick_restart_steps(trained, xxz28):
    """The plain FP64 thick restart (Krylov 40) with the predicted restart size
    against the reference's size: fewer operator applications, the same
    eigenvalues within 1e-10, every residual verified."""
    model = trained[0]
    hint = model.hint(SITES, 0.0, DELTA, 0, eigenpairs=6)
    assert hint["restart_keep"] == 8  # small relative gap: the wanted pairs and two more
    base = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="fp64")
    hinted = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="fp64", hint=hint)
    assert hinted.operator_applications < base.operator_applications
    assert np.max(np.abs(hinted.eigenvalues - base.eigenvalues) / np.abs(base.eigenvalues)) <= 1e-10
    assert np.all(hinted.residuals <= 1e-10 * np.maximum(np.abs(hinted.eigenvalues), 1.0))


def test_wrong_hint_is_rejected(xxz28):
    bad = {"lower": -1.0, "upper": 1.0, "gap": 0.1, "restart_keep": 0, "check_steps": 8}
    r = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="filtered", hint=bad)
    base = xxz28.eigsh(6, krylov_dimension=40, tolerance=1e-10, seed=0, mode="filtered")
    assert not r.hint_used
    assert np.max(np.abs(r.eigenvalues - base.eigenvalues) / np.abs(base.eigenvalues)) <= 1e-10
