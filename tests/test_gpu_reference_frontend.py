"""The reference's own Python frontend driving libqmbed_b200.so on the GPU.

The reference's pure-Python packages (``qmbed`` and its QuSpin-compatible
``quspin``, bindings/python/src) are installed offline into ``baseline/_ref``
(``pip install --no-index --no-build-isolation --no-deps --target
baseline/_ref`` of a copy of bindings/python; the Rust extension is not
built). They load a native library named by ``QMBED_LIBRARY_PATH``
(bindings/python/src/qmbed/_ffi.py:128-186); pointing it at this library runs
the unmodified frontend on the GPU. The flows and tolerances follow the
reference's QuSpin compatibility tests ``test_Lanczos.py`` (Lanczos
exponential and ground state, 1e-10) and ``test_expm_multiply_parallel.py``
(imaginary-time projection and random sparse matrices against SciPy's
``expm_multiply``) on the 20-site ``m=0, kblock=0, pblock=1, zblock=1``
Heisenberg sector. The tests skip when ``baseline/_ref`` is absent.
"""

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
FRONTEND = ROOT / "baseline" / "_ref"
LIBRARY = ROOT / "qmbed_b200" / "libqmbed_b200.so"

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not (FRONTEND / "quspin").is_dir(), reason="reference frontend not installed in baseline/_ref"),
]


@pytest.fixture(scope="module")
def quspin():
    os.environ["QMBED_LIBRARY_PATH"] = str(LIBRARY)
    if str(FRONTEND) not in sys.path:
        sys.path.insert(0, str(FRONTEND))
    import quspin.basis
    import quspin.operators
    import quspin.tools.evolution
    import quspin.tools.lanczos
    return quspin


def _heisenberg(quspin, sites, sign=1.0):
    basis = quspin.basis.spin_basis_1d(sites, m=0, kblock=0, pblock=1, zblock=1)
    bonds = [[1.0, i, (i + 1) % sites] for i in range(sites)]
    h = quspin.operators.hamiltonian([[op, bonds] for op in ("xx", "yy", "zz")], [], basis=basis,
                                     dtype=np.float64)
    return basis, (-h if sign < 0 else h)


def test_lanczos_exponential_and_ground_state(quspin):
    from scipy.sparse.linalg import expm_multiply
    lz = quspin.tools.lanczos
    basis, H = _heisenberg(quspin, 20, sign=-1.0)
    rng = np.random.default_rng(0)
    v0 = rng.normal(0, 1, size=basis.Ns)
    v0 /= np.linalg.norm(v0)
    v1, v2 = v0.copy(), v0.copy()
    static = H.static
    for _ in range(10):
        E1, V1, q1 = lz.lanczos_full(H, v1, 20)
        E2, V2, q2 = lz.lanczos_iter(H, v2, 20)
        v0 = expm_multiply(-0.1j * static, v0)
        v1 = lz.expm_lanczos(E1, V1, q1, a=-0.1j)
        v2 = lz.expm_lanczos(E2, V2, q2, a=-0.1j)
        np.testing.assert_allclose(v1, v0, atol=1e-10, rtol=0)
        np.testing.assert_allclose(v2, v0, atol=1e-10, rtol=0)

    E_gs, psi_gs = H.eigsh(k=1, which="LA")
    psi_gs = psi_gs.ravel()
    v0 = rng.normal(0, 1, size=basis.Ns)
    v0 /= np.linalg.norm(v0)
    E, V, Q = lz.lanczos_full(H, v0, 50, full_ortho=False)
    v1 = lz.lin_comb_Q_T(V[:, -1], Q)
    assert abs(E[-1] - E_gs[-1]) < 1e-10
    assert abs(np.log(abs(np.vdot(v1, psi_gs)))) < 1e-10
    E, V, Q_iter = lz.lanczos_iter(H, v0, 50, return_vec_iter=True)
    np.testing.assert_allclose(lz.lin_comb_Q_T(V[:, -1], Q_iter), v1, atol=1e-10, rtol=0)


def test_imaginary_time_projection(quspin):
    import scipy.sparse as sp
    from scipy.sparse.linalg import expm_multiply
    basis, H = _heisenberg(quspin, 20)
    (E,), _ = H.eigsh(k=1, which="SA")
    A = -(H.tocsr() - E * sp.eye(H.Ns, format="csr", dtype=np.float64))
    U = quspin.tools.evolution.expm_multiply_parallel(A)
    rng = np.random.default_rng(0)
    v1 = rng.uniform(-1, 1, size=H.Ns)
    v1 /= np.linalg.norm(v1)
    v2 = v1.copy()
    for _ in range(100):
        v2 = U.dot(v2)
        v2 /= np.linalg.norm(v2)
        v1 = expm_multiply(A, v1)
        v1 /= np.linalg.norm(v1)
        if abs(H.expt_value(v2) - E) < 1e-15:
            break
    np.testing.assert_allclose(v1, v2, rtol=0, atol=1e-15)


@pytest.mark.parametrize("seed", [0, 1])
def test_random_sparse_matrices(quspin, seed):
    import scipy.sparse as sp
    from scipy.sparse.linalg import expm_multiply
    rng = np.random.default_rng(seed)
    n = 3500
    density = np.log(n) / n
    A = (sp.random(n, n, density=density, random_state=seed)
         + 1j * sp.random(n, n, density=density, random_state=seed + 100)).tocsr()
    v = rng.normal(0, 1, size=n) + 1j * rng.normal(0, 1, size=n)
    v /= np.linalg.norm(v)
    got = quspin.tools.evolution.expm_multiply_parallel(A).dot(v)
    np.testing.assert_allclose(got, expm_multiply(A, v), rtol=0, atol=1e-15)
    got = quspin.tools.evolution.expm_multiply_parallel(A, a=-0.01j, dtype=np.complex128).dot(v)
    np.testing.assert_allclose(got, expm_multiply(-0.01j * A, v), rtol=0, atol=1e-15)


def test_driven_evolution_through_the_drive_callback(quspin):
    """hamiltonian.evolve(solver_name="qmbed") with a dynamic term calls qmbed_evolve_model_with_drive_json with
    the frontend's own coefficient callback; it must agree with the frontend's SciPy integration, which
    applies the same model through apply_model at every right-hand-side evaluation."""
    L = 10
    basis = quspin.basis.spin_basis_1d(L, Nup=L // 2, kblock=0, pblock=1, pauli=False)
    bonds = [[1.0, i, (i + 1) % L] for i in range(L)]

    def drive(t, omega):
        return np.cos(omega * t)

    dynamic = [["zz", [[0.4, i, (i + 2) % L] for i in range(L)], drive, [2.0]]]
    H = quspin.operators.hamiltonian([[op, bonds] for op in ("xx", "yy", "zz")], dynamic, basis=basis,
                                     dtype=np.float64)
    rng = np.random.default_rng(2)
    psi = rng.standard_normal(H.Ns) + 1j * rng.standard_normal(H.Ns)
    psi /= np.linalg.norm(psi)
    times = np.array([0.5, 1.0, 1.5])
    ours = H.evolve(psi, 0.0, times, solver_name="qmbed")
    scipy_path = H.evolve(psi, 0.0, times, atol=1e-12, rtol=1e-12)
    assert ours.shape == scipy_path.shape
    assert np.abs(ours - scipy_path).max() <= 1e-8
