"""GPU engine against the CPU oracle on the same seeded inputs.

Bit-exact: sector states, orbit sizes, indices. FP64 actions: relative 2-norm
error <= 1e-13. Eigenvalues: <= 1e-10 relative. Exponential actions:
<= 1e-9 in 2-norm (FP64 working vectors), <= 1e-5 (complex64 working vectors).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SECTORS = [
    (2, None, None, None), (4, 2, 0, None), (4, 2, 1, None), (4, 2, None, 1), (4, 2, None, -1),
    (6, 3, 1, None), (8, 4, 0, 1), (8, 4, 4, -1), (8, None, 0, 1), (9, 4, 3, None), (10, 5, 0, -1),
    (12, 6, 6, 1), (12, None, 2, None), (14, 7, 0, 1), (16, 8, 3, None), (18, 9, 0, None), (20, 10, 0, 1),
    (12, 6, None, None), (11, None, None, -1),
]


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _states_int(lo, hi):
    return [int(a) | (int(b) << 64) for a, b in zip(lo, hi)]


@pytest.mark.parametrize("sites,up,momentum,parity", SECTORS)
def test_basis_bit_exact(engine, oracle, sites, up, momentum, parity):
    g = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity)
    o = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    assert len(g) == len(o)
    lo, hi, orbit = g.states()
    ostates, oorbit = o.states()
    assert np.array_equal(lo, ostates.astype(np.uint64))
    assert np.array_equal(orbit.astype(np.uint64), oorbit)


def test_wide_state_bases(engine, oracle):
    for sites, up, momentum in ((70, 2, 3), (96, 1, None), (65, 2, 0), (100, 2, None)):
        g = engine.GpuBasis(sites, up=up, momentum=momentum)
        o = oracle.Basis(sites, up=up, momentum=momentum)
        lo, hi, orbit = g.states()
        ostates, oorbit = o.states()
        assert _states_int(lo, hi) == [int(s) for s in ostates]
        assert np.array_equal(orbit.astype(np.uint64), np.asarray(oorbit, np.uint64))
    g = engine.GpuBasis(96, up=1)
    lo, hi, _ = g.states(95, 1)
    assert (int(hi[0]) << 64 | int(lo[0])) == 1 << 95


@pytest.mark.parametrize("sites,up,momentum,parity", [(8, 4, 3, None), (10, 5, 0, 1), (12, 6, 6, -1),
                                                       (12, None, 4, None), (9, None, None, 1)])
def test_images_match_oracle(engine, oracle, sites, up, momentum, parity):
    g = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity)
    o = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    ostates, _ = o.states()
    position = {int(s): i for i, s in enumerate(ostates)}
    rng = np.random.default_rng(sites)
    physical = rng.integers(0, 1 << sites, size=400, dtype=np.uint64)
    index, phase, orbit = g.images(physical)
    for s, i, ph, r in zip(physical.tolist(), index, phase, orbit):
        image = o.image(int(s))
        if image is None:
            assert i == -1
            continue
        rep, ophase, osize = image
        assert i == position[rep] and r == osize
        assert abs(ph - ophase) < 1e-12


def _models(sites):
    rng = np.random.default_rng(7)
    j1j2 = __import__("qmbed_b200.engine", fromlist=["x"]).heisenberg_terms(sites, j2=0.37, delta=0.9)
    fields = rng.uniform(-2, 2, size=sites)
    return {
        "heisenberg": __import__("oracle.oracle", fromlist=["x"]).heisenberg_terms(sites),
        "xxz": __import__("oracle.oracle", fromlist=["x"]).heisenberg_terms(sites, delta=0.73),
        "j1j2": j1j2,
        "xy_y": [("xx", [(0.4, (i, (i + 1) % sites)) for i in range(sites)]),
                 ("yy", [(0.4, (i, (i + 1) % sites)) for i in range(sites)]),
                 ("zz", [(1.1, (i, (i + 1) % sites)) for i in range(sites)])],
        "tfim_fields": [("zz", [(-1.0, (i, i + 1)) for i in range(sites - 1)]),
                        ("x", [(-1.0, (i,)) for i in range(sites)]),
                        ("z", [(float(h), (i,)) for i, h in enumerate(fields)])],
    }


CASES = [
    ("heisenberg", 12, 6, 0, 1, "angular_momentum"), ("heisenberg", 12, 6, 3, None, "angular_momentum"),
    ("heisenberg", 14, 7, 7, -1, "angular_momentum"), ("xxz", 14, 7, 0, None, "angular_momentum"),
    ("j1j2", 12, 6, 5, None, "angular_momentum"), ("j1j2", 14, 7, 0, -1, "angular_momentum"),
    ("xy_y", 10, 5, 2, None, "angular_momentum"), ("xy_y", 10, 5, 0, 1, "pauli"),
    ("tfim_fields", 10, None, None, None, "pauli_cartesian"), ("heisenberg", 12, 6, None, None, "angular_momentum"),
    ("heisenberg", 10, None, 0, 1, "pauli"),
]


@pytest.mark.parametrize("model,sites,up,momentum,parity,norm", CASES)
@pytest.mark.parametrize("storage", ["packed", "matrix_free"])
def test_hv_matches_oracle(engine, oracle, model, sites, up, momentum, parity, norm, storage):
    terms = _models(sites)[model]
    checks = dict(check_particles=(model != "tfim_fields"))
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity, normalization=norm),
                              terms, **checks)
    gb = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity, normalization=norm)
    g = engine.GpuOperator(gb, terms, storage=storage, **checks)
    n = o.dim
    rng = np.random.default_rng(3)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    expected = o.apply(x)
    got = g.apply(x)
    assert np.linalg.norm(got - expected) <= 1e-13 * max(np.linalg.norm(expected), 1.0)
    if o.is_real:
        assert g.is_real
        xr = rng.normal(size=n)
        er = o.apply(xr).real
        gr = g.apply(xr)
        assert np.linalg.norm(gr - er) <= 1e-13 * max(np.linalg.norm(er), 1.0)


@pytest.mark.parametrize("model,sites,up,momentum,parity,norm", CASES[:6])
def test_assembled_rows_match_oracle(engine, oracle, model, sites, up, momentum, parity, norm):
    terms = _models(sites)[model]
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity, normalization=norm), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity, normalization=norm), terms)
    a = o.to_scipy().tocsr()
    b = g.to_scipy().tocsr()
    # values agree entry by entry; exact cancellations in the reference's
    # phase sums can leave ~1e-16 residues, so the pattern is compared above 1e-13
    assert abs(a - b).max() <= 1e-13
    for m in (a, b):
        m.data[np.abs(m.data) <= 1e-13] = 0
        m.eliminate_zeros()
        m.sort_indices()
    assert np.array_equal(a.indptr, b.indptr) and np.array_equal(a.indices, b.indices)


def test_fp32_action(engine, oracle):
    import torch
    sites = 16
    terms = oracle.heisenberg_terms(sites, delta=0.8)
    o = oracle.Operator.build(oracle.Basis(sites, up=8, momentum=0, parity=1), terms)
    for storage in ("packed", "matrix_free"):
        g = engine.GpuOperator(engine.GpuBasis(sites, up=8, momentum=0, parity=1), terms, storage=storage)
        x = np.random.default_rng(1).normal(size=o.dim)
        expected = o.apply(x).real
        xd = torch.tensor(x, dtype=torch.float32, device="cuda")
        yd = torch.empty_like(xd)
        g.apply_device(xd, yd, precision=32)
        torch.cuda.synchronize()
        got = yd.double().cpu().numpy()
        assert np.linalg.norm(got - expected) <= 2e-6 * np.linalg.norm(expected)


def test_operator_errors_match_reference_categories(engine):
    from qmbed_b200 import QmbedError
    b = engine.GpuBasis(4, up=2)
    with pytest.raises(QmbedError) as e:
        engine.GpuOperator(b, [("+-", [(1.0, (0, 1))])])
    assert e.value.code == 7 and "Hermitian" in str(e.value)
    with pytest.raises(QmbedError) as e:
        engine.GpuOperator(b, [("x", [(1.0, (0,))])])
    assert e.value.code == 5
    with pytest.raises(QmbedError) as e:
        engine.GpuOperator(b, [("zz", [(1.0, (0, 4))])])
    assert e.value.code == 3
    with pytest.raises(QmbedError) as e:
        engine.GpuOperator(b, [("zz", [(1.0, (0,))])])
    assert e.value.code == 2
    with pytest.raises(QmbedError) as e:
        engine.GpuBasis(4, up=2, momentum=1, parity=1)
    assert e.value.code == 6


def test_eigsh_rejects_null_outputs(engine):
    """Null eigenvalue/residual buffers are QMBED_STATUS_INVALID_OPTIONS, and the operator stays usable."""
    import ctypes
    from qmbed_b200._lib import EigshOptionsC, lib
    op = engine.GpuOperator(engine.GpuBasis(8, up=4), engine.heisenberg_terms(8))
    options = EigshOptionsC()
    values = np.zeros(2)
    assert lib().qmbed_gpu_eigsh_hinted(op.handle, ctypes.byref(options), None, None, 0, None, None, None, None) == 8
    assert lib().qmbed_gpu_eigsh(op.handle, ctypes.byref(options), None, 0,
                                 values.ctypes.data_as(ctypes.c_void_p), None, None, None) == 8
    assert b"null eigenvalue or residual buffer" in lib().qmbed_gpu_last_error()
    r = op.eigsh(2, tolerance=1e-12)
    dense = np.linalg.eigvalsh(op.to_scipy().toarray())[:2]
    assert r.converged and np.allclose(r.eigenvalues, dense, rtol=1e-10, atol=1e-10)


def test_deterministic_start_matches_oracle(engine, oracle):
    for n, seed in ((1000, 31), (123457, 0), (5, 2**63 + 11)):
        np.testing.assert_allclose(engine.deterministic_start(n, seed), oracle.deterministic_start(n, seed),
                                   rtol=1e-14, atol=1e-16)


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), 1.0))


def test_eigsh_dimer_and_small_sectors(engine, oracle, anchors):
    a = anchors["dimer"]
    g = engine.GpuOperator(engine.GpuBasis(2), oracle.heisenberg_terms(2, periodic=False))
    r = g.eigsh(2, tolerance=a["tolerance"], max_iterations=a["max_iterations"], seed=a["seed"])
    np.testing.assert_allclose(r.eigenvalues, a["eigenvalues"], atol=a["abs_tol"])
    assert np.all(r.residuals < a["residual_below"])
    g = engine.GpuOperator(engine.GpuBasis(4, up=2, momentum=0), oracle.heisenberg_terms(4))
    r = g.eigsh(1, tolerance=1e-12, max_iterations=100, seed=5)
    assert abs(r.eigenvalues[0] + 2.0) < 1e-12


def test_eigsh_l18_anchor(engine, oracle, anchors):
    a = anchors["l18_k0"]
    g = engine.GpuOperator(engine.GpuBasis(18, up=9, momentum=0), oracle.heisenberg_terms(18))
    o = oracle.Operator.build(oracle.Basis(18, up=9, momentum=0), oracle.heisenberg_terms(18))
    assert g.dim == a["dimension"]
    kw = dict(krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"], max_iterations=a["max_iterations"],
              seed=a["seed"])
    r = g.eigsh(a["eigenpairs"], **kw)
    assert np.all(r.residuals < a["residual_below"])
    ro = o.eigsh(a["eigenpairs"], **kw)
    assert _rel(r.eigenvalues, ro.eigenvalues) <= 1e-10
    assert r.iterations == ro.iterations


@pytest.mark.parametrize("sites,up,momentum,parity,krylov,k,mode", [
    (20, 10, 0, None, None, 4, "fp64"),     # expanding Lanczos window (config 1 sector)
    (16, 8, 0, 1, 40, 4, "fp64"),           # thick restart
    (16, 8, 3, None, 24, 3, "fp64"),        # complex sector, thick restart
    (14, 7, 1, None, None, 2, "fp64"),      # complex sector, expanding window
    (20, 10, 0, None, None, 4, "mixed"),
    (16, 8, 0, 1, 40, 4, "mixed"),
    (16, 8, 3, None, 24, 3, "mixed"),
    (20, 10, 0, None, None, 4, "filtered"),  # block Chebyshev filter
    (16, 8, 0, 1, 40, 4, "filtered"),        # below the block method's size: mixed Lanczos
    (16, 8, 3, None, 24, 3, "filtered"),     # complex sector: mixed Lanczos
])
def test_eigsh_matches_oracle(engine, oracle, sites, up, momentum, parity, krylov, k, mode):
    terms = oracle.heisenberg_terms(sites, delta=0.95)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms)
    tol = 1e-12 if krylov is None else 1e-10
    ro = o.eigsh(k, krylov_dimension=krylov, tolerance=tol, seed=11)
    r = g.eigsh(k, krylov_dimension=krylov, tolerance=tol, seed=11, mode=mode, eigenvectors=True)
    assert _rel(r.eigenvalues, ro.eigenvalues) <= 1e-10
    # every returned pair passes the reference acceptance test in FP64
    for value, vector, residual in zip(r.eigenvalues, r.eigenvectors, r.residuals):
        x = vector if not g.is_real else vector.real
        hv = g.apply(x)
        true_residual = np.linalg.norm(hv - value * x)
        assert true_residual <= tol * max(abs(value), 1.0) * 1.5
        assert abs(np.linalg.norm(x) - 1.0) < 1e-10
    if mode == "fp64" and krylov is None:
        assert r.iterations == ro.iterations
    if mode in ("mixed", "filtered"):
        assert r.fp32_iterations > 0


@pytest.mark.parametrize("sites,up,momentum,parity,k,delta,storage", [
    (20, 10, 0, 1, 4, 1.0, "packed"),        # symmetry sector: weighted block coordinates, 8-wide block
    (18, 9, None, None, 4, 0.8, "packed"),   # no symmetry: unit weights
    (20, 10, 0, None, 7, 0.7, "packed"),     # 16-wide block
    (22, 11, 11, -1, 2, 1.2, "packed"),      # k = pi sector
    (20, 10, 0, 1, 6, 1.3, "matrix_free"),   # block action expanded on the fly
    (18, 9, None, None, 4, 0.8, "matrix_free"),
])
def test_filtered_eigsh_matches_oracle(engine, oracle, sites, up, momentum, parity, k, delta, storage):
    terms = oracle.heisenberg_terms(sites, delta=delta)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms, storage=storage)
    ro = o.eigsh(k, tolerance=1e-12, seed=3)
    r = g.eigsh(k, tolerance=1e-10, seed=3, mode="filtered", eigenvectors=True)
    # the block method ran (it makes no Gram-Schmidt passes) in both precisions
    assert r.reorthogonalization_passes == 0
    assert r.fp32_iterations > 0 and r.fp64_iterations > 0
    assert _rel(r.eigenvalues, ro.eigenvalues) <= 1e-10
    for value, vector, residual in zip(r.eigenvalues, r.eigenvectors, r.residuals):
        x = vector.real
        assert np.max(np.abs(vector.imag)) == 0.0
        true_residual = np.linalg.norm(g.apply(x) - value * x)
        assert true_residual <= 1e-10 * max(abs(value), 1.0) * 1.5
        assert abs(true_residual - residual) <= 1e-12 * max(abs(value), 1.0)
        assert abs(np.linalg.norm(x) - 1.0) < 1e-10
    again = g.eigsh(k, tolerance=1e-10, seed=3, mode="filtered")
    assert np.array_equal(again.eigenvalues, r.eigenvalues)  # bitwise reproducible


def test_filtered_eigsh_warm_start(engine, oracle):
    terms = oracle.heisenberg_terms(20, delta=0.9)
    g = engine.GpuOperator(engine.GpuBasis(20, up=10, momentum=0, parity=1), terms)
    first = g.eigsh(3, tolerance=1e-10, seed=8, mode="filtered", eigenvectors=True)
    second = g.eigsh(3, tolerance=1e-10, seed=8, mode="filtered", initial=first.eigenvectors)
    assert 2 * second.operator_applications < first.operator_applications
    np.testing.assert_allclose(second.eigenvalues, first.eigenvalues, rtol=1e-12)


def test_filtered_eigsh_with_the_default_start_as_initial_vector(engine, oracle):
    """A caller's vector equal to the solver's own first start column (the
    deterministic start of the seed) must not be repeated in the start block:
    the solve costs what the solve without an initial vector costs."""
    terms = oracle.heisenberg_terms(20, delta=0.9)
    g = engine.GpuOperator(engine.GpuBasis(20, up=10, momentum=0, parity=1), terms)
    plain = g.eigsh(4, tolerance=1e-10, seed=0, mode="filtered")
    v0 = engine.deterministic_start(g.dim, 0)
    seeded = g.eigsh(4, tolerance=1e-10, seed=0, mode="filtered", initial=v0[None, :])
    np.testing.assert_allclose(seeded.eigenvalues, plain.eigenvalues, rtol=1e-12)
    assert seeded.operator_applications <= 1.25 * plain.operator_applications
    assert seeded.fp32_iterations > 0  # the random start is not taken for a converged subspace


@pytest.mark.parametrize("shape", ["0", "1", "2", "3", "matrix_free"])
@pytest.mark.parametrize("sites,up,momentum,parity,nb,precision", [
    (16, 8, 0, 1, 8, 64), (16, 8, 0, 1, 16, 64), (16, 8, 0, 1, 8, 32), (14, 7, None, None, 16, 32),
    (18, 9, 9, 1, 8, 64),
])
def test_block_action_matches_columnwise_apply(engine, oracle, monkeypatch, sites, up, momentum, parity, nb,
                                               precision, shape):
    import torch
    storage = "matrix_free" if shape == "matrix_free" else "packed"
    if storage == "packed":
        monkeypatch.setenv("QMBED_BLOCK_SHAPE", shape)  # every kernel shape the autotuner may pick
    terms = oracle.heisenberg_terms(sites, delta=0.85)
    ob = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    o = oracle.Operator.build(ob, terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms, storage=storage)
    n = g.dim
    _, orbits = ob.states()
    s = np.sqrt(np.asarray(orbits, np.float64)) if momentum is not None or parity is not None else np.ones(n)
    rng = np.random.default_rng(5)
    z, p = rng.standard_normal((n, nb)), rng.standard_normal((n, nb))
    alpha, beta, gamma = 0.7, -0.3, 0.45
    expected = np.empty((n, nb))
    for j in range(nb):
        hx = o.apply(s * z[:, j]).real
        expected[:, j] = alpha * hx / s + beta * z[:, j] + gamma * p[:, j]
    dtype = torch.float64 if precision == 64 else torch.float32
    zd = torch.tensor(z, dtype=dtype, device="cuda").contiguous()
    pd = torch.tensor(p, dtype=dtype, device="cuda").contiguous()
    g.apply_block_device(zd, pd, nb, precision=precision, alpha=alpha, beta=beta, gamma=gamma, p=pd)
    torch.cuda.synchronize()
    got = pd.double().cpu().numpy()
    err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
    assert err <= (1e-14 if precision == 64 else 1e-6)
    # without the third term
    out = torch.empty_like(zd)
    g.apply_block_device(zd, out, nb, precision=precision, alpha=1.0, beta=0.0)
    torch.cuda.synchronize()
    ref = np.stack([o.apply(s * z[:, j]).real / s for j in range(nb)], axis=1)
    err = np.linalg.norm(out.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= (1e-14 if precision == 64 else 1e-6)


def test_eigsh_initial_subspace_warm_start(engine, oracle):
    terms = oracle.heisenberg_terms(16, delta=1.1)
    g = engine.GpuOperator(engine.GpuBasis(16, up=8, momentum=0, parity=1), terms)
    first = g.eigsh(3, krylov_dimension=16, tolerance=1e-10, seed=19, eigenvectors=True)
    second = g.eigsh(3, krylov_dimension=16, tolerance=1e-10, seed=19, initial=first.eigenvectors)
    assert second.iterations <= 16 < first.iterations
    np.testing.assert_allclose(first.eigenvalues, second.eigenvalues, atol=1e-12)


def test_eigsh_failure_is_nonconvergence(engine, oracle):
    from qmbed_b200 import QmbedError
    g = engine.GpuOperator(engine.GpuBasis(16, up=8, momentum=0), oracle.heisenberg_terms(16))
    with pytest.raises(QmbedError) as e:
        g.eigsh(2, krylov_dimension=4, tolerance=1e-14, max_iterations=6, seed=1)
    assert e.value.code == 14
    with pytest.raises(QmbedError) as e:
        g.eigsh(0)
    assert e.value.code == 8


@pytest.mark.parametrize("coefficient", [-1.0j, -0.25 + 0j, -0.3 - 0.8j])
def test_expm_matches_oracle(engine, oracle, coefficient):
    sites = 12
    terms = oracle.heisenberg_terms(sites, delta=0.6)
    o = oracle.Operator.build(oracle.Basis(sites, up=6, momentum=2), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=6, momentum=2), terms)
    plan_o = o.expm_plan(coefficient)
    plan_g = g.expm_plan(coefficient)
    assert plan_o[:2] == plan_g[:2]
    assert abs(plan_o[2] - plan_g[2]) <= 1e-12 * max(1.0, abs(plan_o[2]))
    assert abs(plan_o[3] - plan_g[3]) <= 1e-12 * plan_o[3]
    x = np.random.default_rng(4).normal(size=o.dim) + 1j * np.random.default_rng(5).normal(size=o.dim)
    x /= np.linalg.norm(x)
    expected = o.expm_apply(coefficient, x)
    got = g.expm_apply(coefficient, x)
    assert np.linalg.norm(got - expected) <= 1e-9
    got32 = g.expm_apply(coefficient, x, precision=32)
    assert np.linalg.norm(got32 - expected) <= 1e-4 * max(1.0, np.linalg.norm(expected))


def test_tfim_quench_step_matches_oracle(engine, oracle):
    sites = 10
    rng = np.random.default_rng(2)
    terms = [("zz", [(-1.0, (i, i + 1)) for i in range(sites - 1)]), ("x", [(-1.0, (i,)) for i in range(sites)]),
             ("z", [(float(h), (i,)) for i, h in enumerate(rng.uniform(-2, 2, sites))])]
    o = oracle.Operator.build(oracle.Basis(sites, normalization="pauli_cartesian"), terms, check_particles=False)
    g = engine.GpuOperator(engine.GpuBasis(sites, normalization="pauli_cartesian"), terms, check_particles=False)
    x = np.zeros(o.dim, np.complex128)
    x[-1] = 1.0  # all up
    for _ in range(3):
        x_o = o.expm_apply(-0.1j, x)
        x_g = g.expm_apply(-0.1j, x)
        assert np.linalg.norm(x_g - x_o) <= 1e-12
        x = x_o


def test_block_action_autotuned_shape_agrees(engine, oracle, monkeypatch):
    import torch
    # above the autotuner's size threshold: the first call times every shape
    g = engine.GpuOperator(engine.GpuBasis(30, up=15, momentum=0, parity=1), oracle.heisenberg_terms(30))
    n, nb = g.dim, 8
    assert n >= 1 << 20
    gen = torch.Generator(device="cuda").manual_seed(3)
    z = torch.randn((n, nb), dtype=torch.float32, device="cuda", generator=gen)
    p = torch.randn((n, nb), dtype=torch.float32, device="cuda", generator=gen)
    tuned, pinned = torch.empty_like(z), torch.empty_like(z)
    g.apply_block_device(z, tuned, nb, precision=32, alpha=0.3, beta=0.1, gamma=-0.2, p=p)
    g.apply_block_device(z, tuned, nb, precision=32, alpha=0.3, beta=0.1, gamma=-0.2, p=p)  # cached shape
    monkeypatch.setenv("QMBED_BLOCK_SHAPE", "0")
    g.apply_block_device(z, pinned, nb, precision=32, alpha=0.3, beta=0.1, gamma=-0.2, p=p)
    torch.cuda.synchronize()
    assert torch.linalg.norm(tuned - pinned) <= 1e-6 * torch.linalg.norm(pinned)
