"""The CPU oracle against the reference's known answers and independent checks.

The reference (Rust) cannot run here, so the oracle is pinned by the numbers
its own tests assert (tests/golden/reference_anchors.json) and by dense
numpy/scipy computations that share no code with it.
"""

import itertools

import numpy as np
import pytest


def test_dimer_anchor(oracle, anchors):
    a = anchors["dimer"]
    op = oracle.Operator.build(oracle.Basis(2), oracle.heisenberg_terms(2, periodic=False))
    assert op.nnz == a["nnz"]
    r = op.eigsh(a["eigenpairs"], tolerance=a["tolerance"], max_iterations=a["max_iterations"], seed=a["seed"])
    np.testing.assert_allclose(r.eigenvalues, a["eigenvalues"], atol=a["abs_tol"])
    assert np.all(r.residuals < a["residual_below"])


def test_l4_momentum_sectors(oracle, anchors):
    a = anchors["l4_momentum"]
    for k, dim in a["dims"].items():
        assert len(oracle.Basis(a["sites"], up=a["up"], momentum=int(k))) == dim
    b0 = oracle.Basis(a["sites"], up=a["up"], momentum=0)
    op = oracle.Operator.build(b0, oracle.heisenberg_terms(4))
    r = op.eigsh(1, tolerance=a["tolerance"], max_iterations=a["max_iterations"], seed=a["seed"])
    assert abs(r.eigenvalues[0] - a["ground_k0"]) < 1e-12
    op1 = oracle.Operator.build(oracle.Basis(4, up=2, momentum=1), oracle.heisenberg_terms(4))
    assert op1.dense()[0, 0] == pytest.approx(a["k1_diagonal"], abs=1e-12)


def test_l4_parity_sectors_and_incompatibility(oracle, anchors):
    a = anchors["l4_parity"]
    full = oracle.Operator.build(oracle.Basis(4, up=2), oracle.heisenberg_terms(4)).dense()
    spectrum = []
    for p, dim in a["dims"].items():
        b = oracle.Basis(4, up=2, parity=int(p))
        assert len(b) == dim
        spectrum += list(np.linalg.eigvalsh(oracle.Operator.build(b, oracle.heisenberg_terms(4)).dense()))
    np.testing.assert_allclose(sorted(spectrum), np.linalg.eigvalsh(full), atol=a["spectrum_abs_tol"])
    with pytest.raises(oracle.OracleError) as error:
        oracle.Basis(4, up=2, momentum=a["incompatible_momentum"], parity=1)
    assert error.value.code == 6 and "incompatible symmetry request" in str(error.value)


def test_l18_translation_sector(oracle, anchors):
    a = anchors["l18_k0"]
    b = oracle.Basis(a["sites"], up=a["up"], momentum=a["momentum"])
    assert len(b) == a["dimension"]
    op = oracle.Operator.build(b, oracle.heisenberg_terms(a["sites"]))
    assert op.nnz < a["nnz_below"]
    r = op.eigsh(a["eigenpairs"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"],
                 max_iterations=a["max_iterations"], seed=a["seed"])
    assert np.all(r.residuals < a["residual_below"])


def test_fixed_weight_and_colex_anchors(oracle, anchors):
    assert len(oracle.Basis(16, up=8)) == anchors["l16_fixed_weight"]["dimension"]
    a = anchors["built_in_anchor"]
    b = oracle.Basis(a["sites"], up=a["up"])
    states, _ = b.states()
    assert len(b) == a["dimension"] and a["state"] in states.tolist()
    c = anchors["colex_order"]
    b = oracle.Basis(c["sites"], up=c["up"])
    states, _ = b.states()
    assert int(states[c["index"]]) == 1 << c["state_bit"]


def _brute_sector(sites, up, momentum, parity):
    """Orbit minima and orbit sizes by direct enumeration (independent of the oracle)."""
    mask = (1 << sites) - 1

    def rot(s, k):
        return ((s << k) & mask) | (s >> (sites - k)) if k else s

    def refl(s):
        return int(format(s, f"0{sites}b")[::-1], 2)

    reps, sizes = [], []
    for s in range(1 << sites):
        if up is not None and bin(s).count("1") != up:
            continue
        coeff = {}
        shifts = range(sites) if momentum is not None else [0]
        for k in shifts:
            chi = np.exp(-2j * np.pi * (momentum or 0) * k / sites)
            t = rot(s, k)
            coeff[t] = coeff.get(t, 0) + chi
            if parity is not None:
                coeff[refl(t)] = coeff.get(refl(t), 0) + parity * chi
        orbit = set(coeff)
        if min(orbit) != s:
            continue
        live = [t for t, c in coeff.items() if abs(c) > 1e-12]
        if live:
            reps.append(s)
            sizes.append(len(live))
    return reps, sizes


@pytest.mark.parametrize("sites,up,momentum,parity", [
    (6, 3, 1, None), (6, 3, 0, 1), (6, 3, 3, -1), (8, 4, 0, -1), (8, 4, 4, 1), (8, 4, 2, None), (8, None, 0, 1),
    (9, 4, 3, None), (10, 5, 0, 1), (10, None, 5, -1), (7, 3, None, 1), (7, None, None, -1),
])
def test_sector_enumeration_matches_brute_force(oracle, sites, up, momentum, parity):
    reps, sizes = _brute_sector(sites, up, momentum, parity)
    states, orbit = oracle.Basis(sites, up=up, momentum=momentum, parity=parity).states()
    assert states.tolist() == reps
    assert orbit.tolist() == sizes


@pytest.mark.parametrize("sites", [8, 10])
def test_momentum_parity_sectors_reconstruct_full_spectrum(oracle, sites):
    """Every (k, p) sector spectrum together equals the unreduced spectrum (Heisenberg, Sz=0)."""
    up = sites // 2
    terms = oracle.heisenberg_terms(sites)
    full = np.linalg.eigvalsh(oracle.Operator.build(oracle.Basis(sites, up=up), terms).dense())
    pieces = []
    for k in range(sites):
        parities = [1, -1] if k in (0, sites // 2) else [None]
        if k not in (0, sites // 2):
            # k and L-k carry equal spectra; take both through the complex sector
            pass
        for p in parities:
            b = oracle.Basis(sites, up=up, momentum=k, parity=p)
            if len(b):
                h = oracle.Operator.build(b, terms).dense()
                assert np.allclose(h, h.conj().T, atol=1e-12)
                pieces += list(np.linalg.eigvalsh(h))
    np.testing.assert_allclose(np.sort(pieces), full, atol=1e-10)


def test_sector_matrix_equals_projected_full_matrix(oracle):
    """H_sector = P^dag H P with P built from the reference coefficient rule, for a complex k sector."""
    sites, up, k = 8, 4, 3
    terms = oracle.heisenberg_terms(sites, delta=0.7)
    full_basis = oracle.Basis(sites, up=up)
    full = oracle.Operator.build(full_basis, terms).dense()
    full_states, _ = full_basis.states()
    position = {int(s): i for i, s in enumerate(full_states)}
    sector = oracle.Basis(sites, up=up, momentum=k)
    reps, orbit = sector.states()
    P = np.zeros((len(full_states), len(reps)), np.complex128)
    for col, rep in enumerate(reps.tolist()):
        for s in full_states.tolist():
            image = sector.image(s)
            if image and image[0] == rep:
                P[position[s], col] = image[1] / np.sqrt(image[2])
    np.testing.assert_allclose(P.conj().T @ P, np.eye(len(reps)), atol=1e-12)
    np.testing.assert_allclose(oracle.Operator.build(sector, terms).dense(), P.conj().T @ full @ P, atol=1e-12)


def test_deterministic_start_is_the_reference_lcg(oracle):
    n, seed = 1000, 31
    state = seed | 1
    values = []
    for _ in range(n):
        state = (state * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        values.append((state >> 11) / float(1 << 53) - 0.5)
    values = np.array(values)
    np.testing.assert_allclose(oracle.deterministic_start(n, seed), values / np.linalg.norm(values), rtol=1e-15,
                               atol=1e-17)


def test_lanczos_diagonal_anchors(oracle, anchors):
    a = anchors["diagonal_lanczos"]
    op = oracle.Operator.diagonal(np.arange(a["size"], dtype=float))
    r = op.eigsh(a["eigenpairs"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"],
                 max_iterations=a["max_iterations"], seed=a["seed"])
    np.testing.assert_allclose(r.eigenvalues, a["eigenvalues"], atol=a["abs_tol"])
    assert r.iterations == a["iterations"]
    b = anchors["real_sparse_eigsh"]
    op = oracle.Operator.from_triplets(b["size"], [0, 1], [0, 1], [-2.0, -1.0])
    r = op.eigsh(b["eigenpairs"], krylov_dimension=b["krylov_dimension"], tolerance=b["tolerance"],
                 max_iterations=b["max_iterations"], seed=b["seed"])
    np.testing.assert_allclose(r.eigenvalues, b["eigenvalues"], atol=1e-12)
    assert r.reorthogonalization_passes >= r.iterations
    assert r.conditional_second_passes < r.iterations


def test_solver_failure_and_expansion_anchors(oracle, anchors):
    a = anchors["loose_ritz_pair"]
    op = oracle.Operator.diagonal(np.arange(a["size"]) * a["scale"] / (a["size"] - 1))
    with pytest.raises(oracle.OracleError) as error:
        op.eigsh(a["eigenpairs"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"],
                 max_iterations=a["max_iterations"], seed=a["seed"])
    assert error.value.code == 14
    b = anchors["expanding_window"]
    op = oracle.Operator.diagonal(np.arange(b["size"]) / (b["size"] - 1))
    r = op.eigsh(b["eigenpairs"], tolerance=b["tolerance"], seed=b["seed"])
    assert abs(r.eigenvalues[0] - b["eigenvalue"]) < b["abs_tol"]
    assert r.iterations > b["iterations_above"]
    c = anchors["workspace_reuse"]
    op = oracle.Operator.diagonal(np.arange(c["size"]) / (c["size"] - 1))
    first = op.eigsh(c["eigenpairs"], krylov_dimension=c["krylov_dimension"], tolerance=c["tolerance"],
                     seed=c["seed"], eigenvectors=True)
    assert first.iterations > c["first_iterations_above"]
    second = op.eigsh(c["eigenpairs"], krylov_dimension=c["krylov_dimension"], tolerance=c["tolerance"],
                      seed=c["seed"], initial=first.eigenvectors)
    assert second.iterations <= c["second_iterations_at_most"]
    np.testing.assert_allclose(first.eigenvalues, second.eigenvalues, atol=1e-14)


def test_expm_anchors(oracle, anchors):
    for key in ("expop_unitary", "expop_thermal"):
        a = anchors[key]
        op = oracle.Operator.diagonal(a["diagonal"])
        x = np.array([1, 1]) / np.sqrt(2)
        c = complex(*a["coefficient"])
        y = op.expm_apply(c, x, max_degree=a["max_degree"], tolerance=a["tolerance"], max_substeps=a["max_substeps"])
        np.testing.assert_allclose(y, x * np.exp(c * np.array(a["diagonal"])), atol=a["abs_tol"])
    a = anchors["expm_rotation"]
    g = np.array(a["generator"])
    rows, cols = np.nonzero(g)
    op = oracle.Operator.from_triplets(2, rows, cols, g[rows, cols])
    t = a["coefficient"][0]
    y0 = op.expm_apply(complex(*a["coefficient"]), [1, 0], max_degree=a["max_degree"], tolerance=a["tolerance"],
                       max_substeps=a["max_substeps"])
    np.testing.assert_allclose(y0, [np.cos(t), np.sin(t)], atol=a["abs_tol"])
    y1 = op.expm_apply(complex(*a["second_coefficient"]), [1, 0], max_degree=a["max_degree"],
                       tolerance=a["tolerance"], max_substeps=a["max_substeps"])
    np.testing.assert_allclose([y1[0].real, y1[1].imag], [np.cosh(0.5), -np.sinh(0.5)], atol=a["second_abs_tol"])
    n = anchors["nilpotent_taylor"]
    e = np.array(n["entries"])
    op = oracle.Operator.from_triplets(4, e[:, 0].astype(int), e[:, 1].astype(int), e[:, 2])
    c = complex(*n["coefficient"])
    _, scaling, _, _ = op.expm_plan(c, max_degree=n["max_degree"], max_substeps=n["max_substeps"])
    assert scaling > n["scaling_above"]
    x = np.array([complex(*v) for v in n["input"]])
    dense = np.zeros((4, 4))
    dense[e[:, 0].astype(int), e[:, 1].astype(int)] = e[:, 2]
    expected = x.copy()
    power = x.copy()
    factorial = 1.0
    for order in range(1, 4):
        power = dense @ power
        factorial *= order
        expected = expected + c ** order * power / factorial
    np.testing.assert_allclose(op.expm_apply(c, x, max_degree=n["max_degree"], max_substeps=n["max_substeps"]),
                               expected, atol=n["abs_tol"])


def test_taylor_plan_matches_scipy_expm_multiply(oracle):
    from scipy.sparse.linalg import expm_multiply
    b = oracle.Basis(10, up=5, momentum=0, parity=1)
    op = oracle.Operator.build(b, oracle.heisenberg_terms(10, delta=0.8))
    x = oracle.deterministic_start(len(b), 3).astype(np.complex128)
    for c in (-0.7j, -0.3 + 0j, -1.0 - 2.0j):
        np.testing.assert_allclose(op.expm_apply(c, x), expm_multiply(c * op.to_scipy(), x), atol=1e-12)


def test_hermitian_and_tridiagonal_eigensolvers_match_numpy(oracle):
    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 40):
        a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        a = a + a.conj().T
        w, v = oracle.hermitian_eigen(a)
        np.testing.assert_allclose(np.sort(w), np.linalg.eigvalsh(a), atol=1e-12 * max(1, np.abs(w).max()))
        np.testing.assert_allclose(a @ v, v * w, atol=1e-11 * max(1, np.abs(w).max()))
        d, e = rng.normal(size=n), rng.normal(size=max(n - 1, 0))
        w, z = oracle.tridiagonal_eigen(d, e)
        t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        np.testing.assert_allclose(np.sort(w), np.linalg.eigvalsh(t), atol=1e-12 * max(1, np.abs(w).max()))


def test_operator_checks(oracle):
    b = oracle.Basis(4, up=2)
    with pytest.raises(oracle.OracleError) as error:
        oracle.Operator.build(b, [("+-", [(1.0, (0, 1))])])
    assert error.value.code == 7
    with pytest.raises(oracle.OracleError) as error:
        oracle.Operator.build(b, [("x", [(1.0, (0,))])])
    assert error.value.code == 5
    op = oracle.Operator.build(b, [("+-", [(1.0, (0, 1))])], check_hermitian=False)
    assert op.nnz > 0


def test_all_formats_share_action(oracle):
    """Dense apply of the assembled operator equals the stored action (visible_contract.rs:1008-1038)."""
    op = oracle.Operator.build(oracle.Basis(2), oracle.heisenberg_terms(2, periodic=False))
    x = np.array([1 - 0.5j, -2 + 0.25j, 0.75 + 1j, 0.5 - 1.5j])
    np.testing.assert_allclose(op.apply(x), op.dense() @ x, atol=1e-12)


def _diagonal32():
    return np.array([-2.0 + 4.0 * i / 31.0 for i in range(32)])


def test_adaptive_evolution_anchor(oracle, anchors):
    a = anchors["adaptive_evolution"]
    values = _diagonal32()
    op = oracle.Operator.diagonal(values)
    initial = np.full(32, 1.0 / np.sqrt(32.0), complex)
    states, d = op.evolve(initial, a["times"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"])
    assert d["lanczos_projections"] > 1
    assert d["matrix_vector_products"] == a["krylov_dimension"] * d["lanczos_projections"]
    assert d["accepted_substeps"] == d["lanczos_projections"]
    assert d["rejected_trial_intervals"] > 0
    np.testing.assert_allclose(states[0], initial, atol=0)
    expected = initial * np.exp(-1j * a["times"][2] * values)
    assert np.max(np.abs(states[2] - expected)) < a["final_state_abs_tol"]


def test_evolve_and_expm_lanczos_match_dense_exponential(oracle):
    from scipy.linalg import expm
    for sites, momentum, parity in ((10, 0, 1), (9, 2, None)):
        basis = oracle.Basis(sites, up=sites // 2, momentum=momentum, parity=parity)
        op = oracle.Operator.build(basis, oracle.heisenberg_terms(sites, delta=0.8))
        n = op.dim
        dense = np.zeros((n, n), complex)
        for j in range(n):
            e = np.zeros(n, complex)
            e[j] = 1.0
            dense[:, j] = op.apply(e)
        rng = np.random.default_rng(sites)
        v = rng.standard_normal(n) + (0.0 if op.is_real else 1j * rng.standard_normal(n))
        v /= np.linalg.norm(v)
        times = [0.0, 0.3, 0.3, 1.7, 4.0]
        states, d = op.evolve(v, times, krylov_dimension=16, tolerance=1e-10)
        for t, s in zip(times, states):
            assert np.linalg.norm(s - expm(-1j * t * dense) @ v) <= 1e-9
        assert d["accepted_substeps"] >= 1
        w = op.expm_lanczos(v, 0.4, krylov_dimension=min(n, 40))
        assert np.linalg.norm(w - expm(-0.4j * dense) @ v) <= 1e-10


def test_evolution_option_errors(oracle):
    from oracle.oracle import OracleError
    op = oracle.Operator.diagonal(_diagonal32())
    v = np.ones(32, complex)
    for times, krylov, tol in (([], 8, 1e-10), ([1.0, 0.5], 8, 1e-10), ([np.inf], 8, 1e-10), ([1.0], 0, 1e-10),
                               ([1.0], 8, 0.0)):
        with pytest.raises(OracleError) as e:
            op.evolve(v, times, krylov_dimension=krylov, tolerance=tol)
        assert e.value.code == 8


def test_thermal_two_level_anchor(oracle, anchors):
    a = anchors["thermal_two_level"]
    op = oracle.Operator.diagonal(a["diagonal"])
    identity = oracle.Operator.diagonal([1.0, 1.0])
    initial = np.full(2, 1.0 / np.sqrt(2.0), complex)
    beta = a["inverse_temperatures"][1]
    lz, energy, m = op.thermal_iteration(initial, a["inverse_temperatures"], a["krylov_dimension"], a["tolerance"])
    partition = np.exp(beta) + np.exp(-2.0 * beta)
    expected = (-np.exp(beta) + 2.0 * np.exp(-2.0 * beta)) / partition
    assert m == 2
    assert abs(lz[0] - np.log(2.0)) <= a["abs_tol"]
    assert abs(lz[1] - np.log(partition)) <= a["abs_tol"]
    assert abs(energy[1] - expected) <= a["abs_tol"]
    for method in ("ftlm", "ltlm"):
        values, ident = op.thermal_observables(initial, [op, identity], [beta], a["krylov_dimension"],
                                               a["tolerance"], method)
        assert abs(values[1, 0].real - ident[0]) <= a["abs_tol"]
        assert abs(values[0, 0].real / ident[0] - expected) <= a["abs_tol"]


def test_lanczos_full_orthonormal_anchor(oracle, anchors):
    a = anchors["lanczos_full_orthonormal"]
    op = oracle.Operator.diagonal(a["diagonal"])
    r = op.lanczos_ritz(np.asarray(a["initial"], complex), a["krylov_dimension"], a["tolerance"])
    q = r["basis"]
    assert q.shape[0] == 3
    assert np.max(np.abs(q.conj() @ q.T - np.eye(3))) <= a["orthonormality_abs_tol"]
    np.testing.assert_allclose(r["values"], sorted(a["diagonal"]), atol=1e-12)


def _exact_thermal(dense, v, betas):
    """ln(D / |v|^2) + ln <v|e^{-beta H}|v> and <v|H e^{-beta H}|v> / <v|e^{-beta H}|v>."""
    w, u = np.linalg.eigh(dense)
    overlap = np.abs(u.conj().T @ v) ** 2
    lz, e = [], []
    for beta in betas:
        boltzmann = overlap * np.exp(-beta * (w - w.min()))
        lz.append(np.log(len(v) / np.vdot(v, v).real) - beta * w.min() + np.log(boltzmann.sum()))
        e.append((boltzmann * w).sum() / boltzmann.sum())
    return np.array(lz), np.array(e)


@pytest.mark.parametrize("sites,momentum,parity", [(10, 0, 1), (9, 2, None)])
def test_thermal_iteration_is_exact_on_an_exhausted_krylov_space(oracle, sites, momentum, parity):
    """With the Krylov space exhausted (beta <= tolerance ends the recurrence)
    the FTLM estimate of one vector equals <v|e^{-beta H}|v> exactly."""
    basis = oracle.Basis(sites, up=sites // 2, momentum=momentum, parity=parity)
    op = oracle.Operator.build(basis, oracle.heisenberg_terms(sites, delta=0.7))
    dense = op.dense()
    rng = np.random.default_rng(sites)
    v = rng.standard_normal(op.dim) + (0.0 if op.is_real else 1j * rng.standard_normal(op.dim))
    betas = [0.0, 0.3, 1.0, 4.0]
    lz, e, m = op.thermal_iteration(v, betas, op.dim + 5, 1e-10)
    assert m <= op.dim
    exact_lz, exact_e = _exact_thermal(dense, v.astype(complex), betas)
    np.testing.assert_allclose(lz, exact_lz, atol=1e-9)
    np.testing.assert_allclose(e, exact_e, atol=1e-9)
    assert abs(lz[0] - np.log(op.dim)) <= 1e-12


def test_thermal_errors(oracle):
    from oracle.oracle import OracleError
    op = oracle.Operator.diagonal([-1.0, 2.0])
    v = np.ones(2, complex)
    for betas, krylov, tol, code in (([], 2, 1e-12, 8), ([-1.0], 2, 1e-12, 8), ([np.nan], 2, 1e-12, 8),
                                     ([1.0], 0, 1e-12, 8), ([1.0], 2, 0.0, 8)):
        with pytest.raises(OracleError) as e:
            op.thermal_iteration(v, betas, krylov, tol)
        assert e.value.code == code
    with pytest.raises(OracleError) as e:
        op.thermal_iteration(np.zeros(2, complex), [1.0], 2, 1e-12)
    assert e.value.code == 14


def _projector(oracle, sector, full_basis):
    """Columns: the sector's basis vectors in the fixed-weight space (P[s, col] = phase / sqrt(R))."""
    full_states, _ = full_basis.states()
    position = {int(s): i for i, s in enumerate(full_states)}
    reps, _ = sector.states()
    P = np.zeros((len(full_states), len(reps)), np.complex128)
    for col, rep in enumerate(reps.tolist()):
        for s in full_states.tolist():
            image = sector.image(s)
            if image and image[0] == rep:
                P[position[s], col] = image[1] / np.sqrt(image[2])
    return P


def _shift_matrix(oracle, source, target, terms):
    n = len(source)
    return np.column_stack([oracle.sector_shift(source, target, terms, np.eye(n)[c]) for c in range(n)])


@pytest.mark.parametrize("sites,up_s,up_t,k_s,k_t,symbol,q", [
    (4, 0, 1, 0, 1, "+", 1),     # tests/general_tensor_wide_basis.rs:164-217
    (8, 4, 4, 1, 4, "z", 3),
    (10, 4, 5, 2, 5, "+", 3),
    (9, 4, 4, 0, 2, "z", 2),
])
def test_sector_shift_equals_projected_full_action(oracle, sites, up_s, up_t, k_s, k_t, symbol, q):
    """apply_sector_shift (src/operator/mod.rs:2305-2351) between momentum
    sectors equals P_t^dag O P_s with O acting on the fixed-weight spaces."""
    terms = [(symbol, [(np.exp(-2j * np.pi * q * j / sites), (j,)) for j in range(sites)])]
    source = oracle.Basis(sites, up=up_s, momentum=k_s)
    target = oracle.Basis(sites, up=up_t, momentum=k_t)
    full_s, full_t = oracle.Basis(sites, up=up_s), oracle.Basis(sites, up=up_t)
    reduced = _shift_matrix(oracle, source, target, terms)
    expected = _projector(oracle, target, full_t).conj().T @ _shift_matrix(oracle, full_s, full_t, terms) \
        @ _projector(oracle, source, full_s)
    np.testing.assert_allclose(reduced, expected, atol=1e-12)
    assert np.max(np.abs(reduced)) > 0.5
    if sites == 4:
        assert reduced.shape == (1, 1) and abs(reduced[0, 0]) > 1.0


def test_sector_shift_errors(oracle):
    from oracle.oracle import OracleError
    source, target = oracle.Basis(6, up=3), oracle.Basis(6, up=4)
    with pytest.raises(OracleError) as e:
        oracle.sector_shift(source, target, [("+", [(1.0, (0,))])], np.ones(3))
    assert e.value.code == 9


def test_spectrum_single_pole_anchor(oracle):
    """tests/visible_contract.rs:1128-1143: H = [1], probe = [1], omega = 1,
    broadening 0.5 gives 2/pi."""
    h = oracle.Operator.diagonal([1.0])
    out = h.spectral_function(np.ones(1, complex), [1.0], 0.0, 0.5, krylov_dimension=8, tolerance=1e-12)
    assert abs(out[0] - 2.0 / np.pi) <= 1e-12


@pytest.mark.parametrize("sites,k", [(10, 0), (14, 0)])
def test_spectral_function_matches_dense_lehmann_sum(oracle, sites, k):
    """S(q=pi, omega) of the ground state: the dense path (D <= 128) and the
    Lanczos measure (D > 128) against the Lehmann sum from numpy."""
    basis = oracle.Basis(sites, up=sites // 2, momentum=k)
    h = oracle.Operator.build(basis, oracle.heisenberg_terms(sites))
    target = oracle.Basis(sites, up=sites // 2, momentum=(k + sites // 2) % sites)
    ht = oracle.Operator.build(target, oracle.heisenberg_terms(sites))
    ground = h.eigsh(1, tolerance=1e-12, seed=1, eigenvectors=True)
    probe = [("z", [((-1.0) ** j, (j,)) for j in range(sites)])]
    created = oracle.sector_shift(basis, target, probe, ground.eigenvectors[0])
    freqs = np.linspace(0.0, 4.0, 41)
    e0, eta = ground.eigenvalues[0], 0.4
    out = ht.spectral_function(created, freqs, e0, eta, krylov_dimension=min(ht.dim, 200))
    w, u = np.linalg.eigh(ht.dense())
    weight = np.abs(u.conj().T @ created) ** 2
    exact = [(weight * eta / (np.pi * ((f + e0 - w) ** 2 + eta ** 2))).sum() for f in freqs]
    tol = 1e-10 if ht.dim <= 128 else 1e-6
    np.testing.assert_allclose(out, exact, atol=tol * max(exact))
    assert np.all(out >= -1e-12)
