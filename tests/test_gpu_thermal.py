"""Full Lanczos decompositions and thermal Lanczos (FTLM / LTLM) on the GPU.

Reference behaviour: src/solve/mod.rs:2694-2857 (lanczos_full with DGKS
reorthogonalisation, lanczos_ritz), 3457-3940 (thermal static iteration,
projected observables, FTLM/LTLM contractions); anchors of
tests/solver_extensions.rs:157-181 and 296-361 and of the JSON Lanczos
resource test (bindings/capi/src/lib.rs:7483-7578). Tridiagonals, Ritz
values and thermal estimates agree with the FP64 oracle within 1e-10
(absolute, on O(1)..O(10) quantities); the basis is orthonormal within 1e-12.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


@pytest.fixture(scope="module")
def lz():
    import qmbed_b200.lanczos as module
    return module


def _two_level(engine, values):
    """One Pauli site with diagonal `values` in basis order: a I + b z."""
    basis = engine.GpuBasis(1, normalization="pauli")
    probe = engine.GpuOperator(basis, [("z", [(1.0, (0,))])])
    z = np.array([probe.apply(np.eye(2)[i])[i].real for i in range(2)])
    b = (values[1] - values[0]) / (z[1] - z[0])
    a = values[0] - b * z[0]
    return engine.GpuOperator(basis, [("I", [(a, (0,))]), ("z", [(b, (0,))])])


def test_thermal_two_level_anchor_on_gpu(engine, lz, anchors):
    a = anchors["thermal_two_level"]
    op = _two_level(engine, a["diagonal"])
    identity = _two_level(engine, [1.0, 1.0])
    initial = np.full(2, 1.0 / np.sqrt(2.0), complex)
    beta = a["inverse_temperatures"][1]
    partition = np.exp(beta) + np.exp(-2.0 * beta)
    expected = (-np.exp(beta) + 2.0 * np.exp(-2.0 * beta)) / partition
    logz, energy, m = lz.thermal_iteration(op, initial, a["inverse_temperatures"], a["krylov_dimension"],
                                           a["tolerance"])
    assert m == 2
    assert abs(logz[0] - np.log(2.0)) <= a["abs_tol"]
    assert abs(logz[1] - np.log(partition)) <= a["abs_tol"]
    assert abs(energy[1] - expected) <= a["abs_tol"]
    e, v, q = lz.lanczos_full(op, initial, a["krylov_dimension"], eps=a["tolerance"])
    for method in ("ftlm", "ltlm"):
        values, ident = q.thermal({"H": op, "I": identity}, [beta], method)
        assert abs(values["I"][0].real - ident[0]) <= a["abs_tol"]
        assert abs(values["H"][0].real / ident[0] - expected) <= a["abs_tol"]
        # QuSpin-compatible form: host contraction of GPU projections
        out, ident2 = (lz.FTLM_static_iteration if method == "ftlm" else lz.LTLM_static_iteration)(
            {"H": op, "I": identity}, e, v, q, beta)
        assert abs(float(out["H"]) / float(ident2) - expected) <= a["abs_tol"]


def _diagonal_operator(engine, values):
    """Two Pauli sites with diagonal `values` (4 entries) in basis order:
    a I + b z0 + c z1 + d z0 z1."""
    basis = engine.GpuBasis(2, normalization="pauli")
    parts = [[("I", [(1.0, (0,))])], [("z", [(1.0, (0,))])], [("z", [(1.0, (1,))])], [("zz", [(1.0, (0, 1))])]]
    cols = [[engine.GpuOperator(basis, t).apply(np.eye(4)[i])[i].real for i in range(4)] for t in parts]
    a, b, c, d = np.linalg.solve(np.array(cols).T, np.asarray(values, float))
    return engine.GpuOperator(basis, [("I", [(a, (0,))]), ("z", [(b, (0,)), (c, (1,))]), ("zz", [(d, (0, 1))])])


def test_lanczos_full_orthonormal_anchor_on_gpu(engine, lz, anchors):
    a = anchors["lanczos_full_orthonormal"]
    op = _diagonal_operator(engine, list(a["diagonal"]) + [7.0])
    diag = np.array([op.apply(np.eye(4)[i])[i].real for i in range(4)])
    np.testing.assert_allclose(diag, list(a["diagonal"]) + [7.0], atol=1e-14)
    v = np.zeros(4, complex)
    v[:3] = a["initial"]
    q = lz.LanczosBasis(op, v, a["krylov_dimension"], a["tolerance"])
    basis_rows = q.to_numpy()
    assert basis_rows.shape == (3, 4)
    assert np.max(np.abs(basis_rows.conj() @ basis_rows.T - np.eye(3))) <= a["orthonormality_abs_tol"]
    np.testing.assert_allclose(q.eigenvalues, np.sort(a["diagonal"]), atol=1e-12)


CASES = [
    (16, 8, 0, 1, "packed"),        # real sector (dim 440)
    (15, 7, 3, None, "packed"),     # complex sector (dim 429)
    (14, 7, None, None, "matrix_free"),
]


def _sector(engine, oracle, sites, up, momentum, parity, storage, delta=0.7):
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity),
                           engine.heisenberg_terms(sites, delta=delta), storage=storage)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity),
                              oracle.heisenberg_terms(sites, delta=delta))
    return g, o


@pytest.mark.parametrize("sites,up,momentum,parity,storage", CASES)
def test_lanczos_ritz_matches_oracle(engine, lz, oracle, sites, up, momentum, parity, storage):
    g, o = _sector(engine, oracle, sites, up, momentum, parity, storage)
    rng = np.random.default_rng(sites)
    v = rng.standard_normal(g.dim) + (0.0 if o.is_real else 1j * rng.standard_normal(g.dim))
    q = lz.LanczosBasis(g, v, 40, 1e-12)
    r = o.lanczos_ritz(v, 40, 1e-12)
    assert q.krylov_dimension == len(r["values"]) == 40
    assert q.is_real == o.is_real
    np.testing.assert_allclose(q.diagonal, r["diagonal"], atol=1e-10)
    np.testing.assert_allclose(q.off_diagonal, r["off_diagonal"], atol=1e-10)
    np.testing.assert_allclose(q.eigenvalues, r["values"], atol=1e-10)
    assert abs(q.initial_norm - r["initial_norm"]) <= 1e-12 * r["initial_norm"]
    rows = q.to_numpy()
    assert np.max(np.abs(rows.conj() @ rows.T - np.eye(40))) <= 1e-12
    # columns agree up to the rounding the recurrence amplifies
    assert np.max(np.abs(rows[:10] - r["basis"][:10])) <= 1e-9
    # thermal weights: squared first components of the Ritz vectors
    np.testing.assert_allclose(q.eigenvectors[0] ** 2, r["vectors"][0] ** 2, atol=1e-8)


@pytest.mark.parametrize("sites,up,momentum,parity,storage", CASES)
def test_thermal_iteration_matches_oracle(engine, lz, oracle, sites, up, momentum, parity, storage):
    g, o = _sector(engine, oracle, sites, up, momentum, parity, storage)
    rng = np.random.default_rng(sites + 1)
    v = rng.standard_normal(g.dim) + (0.0 if o.is_real else 1j * rng.standard_normal(g.dim))
    betas = [0.0, 0.1, 0.5, 2.0, 10.0]
    lzg, eg, mg = lz.thermal_iteration(g, v, betas, 60)
    lzo, eo, mo = o.thermal_iteration(v, betas, 60)
    assert mg == mo == 60
    np.testing.assert_allclose(lzg, lzo, atol=1e-10)
    np.testing.assert_allclose(eg, eo, atol=1e-10)
    assert abs(lzg[0] - np.log(g.dim)) <= 1e-12 * np.log(g.dim)


def test_thermal_iteration_exact_on_exhausted_krylov_space(engine, lz, oracle):
    g, o = _sector(engine, oracle, 10, 5, 0, 1, "packed")
    dense = o.dense()
    w, u = np.linalg.eigh(dense)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(g.dim)
    betas = [0.0, 0.3, 1.0, 4.0]
    logz, energy, m = lz.thermal_iteration(g, v, betas, g.dim + 5, 1e-10)
    assert m <= g.dim
    overlap = np.abs(u.T @ v) ** 2
    for b, l_, e_ in zip(betas, logz, energy):
        boltz = overlap * np.exp(-b * (w - w.min()))
        exact = np.log(g.dim / np.dot(v, v)) - b * w.min() + np.log(boltz.sum())
        assert abs(l_ - exact) <= 1e-9
        assert abs(e_ - (boltz * w).sum() / boltz.sum()) <= 1e-9
    # exponential action through the stored basis equals the dense exponential
    from scipy.linalg import expm
    q = lz.LanczosBasis(g, v, g.dim + 5, 1e-10)
    np.testing.assert_allclose(q.exponential_action(-0.4 + 0.3j), expm((-0.4 + 0.3j) * dense) @ v, atol=1e-9)
    coeff = rng.standard_normal(q.krylov_dimension) + 1j * rng.standard_normal(q.krylov_dimension)
    np.testing.assert_allclose(lz.lin_comb_Q_T(coeff, q), coeff @ q.to_numpy(), atol=1e-12)


@pytest.mark.parametrize("sites,up,momentum,parity,storage", CASES)
@pytest.mark.parametrize("method", ["ftlm", "ltlm"])
def test_thermal_observables_match_oracle(engine, lz, oracle, sites, up, momentum, parity, storage, method):
    g, o = _sector(engine, oracle, sites, up, momentum, parity, storage)
    gb = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity)
    ob = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    zz = [("zz", [(1.0, (i, (i + 1) % sites)) for i in range(sites)])]
    xy = [("+-", [(0.5, (i, (i + 2) % sites)) for i in range(sites)]),
          ("-+", [(0.5, (i, (i + 2) % sites)) for i in range(sites)])]
    g_obs = [engine.GpuOperator(gb, zz, storage=storage), engine.GpuOperator(gb, xy, storage=storage)]
    o_obs = [oracle.Operator.build(ob, zz), oracle.Operator.build(ob, xy)]
    rng = np.random.default_rng(sites + 2)
    v = rng.standard_normal(g.dim) + (0.0 if o.is_real else 1j * rng.standard_normal(g.dim))
    betas = [0.0, 0.5, 3.0]
    q = lz.LanczosBasis(g, v, 30, 1e-12)
    values, identity = q.thermal({"zz": g_obs[0], "xy": g_obs[1]}, betas, method)
    ref, ref_identity = o.thermal_observables(v, o_obs, betas, 30, 1e-12, method)
    scale = np.max(np.abs(ref_identity))
    np.testing.assert_allclose(identity, ref_identity, atol=1e-10 * scale)
    np.testing.assert_allclose(values["zz"], ref[0], atol=1e-9 * scale)
    np.testing.assert_allclose(values["xy"], ref[1], atol=1e-9 * scale)


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def _rademacher(n, seed, r):
    """The sampler's start vector r (random_start_kernel), restated in numpy."""
    with np.errstate(over="ignore"):
        key = np.uint64((seed * 0xD1B54A32D192ED03 + r * 0x8CB92BA72F3D8DD7 + 1) & 0xFFFFFFFFFFFFFFFF)
        bits = _splitmix64(key ^ _splitmix64(np.arange(n, dtype=np.uint64)))
    return np.where(bits >> np.uint64(63), -1.0, 1.0)


def test_ftlm_sample_matches_oracle_per_vector(engine, lz, oracle):
    g, o = _sector(engine, oracle, 12, 6, 0, 1, "packed")
    betas = [0.0, 0.5, 2.0]
    logz, energy, lengths = lz.ftlm_sample(g, 4, betas, 40, seed=9)
    assert list(lengths) == [40] * 4
    for r in range(4):
        v = _rademacher(g.dim, 9, r)
        np.testing.assert_array_equal(lz.ftlm_start(g, r, seed=9), v.astype(complex))
        lzo, eo, _ = o.thermal_iteration(v, betas, 40)
        np.testing.assert_allclose(logz[r], lzo, atol=1e-10)
        np.testing.assert_allclose(energy[r], eo, atol=1e-10)
    np.testing.assert_allclose(logz[:, 0], np.log(g.dim), rtol=1e-13)


def test_ftlm_average_approaches_the_exact_thermodynamics(engine, lz, oracle):
    g, o = _sector(engine, oracle, 12, 6, None, None, "packed")
    w = np.linalg.eigvalsh(o.dense())
    betas = np.array([0.2, 1.0])
    logz, energy, _ = lz.ftlm_sample(g, 40, betas, 60, seed=1)
    avg_lz, avg_e = lz.ftlm_average(logz, energy)
    exact_lz = np.log(np.exp(-betas[:, None] * (w - w.min())).sum(axis=1)) - betas * w.min()
    exact_e = (np.exp(-betas[:, None] * (w - w.min())) * w).sum(axis=1) / np.exp(
        -betas[:, None] * (w - w.min())).sum(axis=1)
    # the sampling error, estimated from the samples themselves: relative
    # standard error of Z, and the standard error of the weighted energy mean
    w = np.exp(logz - logz.max(axis=0))
    z_err = w.std(axis=0) / w.mean(axis=0) / np.sqrt(len(w))
    e_err = np.sqrt((w ** 2 * (energy - avg_e) ** 2).sum(axis=0)) / w.sum(axis=0)
    assert np.all(np.abs(avg_lz - exact_lz) <= 4.0 * z_err + 1e-3)
    assert np.all(np.abs(avg_e - exact_e) <= 4.0 * e_err + 1e-3)
    assert np.all(z_err < 0.2)


def test_large_sector_properties(engine, lz):
    """L=24 Sz=0 k=0 p=+1 with 120 steps: orthonormal basis (LTLM projection of
    the identity is Q^H Q), log Z(0) = ln D, E(0) = <v|H|v>/<v|v>."""
    sites = 24
    gb = engine.GpuBasis(sites, up=12, momentum=0, parity=1)
    g = engine.GpuOperator(gb, engine.heisenberg_terms(sites, delta=1.0))
    identity = engine.GpuOperator(gb, [("I", [(1.0, (0,))])])
    rng = np.random.default_rng(24)
    v = rng.standard_normal(g.dim)
    q = lz.LanczosBasis(g, v, 120, 1e-12)
    assert q.krylov_dimension == 120
    gram = q.project(identity, "ltlm")
    assert np.max(np.abs(gram - np.eye(120))) <= 1e-12
    logz, energy, _ = lz.thermal_iteration(g, v, [0.0, 1.0], 120)
    assert abs(logz[0] - np.log(g.dim)) <= 1e-12 * np.log(g.dim)
    assert abs(energy[0] - np.vdot(v, g.apply(v)).real / np.dot(v, v)) <= 1e-9
    assert abs(energy[0] - q.diagonal[0]) <= 1e-9


def test_thermal_errors(engine, lz):
    from qmbed_b200 import QmbedError
    op = _two_level(engine, [-1.0, 2.0])
    v = np.ones(2, complex)
    for betas, krylov, tol, code in (([], 2, 1e-12, 8), ([-1.0], 2, 1e-12, 8), ([np.nan], 2, 1e-12, 8),
                                     ([1.0], 0, 1e-12, 8), ([1.0], 2, 0.0, 8)):
        with pytest.raises(QmbedError) as e:
            lz.thermal_iteration(op, v, betas, krylov, tol)
        assert e.value.code == code
    with pytest.raises(QmbedError) as e:
        lz.thermal_iteration(op, np.zeros(2, complex), [1.0], 2)
    assert e.value.code == 14
    big = engine.GpuOperator(engine.GpuBasis(16, up=8), engine.heisenberg_terms(16))
    with pytest.raises(QmbedError) as e:
        lz.LanczosBasis(big, np.ones(big.dim), 9000)
    assert e.value.code == 11
    with pytest.raises(QmbedError) as e:
        lz.ftlm_sample(op, 0, [1.0], 2)
    assert e.value.code == 8


def test_lanczos_json_resource_anchor(anchors):
    """The JSON Lanczos resource round trip (bindings/capi/src/lib.rs:7483-7578)
    on a model expression."""
    from qmbed_b200 import QmbedError, _lib
    a = anchors["lanczos_json_resource"]

    def model(c_identity, c_z):
        return _lib.command({"operation": "create_model", "basis": {"kind": "spin", "sites": 1},
                             "terms": [{"product": {"local": ["identity"]},
                                        "couplings": [{"coefficient": [c_identity, 0.0], "sites": [0]}]},
                                       {"product": {"local": ["z"]},
                                        "couplings": [{"coefficient": [c_z, 0.0], "sites": [0]}]}]})["handle"]

    probe = model(0.0, 1.0)
    z = [_lib.command({"operation": "apply_model", "handle": probe, "action": "normal",
                       "vectors": [[[1.0 if i == j else 0.0, 0.0] for i in range(2)]]})["vectors"][0][j][0]
         for j in range(2)]
    d = a["diagonal"]
    b = (d[1] - d[0]) / (z[1] - z[0])
    h = model(d[0] - b * z[0], b)
    one = model(1.0, 0.0)
    # the form the reference's QuSpin-compatible tools send for a hamiltonian
    expr = {"kind": "model", "handle": h, "parameters": {}, "action": "normal"}
    result = _lib.command({"operation": "lanczos_operator", "expression": expr, "initial": a["initial"],
                           "krylov_dimension": a["krylov_dimension"], "tolerance": a["tolerance"]})
    assert result["kind"] == "lanczos" and result["krylov_dimension"] == 2
    handle = result["handle"]
    assert handle.startswith("lanczos:")
    exp = _lib.command({"operation": "lanczos_exponential", "lanczos_handle": handle,
                        "coefficient": a["exponential_coefficient"]})
    expected = [0.6 * np.exp(0.25j), 0.8 * np.exp(-0.5j)]
    for actual, e in zip(exp["vectors"][0], expected):
        assert abs(actual[0] - e.real) < a["abs_tol"] and abs(actual[1] - e.imag) < a["abs_tol"]
    exported = _lib.command({"operation": "export_lanczos_basis", "lanczos_handle": handle})
    assert len(exported["vectors"]) == 2
    thermal = _lib.command({"operation": "lanczos_thermal", "lanczos_handle": handle, "method": "ftlm",
                            "eigenvalues": result["eigenvalues"], "eigenvectors": result["eigenvectors"],
                            "inverse_temperatures": a["inverse_temperatures"],
                            "observables": [{"name": "I", "expression": {"kind": "model", "handle": one}}]})
    # exact equality in the reference; here the basis overlap <q_1|q_0> is zero to rounding
    for value, ident in zip(thermal["values"]["I"], thermal["identity"]):
        assert abs(value[0] - ident) <= 1e-15 * abs(ident) and abs(value[1]) <= 1e-15
    # projected matrix elements need no handle
    pre = _lib.command({"operation": "lanczos_thermal", "method": "ltlm", "eigenvalues": [0.0],
                        "eigenvectors": [[1.0]], "inverse_temperatures": [1.0],
                        "observables": [{"name": "A", "matrix_elements": [[2.0, 0.0]]}]})
    assert abs(pre["values"]["A"][0][0] - 2.0) < 1e-15 and abs(pre["identity"][0] - 1.0) < 1e-15
    with pytest.raises(QmbedError, match="exactly one expression"):
        _lib.command({"operation": "lanczos_thermal", "method": "ftlm", "eigenvalues": [0.0], "eigenvectors": [[1.0]],
                      "inverse_temperatures": [1.0], "observables": [{"name": "A"}]})
    with pytest.raises(QmbedError, match="^unsupported backend: conjugate and transpose actions"):
        _lib.command({"operation": "lanczos_operator", "expression": {**expr, "action": "transpose"},
                      "initial": a["initial"], "krylov_dimension": 2})
    assert _lib.command({"operation": "release_lanczos", "lanczos_handle": handle})["kind"] == "released"
    with pytest.raises(QmbedError):
        _lib.command({"operation": "export_lanczos_basis", "lanczos_handle": handle})
    for m in (probe, h, one):
        _lib.command({"operation": "release_model", "handle": m})
