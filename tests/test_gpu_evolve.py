"""Krylov exponential action on the GPU against the CPU oracle.

Reference behaviour: src/solve/mod.rs:2909-3316 (Lanczos projections without
reorthogonalisation, a-posteriori error bound, adaptive time grid) and
3432-3454 (expm_lanczos). States agree with the FP64 oracle within 1e-9 in
2-norm; the reference anchor of tests/solver_extensions.rs:264-293 holds.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _ladder_terms(levels_log2):
    # Pauli z on site i with coefficient 2^i * 2/31 gives the 32 levels -2 + 4 idx / 31
    return [("z", [(-(2.0 ** i) * 2.0 / 31.0, (i,)) for i in range(levels_log2)])]


def test_adaptive_evolution_anchor_on_gpu(engine, oracle, anchors):
    a = anchors["adaptive_evolution"]
    terms = _ladder_terms(5)
    g = engine.GpuOperator(engine.GpuBasis(5, normalization="pauli"), terms)
    o = oracle.Operator.build(oracle.Basis(5, normalization="pauli"), terms)
    energies = np.array([o.apply(np.eye(32)[i])[i].real for i in range(32)])
    assert np.allclose(np.sort(energies), [-2.0 + 4.0 * i / 31.0 for i in range(32)], atol=1e-14)
    initial = np.full(32, 1.0 / np.sqrt(32.0), complex)
    states, d = g.evolve(initial, a["times"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"])
    assert d["lanczos_projections"] > 1
    assert d["matrix_vector_products"] == a["krylov_dimension"] * d["lanczos_projections"]
    assert d["accepted_substeps"] == d["lanczos_projections"]
    assert d["rejected_trial_intervals"] > 0
    assert d["real_lanczos_projections"] == 1
    expected = initial * np.exp(-1j * a["times"][2] * energies)
    assert np.max(np.abs(states[2] - expected)) < a["final_state_abs_tol"]
    ostates, od = o.evolve(initial, a["times"], krylov_dimension=a["krylov_dimension"], tolerance=a["tolerance"])
    for s, t in zip(states, ostates):
        assert np.linalg.norm(s - t) <= 1e-9
    assert d["lanczos_projections"] == od["lanczos_projections"]


@pytest.mark.parametrize("sites,up,momentum,parity,storage", [
    (16, 8, 0, 1, "packed"),        # real sector: first projection on the real path
    (15, None, 3, None, "packed"),  # complex sector
    (14, 7, None, None, "matrix_free"),
])
def test_evolve_matches_oracle(engine, oracle, sites, up, momentum, parity, storage):
    terms = oracle.heisenberg_terms(sites, delta=0.7)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms, storage=storage)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity), terms)
    n = g.dim
    rng = np.random.default_rng(sites)
    v = rng.standard_normal(n)
    if not g.is_real:
        v = v + 1j * rng.standard_normal(n)
    v = v / np.linalg.norm(v)
    times = [0.0, 0.25, 0.25, 1.0, 3.0]
    states, d = g.evolve(v, times, krylov_dimension=24, tolerance=1e-10)
    ostates, od = o.evolve(v, times, krylov_dimension=24, tolerance=1e-10)
    errors = [float(np.linalg.norm(s - t)) for s, t in zip(states, ostates)]
    assert max(errors) <= 1e-9, errors
    for s in states:
        assert abs(np.linalg.norm(s) - 1.0) < 1e-12
    assert d["matrix_vector_products"] == od["matrix_vector_products"]
    assert d["accepted_substeps"] == od["accepted_substeps"]
    assert (d["real_lanczos_projections"] > 0) == g.is_real


def test_complex_vectors_on_real_packed_rows(engine, oracle):
    terms = oracle.heisenberg_terms(18, delta=0.9)
    g = engine.GpuOperator(engine.GpuBasis(18, up=9, momentum=0, parity=1), terms)
    o = oracle.Operator.build(oracle.Basis(18, up=9, momentum=0, parity=1), terms)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(g.dim) + 1j * rng.standard_normal(g.dim)
    y = g.apply(x)
    ref = o.apply(x)
    assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)


def test_expm_lanczos_matches_oracle(engine, oracle):
    terms = oracle.heisenberg_terms(14, delta=1.3)
    g = engine.GpuOperator(engine.GpuBasis(14, up=7, momentum=0), terms)
    o = oracle.Operator.build(oracle.Basis(14, up=7, momentum=0), terms)
    v = oracle.deterministic_start(g.dim, 4).astype(complex)
    for t, m in ((0.3, 30), (-1.1, 40), (0.0, 5)):
        w = g.expm_lanczos(v, t, krylov_dimension=m)
        assert np.linalg.norm(w - o.expm_lanczos(v, t, krylov_dimension=m)) <= 1e-9


def test_evolution_errors(engine, oracle):
    from qmbed_b200 import QmbedError
    g = engine.GpuOperator(engine.GpuBasis(8, up=4), oracle.heisenberg_terms(8))
    v = np.zeros(g.dim, complex)
    v[0] = 1.0
    for times, m, tol in (([], 8, 1e-10), ([1.0, 0.5], 8, 1e-10), ([float("nan")], 8, 1e-10), ([1.0], 0, 1e-10),
                          ([1.0], 8, -1.0)):
        with pytest.raises(QmbedError) as e:
            g.evolve(v, times, krylov_dimension=m, tolerance=tol)
        assert e.value.code == 8
    with pytest.raises(QmbedError) as e:
        g.evolve(v, [100.0], krylov_dimension=2, tolerance=1e-14, max_substeps=3)
    assert e.value.code == 14
    with pytest.raises(QmbedError) as e:
        g.expm_lanczos(v, float("inf"))
    assert e.value.code == 8


def test_evolve_model_json_anchor(anchors):
    from qmbed_b200 import QmbedError, _lib
    a = anchors["evolve_model_json"]
    created = _lib.command({"operation": "create_model", **a["request"]})
    handle = created["handle"]
    result = _lib.command({"operation": "evolve_model", "handle": handle, "vectors": a["vectors"],
                           "evolution": a["evolution"]})
    assert result["kind"] == "trajectory" and result["dimension"] == 2
    assert result["times"] == a["evolution"]["times"]
    states = result["states"]
    assert len(states) == 2 and len(states[0]) == 2
    for column in range(2):
        for component in range(2):
            expected = 1.0 if column == component else 0.0
            initial = states[0][column][component]
            assert abs(initial[0] - expected) < a["abs_tol"] and abs(initial[1]) < a["abs_tol"]
            final = states[1][column][component]
            assert abs(final[0]) < a["abs_tol"] and abs(final[1] + expected) < a["abs_tol"]
    with pytest.raises(QmbedError, match="imaginary-time"):
        _lib.command({"operation": "evolve_model", "handle": handle, "vectors": a["vectors"],
                      "evolution": {"times": [1.0], "imaginary_time": True}})
    with pytest.raises(QmbedError, match="at least one column"):
        _lib.command({"operation": "evolve_model", "handle": handle, "vectors": [], "evolution": {"times": [1.0]}})
    assert _lib.command({"operation": "release_model", "handle": handle})["kind"] == "released"


def test_native_model_evolve(oracle):
    from qmbed_b200.model import NativeModel
    bonds = [[i, (i + 1) % 10] for i in range(10)]
    request = {"basis": {"kind": "spin", "sites": 10, "up": 5, "momentum": 0},
               "terms": [{"product": {"local": ["z", "z"]},
                          "couplings": [{"coefficient": [1.0, 0.0], "sites": b} for b in bonds]},
                         {"product": {"local": ["raising", "lowering"]},
                          "couplings": [{"coefficient": [0.5, 0.0], "sites": b} for b in bonds]},
                         {"product": {"local": ["lowering", "raising"]},
                          "couplings": [{"coefficient": [0.5, 0.0], "sites": b} for b in bonds]}]}
    o = oracle.Operator.build(oracle.Basis(10, up=5, momentum=0), oracle.heisenberg_terms(10))
    v = oracle.deterministic_start(o.dim, 3).astype(complex)
    with NativeModel(request) as model:
        states = model.evolve([v], [0.5, 1.5], krylov_dimension=30)
    ref, _ = o.evolve(v, [0.5, 1.5], krylov_dimension=30)
    assert states.shape == (2, 1, o.dim)
    for t in range(2):
        assert np.linalg.norm(states[t][0] - ref[t]) <= 1e-9
