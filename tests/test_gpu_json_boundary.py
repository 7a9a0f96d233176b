"""The JSON drop-in boundary (qmbed_run_json / qmbed_command_json) on the GPU.

Requests use the reference schema (bindings/capi/src/lib.rs:55-741,
2064-2204); answers are checked against the reference's own C-ABI test
anchors and against the CPU oracle.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def heisenberg_request_terms(sites, periodic=True, delta=1.0):
    bonds = [[i, (i + 1) % sites] for i in range(sites if periodic else sites - 1)]
    return [
        {"product": {"local": ["z", "z"]}, "couplings": [{"coefficient": [delta, 0.0], "sites": b} for b in bonds]},
        {"product": {"local": ["raising", "lowering"]},
         "couplings": [{"coefficient": [0.5, 0.0], "sites": b} for b in bonds]},
        {"product": {"local": ["lowering", "raising"]},
         "couplings": [{"coefficient": [0.5, 0.0], "sites": b} for b in bonds]},
    ]


def test_typed_json_request_reaches_the_solver():
    """bindings/capi/src/lib.rs:6311-6329: the dimer answers -0.75, 0.25."""
    from qmbed_b200._lib import run
    result = run({"basis": {"kind": "spin", "sites": 2}, "terms": heisenberg_request_terms(2, periodic=False),
                  "solver": {"eigenpairs": 2, "target": {"kind": "smallest_algebraic"}, "tolerance": 1e-12}})
    assert result["dimension"] == 4
    np.testing.assert_allclose(result["eigenvalues"], [-0.75, 0.25], atol=1e-12)
    assert result["converged"] is True


def test_reference_style_python_api(oracle):
    import qmbed_b200 as q
    basis = q.SpinBasis(sites=16, up=8, momentum=0, parity=1)
    for precision in ("fp64", "mixed"):
        result = q.eigsh(basis, q.heisenberg_specs(16), q.EigshOptions(3, krylov_dimension=32, tolerance=1e-10,
                                                                        seed=3, precision=precision))
        o = oracle.Operator.build(oracle.Basis(16, up=8, momentum=0, parity=1), oracle.heisenberg_terms(16))
        expected = o.eigsh(3, krylov_dimension=32, tolerance=1e-10, seed=3).eigenvalues
        np.testing.assert_allclose(result.eigenvalues, expected, rtol=1e-10)


def test_models_apply_and_expm_commands(oracle):
    import qmbed_b200 as q
    request = {"basis": {"kind": "spin", "sites": 10, "up": 5, "momentum": 0},
               "terms": heisenberg_request_terms(10)[1:],
               "components": [{"name": "delta", "terms": heisenberg_request_terms(10)[:1], "default": [1.0, 0.0]}]}
    with q.NativeModel(request) as model:
        o = oracle.Operator.build(oracle.Basis(10, up=5, momentum=0), oracle.heisenberg_terms(10, delta=0.4))
        x = oracle.deterministic_start(model.dimension, 5)
        y = model.apply(x, parameters={"delta": 0.4})
        np.testing.assert_allclose(y[0], o.apply(x), atol=1e-13)
        r = model.eigsh(q.EigshOptions(2, tolerance=1e-12, seed=2), parameters={"delta": 0.4})
        np.testing.assert_allclose(r.eigenvalues, o.eigsh(2, tolerance=1e-12, seed=2).eigenvalues, rtol=1e-10)
        with q.NativeExpmAction(model, -0.5j, parameters={"delta": 0.4}) as plan:
            out = plan.apply(x)
            np.testing.assert_allclose(out[0], o.expm_apply(-0.5j, x), atol=1e-12)


def test_error_responses_carry_reference_texts():
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command, run
    with pytest.raises(QmbedError, match="incompatible symmetry request"):
        run({"basis": {"kind": "spin", "sites": 4, "up": 2, "momentum": 1, "parity": 1},
             "terms": heisenberg_request_terms(4), "solver": {"eigenpairs": 1, "target": {"kind": "smallest_algebraic"}}})
    with pytest.raises(QmbedError, match="model handle 99999 is not registered"):
        command({"operation": "eigsh_model", "handle": "99999",
                 "solver": {"eigenpairs": 1, "target": {"kind": "smallest_algebraic"}}})
    with pytest.raises(QmbedError, match="a Hermitian operator is required"):
        run({"basis": {"kind": "spin", "sites": 4, "up": 2},
             "terms": heisenberg_request_terms(4)[1:2],
             "solver": {"eigenpairs": 1, "target": {"kind": "smallest_algebraic"}}})


def test_describe_basis_lists_decimal_states(oracle):
    from qmbed_b200._lib import command
    result = command({"operation": "describe_basis", "basis": {"kind": "spin", "sites": 8, "up": 4, "momentum": 0}})
    states, _ = oracle.Basis(8, up=4, momentum=0).states()
    assert result["dimension"] == len(states)
    assert result["states"] == [str(int(s)) for s in states]


def test_operator_expression_commands(oracle):
    """eigsh/apply/expm_operator_expression (bindings/capi/src/lib.rs:4078-4190)
    on the model expressions the reference's QuSpin-compatible layer sends."""
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    request = {"basis": {"kind": "spin", "sites": 10, "up": 5, "momentum": 0},
               "terms": heisenberg_request_terms(10)[1:],
               "components": [{"name": "delta", "terms": heisenberg_request_terms(10)[:1], "default": [1.0, 0.0]}]}
    handle = command({"operation": "create_model", **request})["handle"]
    o = oracle.Operator.build(oracle.Basis(10, up=5, momentum=0), oracle.heisenberg_terms(10, delta=0.4))
    expr = {"kind": "model", "handle": handle, "parameters": {"delta": [0.4, 0.0]}, "action": "normal"}
    x = oracle.deterministic_start(o.dim, 5)
    xs = [[[float(v), 0.0] for v in x]]
    applied = command({"operation": "apply_operator_expression", "expression": expr, "vectors": xs})
    assert applied["kind"] == "vectors" and applied["dimension"] == o.dim
    np.testing.assert_allclose([complex(*p) for p in applied["vectors"][0]], o.apply(x), atol=1e-13)
    solved = command({"operation": "eigsh_operator_expression", "expression": expr, "format": "csr",
                      "solver": {"eigenpairs": 2, "target": {"kind": "smallest_algebraic"}, "tolerance": 1e-12,
                                 "seed": 2}})
    np.testing.assert_allclose(solved["eigenvalues"], o.eigsh(2, tolerance=1e-12, seed=2).eigenvalues, rtol=1e-10)
    exp = command({"operation": "expm_operator_expression", "expression": expr, "coefficient": [0.0, -0.5],
                   "vectors": xs})
    np.testing.assert_allclose([complex(*p) for p in exp["vectors"][0]], o.expm_apply(-0.5j, x), atol=1e-12)
    # JSON errors carry the reference's Display texts (src/error.rs:6-35)
    with pytest.raises(QmbedError, match="^dimension mismatch: operator expression inputs"):
        command({"operation": "apply_operator_expression", "expression": expr, "vectors": []})
    with pytest.raises(QmbedError, match="^invalid options: operator exponential requires a nonempty"):
        command({"operation": "expm_operator_expression", "expression": expr, "coefficient": [0.0, -0.5],
                 "vectors": []})
    with pytest.raises(QmbedError, match="^unsupported backend: operator expressions of kind `matrix`"):
        command({"operation": "apply_operator_expression", "vectors": xs,
                 "expression": {"kind": "matrix", "operator": {"shape": [1, 1], "entries": []}}})
    command({"operation": "release_model", "handle": handle})


@pytest.mark.parametrize("sites", [20, 100])
def test_apply_terms_between_models(oracle, sites):
    """apply_terms_between_models (bindings/capi/src/lib.rs:4871-4915; anchor
    6586-6626): sum_j S+_j from the k=0 all-down sector into the k=0 one-magnon
    sector multiplies by sqrt(L)."""
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    src = command({"operation": "create_model", "basis": {"kind": "spin", "sites": sites, "up": 0, "momentum": 0},
                   "terms": []})["handle"]
    tgt = command({"operation": "create_model", "basis": {"kind": "spin", "sites": sites, "up": 1, "momentum": 0},
                   "terms": []})["handle"]
    raising = [{"product": {"local": ["raising"]},
                "couplings": [{"coefficient": [1.0, 0.0], "sites": [j]} for j in range(sites)]}]
    out = command({"operation": "apply_terms_between_models", "source_handle": src, "target_handle": tgt,
                   "terms": raising, "vectors": [[[1.0, 0.0]]]})
    assert out["kind"] == "vectors" and out["dimension"] == 1
    assert abs(out["vectors"][0][0][0] - np.sqrt(sites)) < 1e-12 and abs(out["vectors"][0][0][1]) < 1e-12
    if sites == 20:
        # a momentum-changing shift on larger sectors against the oracle
        a = command({"operation": "create_model", "basis": {"kind": "spin", "sites": 12, "up": 6, "momentum": 1},
                     "terms": []})["handle"]
        b = command({"operation": "create_model", "basis": {"kind": "spin", "sites": 12, "up": 5, "momentum": 4},
                     "terms": []})["handle"]
        coeff = [np.exp(-2j * np.pi * 3 * j / 12) for j in range(12)]
        lowering = [{"product": {"local": ["lowering"]},
                     "couplings": [{"coefficient": [c.real, c.imag], "sites": [j]} for j, c in enumerate(coeff)]}]
        ob_s, ob_t = oracle.Basis(12, up=6, momentum=1), oracle.Basis(12, up=5, momentum=4)
        x = np.random.default_rng(1).standard_normal(len(ob_s))
        out = command({"operation": "apply_terms_between_models", "source_handle": a, "target_handle": b,
                       "terms": lowering, "vectors": [[[float(v), 0.0] for v in x]]})
        ref = oracle.sector_shift(ob_s, ob_t, [("-", [(c, (j,)) for j, c in enumerate(coeff)])], x)
        np.testing.assert_allclose([complex(*p) for p in out["vectors"][0]], ref, atol=1e-13)
        with pytest.raises(QmbedError, match="^dimension mismatch"):
            command({"operation": "apply_terms_between_models", "source_handle": a, "target_handle": b,
                     "terms": lowering, "vectors": [[[1.0, 0.0]]]})
        for m in (a, b):
            command({"operation": "release_model", "handle": m})
    for m in (src, tgt):
        command({"operation": "release_model", "handle": m})


@pytest.mark.parametrize("momentum,parity", [(0, 1), (3, None)])
def test_eigh_model_matches_dense_spectrum(oracle, momentum, parity):
    """eigh_model / eigh_operator_expression (bindings/capi/src/lib.rs:5290-5300,
    src/solve/mod.rs:585-605): every eigenpair, ascending, with residuals."""
    from qmbed_b200._lib import command
    sites = 10
    basis = {"kind": "spin", "sites": sites, "up": 5, "momentum": momentum}
    if parity is not None:
        basis["parity"] = parity
    handle = command({"operation": "create_model", "basis": basis,
                      "terms": heisenberg_request_terms(sites, delta=0.6)})["handle"]
    o = oracle.Operator.build(oracle.Basis(sites, up=5, momentum=momentum, parity=parity),
                              oracle.heisenberg_terms(sites, delta=0.6))
    w = np.linalg.eigvalsh(o.dense())
    out = command({"operation": "eigh_model", "handle": handle, "eigenvectors": True})
    assert out["kind"] == "eigensystem" and out["dimension"] == o.dim and out["converged"] is True
    assert out["iterations"] == 1
    np.testing.assert_allclose(out["eigenvalues"], w, atol=1e-12)
    assert max(out["residuals"]) < 1e-11
    vecs = np.array([[complex(*p) for p in v] for v in out["eigenvectors"]])
    np.testing.assert_allclose(vecs.conj() @ vecs.T, np.eye(o.dim), atol=1e-11)
    for lam, v in zip(out["eigenvalues"], vecs[:3]):
        assert np.linalg.norm(o.apply(v) - lam * v) < 1e-11
    expr = command({"operation": "eigh_operator_expression",
                    "expression": {"kind": "model", "handle": handle, "action": "normal"}})
    np.testing.assert_allclose(expr["eigenvalues"], w, atol=1e-12)
    assert "eigenvectors" not in expr
    command({"operation": "release_model", "handle": handle})


def test_eigh_model_dimer_and_size_limit():
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    dimer = command({"operation": "create_model", "basis": {"kind": "spin", "sites": 2},
                     "terms": heisenberg_request_terms(2, periodic=False)})["handle"]
    out = command({"operation": "eigh_model", "handle": dimer})
    np.testing.assert_allclose(out["eigenvalues"], [-0.75, 0.25, 0.25, 0.25], atol=1e-13)
    # a sector of 3432 states through the dense solver, against the oracle's Lanczos
    mid = command({"operation": "create_model", "basis": {"kind": "spin", "sites": 14, "up": 7},
                   "terms": heisenberg_request_terms(14)})["handle"]
    full = command({"operation": "eigh_model", "handle": mid})
    assert full["dimension"] == 3432 and max(full["residuals"]) < 1e-10
    lowest = command({"operation": "eigsh_model", "handle": mid,
                      "solver": {"eigenpairs": 3, "target": {"kind": "smallest_algebraic"}, "tolerance": 1e-12}})
    np.testing.assert_allclose(full["eigenvalues"][:3], lowest["eigenvalues"], atol=1e-10)
    command({"operation": "release_model", "handle": mid})
    big = command({"operation": "create_model", "basis": {"kind": "spin", "sites": 20, "up": 10},
                   "terms": heisenberg_request_terms(20)})["handle"]
    with pytest.raises(QmbedError, match="^unsupported backend: dense eigh"):
        command({"operation": "eigh_model", "handle": big})
    for h in (dimer, big):
        command({"operation": "release_model", "handle": h})


def test_materialize_model_matches_oracle(oracle):
    """materialize_model (bindings/capi/src/lib.rs:5652-5659) with a component parameter."""
    from qmbed_b200._lib import command
    request = {"basis": {"kind": "spin", "sites": 8, "up": 4, "momentum": 0},
               "terms": heisenberg_request_terms(8)[1:],
               "components": [{"name": "delta", "terms": heisenberg_request_terms(8)[:1], "default": [1.0, 0.0]}]}
    handle = command({"operation": "create_model", **request})["handle"]
    out = command({"operation": "materialize_model", "handle": handle, "parameters": {"delta": [0.3, 0.0]}})
    o = oracle.Operator.build(oracle.Basis(8, up=4, momentum=0), oracle.heisenberg_terms(8, delta=0.3))
    n = o.dim
    assert out["kind"] == "operator" and out["shape"] == [n, n]
    dense = np.zeros((n, n), complex)
    for e in out["entries"]:
        dense[e["row"], e["column"]] += complex(*e["value"])
    np.testing.assert_allclose(dense, o.dense(), atol=1e-13)
    command({"operation": "release_model", "handle": handle})


def test_native_model_eigh(oracle):
    import qmbed_b200 as q
    request = {"basis": {"kind": "spin", "sites": 10, "up": 5, "momentum": 0},
               "terms": heisenberg_request_terms(10)[1:],
               "components": [{"name": "delta", "terms": heisenberg_request_terms(10)[:1], "default": [1.0, 0.0]}]}
    with q.NativeModel(request) as model:
        r = model.eigh(eigenvectors=True, parameters={"delta": 0.4})
    o = oracle.Operator.build(oracle.Basis(10, up=5, momentum=0), oracle.heisenberg_terms(10, delta=0.4))
    np.testing.assert_allclose(r.eigenvalues, np.linalg.eigvalsh(o.dense()), atol=1e-12)
    assert len(r.eigenvectors) == o.dim and max(r.residuals) < 1e-11
