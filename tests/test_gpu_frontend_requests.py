"""Requests of the reference's unmodified Python frontend, replayed on the GPU.

``tests/golden/frontend_requests.json`` holds, in order, the JSON requests that
the reference's ``qmbed`` package and its QuSpin-compatible ``quspin`` package
send for a few ordinary user scripts (recorded by
``tests/golden/make_frontend_requests.py``): the native ``qmbed.eigsh`` and
QuSpin ``hamiltonian`` objects on ``spin_basis_1d`` with ``kblock``/``pblock``
lattice maps, reversed row order and the reversed site labelling, with
``eigsh``, ``dot``, ``expt_value``, ``quant_fluct``, ``matrix_ele``,
``eigvalsh``, the Krylov ``evolve``, the Lanczos tools on a ``zblock``
sector and ``expm_multiply_parallel`` on explicit sparse matrices. Each
request goes unchanged through
``qmbed_run_json`` / ``qmbed_command_json`` of ``libqmbed_b200.so`` (model
handles are mapped to the ones this library returned) and each answer is
checked against the oracle's answer to the same request
(``tests/frontend_protocol.py``).
"""

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "frontend_requests.json"
SCENARIOS = json.loads(FIXTURE.read_text())


def _complex(vectors):
    return [np.array([complex(*v) for v in vec]) for vec in vectors]


def _check_eigensystem(got, expected, h, solver):
    scale = np.maximum(1.0, np.abs(expected["eigenvalues"]))
    np.testing.assert_allclose(sorted(got["eigenvalues"]), sorted(expected["eigenvalues"]), atol=1e-8 * scale.max())
    assert got["dimension"] == expected["dimension"]
    if solver.get("eigenvectors"):
        vectors = _complex(got["eigenvectors"])
        assert len(vectors) == len(got["eigenvalues"])
        for value, v in zip(got["eigenvalues"], vectors):
            assert abs(np.linalg.norm(v) - 1.0) <= 1e-10
            assert np.linalg.norm(h @ v - value * v) <= 1e-7 * max(1.0, abs(value))


def _substitute(value, handles):
    """The request with every recorded handle (model or Lanczos, at any depth) replaced by this library's."""
    if isinstance(value, dict):
        return {k: _substitute(v, handles) for k, v in value.items()}
    if isinstance(value, list):
        return [_substitute(v, handles) for v in value]
    if isinstance(value, str) and value in handles:
        return handles[value]
    return value


def _dense(result):
    h = np.zeros(result["shape"], dtype=complex)
    for e in result["entries"]:
        h[e["row"], e["column"]] += complex(*e["value"])
    return h


@pytest.mark.parametrize("scenario", sorted(SCENARIOS))
def test_frontend_requests_replay(scenario):
    from frontend_protocol import OracleProtocol, model_matrix
    from qmbed_b200._lib import command, run

    oracle = OracleProtocol()
    handles = {}
    for call in SCENARIOS[scenario]["calls"]:
        request = call["request"]
        expected = oracle.call(call["symbol"], request)
        sent = _substitute(request, handles)
        got = run(sent) if call["symbol"] == "qmbed_run_json" else command(sent)
        op = request.get("operation", "run")
        if op == "run":
            _check_eigensystem(got, expected, model_matrix(request), request["solver"])
        elif op in ("create_model", "create_operator_model", "create_expm_action"):
            handles[expected["handle"]] = got["handle"]
            assert got["dimension"] == expected["dimension"]
        elif op == "describe_basis":
            assert got["dimension"] == expected["dimension"] and got["states"] == expected["states"]
        elif op == "eigsh_model":
            _check_eigensystem(got, expected, oracle.matrix(request["handle"], request.get("parameters")),
                               request["solver"])
        elif op == "eigsh_operator_expression":
            _check_eigensystem(got, expected, oracle.expression_matrix(request["expression"]), request["solver"])
        elif op == "lanczos_operator":
            handles[expected["handle"]] = got["handle"]
            assert got["krylov_dimension"] == expected["krylov_dimension"]
            assert abs(got["initial_norm"] - expected["initial_norm"]) <= 1e-12 * expected["initial_norm"]
            scale = max(1.0, np.abs(expected["eigenvalues"]).max())
            np.testing.assert_allclose(got["eigenvalues"], expected["eigenvalues"], atol=1e-10 * scale)
            for a, b in zip(got["eigenvectors"], expected["eigenvectors"]):  # columns up to sign
                a, b = np.array(a), np.array(b)
                assert min(np.abs(a - b).max(), np.abs(a + b).max()) <= 1e-8
        elif op in ("materialize_model", "evaluate_operator_expression", "materialize_component_model"):
            assert got["shape"] == expected["shape"]
            assert np.abs(_dense(got) - _dense(expected)).max() <= 1e-12 * max(1.0, np.abs(_dense(expected)).max())
        elif op in ("lanczos_combine", "lanczos_exponential"):
            a = np.array(got["vectors"], dtype=float)
            b = np.array(expected["vectors"], dtype=float)
            assert a.shape == b.shape and np.abs(a - b).max() <= 1e-10 * max(1.0, np.abs(b).max())
        elif op in ("release_lanczos", "release_expm_action"):
            pass
        elif op in ("apply_model", "evolve_model", "apply_expm_action"):
            key = "states" if op == "evolve_model" else "vectors"
            a = np.array(got[key], dtype=float)
            b = np.array(expected[key], dtype=float)
            assert a.shape == b.shape
            tol = {"apply_model": 1e-12, "evolve_model": 1e-8, "apply_expm_action": 1e-12}[op]
            assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())
        elif op in ("measure_model", "matrix_elements_model"):
            assert got["kind"] == "measurements" and got["shape"] == expected["shape"]
            np.testing.assert_allclose(np.array(got["values"]), np.array(expected["values"]), rtol=1e-10, atol=1e-10)
        elif op == "eigh_model":
            np.testing.assert_allclose(got["eigenvalues"], expected["eigenvalues"], atol=1e-10)
        elif op == "release_model":
            pass
        else:
            raise AssertionError(f"unexpected request {op}")


def _quspin_maps(sites, kblock=None, pblock=None, zblock=None):
    """QuSpin's spin_basis_1d lattice maps: translation i -> i-1, reflection i -> L-1-i, global spin flip."""
    maps = []
    if kblock is not None:
        maps.append({"destinations": [(i - 1) % sites for i in range(sites)], "sector": kblock})
    if pblock is not None:
        maps.append({"destinations": [sites - 1 - i for i in range(sites)], "sector": 0 if pblock == 1 else 1})
    if zblock is not None:
        maps.append({"destinations": list(range(sites)), "sector": 0 if zblock == 1 else 1,
                     "local_permutations": [[1, 0]] * sites})
    return maps


@pytest.mark.parametrize("sites,up,kblock,pblock,zblock,reverse", [
    (10, 5, 0, 1, None, True), (10, 4, 3, None, None, True), (11, 5, 2, None, None, False),
    (9, None, 0, -1, None, True), (8, 3, None, None, None, True), (8, None, None, None, None, True),
    (10, 5, 0, 1, 1, True), (10, 5, 0, 1, -1, True), (12, 6, 6, -1, 1, True), (12, 6, 3, None, -1, True),
    (8, None, None, None, -1, True), (9, None, 0, 1, 1, False), (14, 7, 0, None, 1, False),
])
def test_lattice_map_bases_list_the_reference_states(sites, up, kblock, pblock, zblock, reverse):
    """describe_basis on lattice-map sectors: representatives, order and count of the oracle's general basis."""
    from oracle import general
    from qmbed_b200._lib import command
    maps = _quspin_maps(sites, kblock, pblock, zblock)
    basis = {"kind": "spin", "sites": sites, "up": up, "symmetries": maps, "reverse": reverse}
    got = command({"operation": "describe_basis", "basis": basis})
    expected = general.GeneralSpinBasis(sites, up, maps, reverse=reverse)
    assert got["dimension"] == len(expected)
    assert [int(s) for s in got["states"]] == [int(s) for s in expected.states]


def test_lattice_maps_and_site_labels_reject_what_the_engine_does_not_build():
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    L = 8
    base = {"kind": "spin", "sites": L, "up": 4}
    terms = [{"product": {"local": ["z", "z"]}, "couplings": [{"coefficient": [1.0, 0.0], "sites": [0, 1]}]}]
    cases = [
        ({**base, "symmetries": [{"destinations": [(i + 2) % L for i in range(L)], "sector": 0}]}, None,
         "^unsupported backend"),
        ({**base, "symmetries": [{"destinations": list(range(L)), "sector": 0,
                                  "local_permutations": [[1, 0]] * (L - 1) + [[0, 1]]}]}, None, "^unsupported backend"),
        ({**base, "up": 3, "symmetries": _quspin_maps(L, zblock=1)}, None, "^unsupported backend"),
        ({**base, "symmetries": [{"destinations": [(i + 1) % L for i in range(L)], "sector": 0,
                                  "local_permutations": [[1, 0]] * L}]}, None, "^unsupported backend"),
        ({**base, "symmetries": [{"destinations": [0] * L, "sector": 0}]}, None, "^incompatible symmetry request"),
        ({**base, "momentum": 0, "reverse": True}, None, "^unsupported backend"),
        ({**base, "momentum": 0, "symmetries": _quspin_maps(L, 0)}, None, "^invalid options"),
        (base, [0, 1, 2, 3, 4, 5, 6, 8], "^site 8 is outside a lattice with 8 sites"),
        (base, [0, 1, 2, 3, 4, 5, 6, 6], "^invalid options: site permutation must be bijective"),
    ]
    for basis, permutation, message in cases:
        request = {"operation": "create_model", "basis": basis, "terms": terms}
        if permutation is not None:
            request["site_permutation"] = permutation
        with pytest.raises(QmbedError, match=message):
            command(request)


def test_reversed_models_match_the_oracle_for_every_local_symbol():
    """C H C on the complemented sector: every local symbol, complex couplings and a site permutation.

    The couplings are translation invariant and symmetric under exchanging the
    two factors, so the operator commutes with the chain's lattice maps (for an
    operator that does not, the reduced matrix depends on how it is assembled).
    """
    from frontend_protocol import model_matrix
    from qmbed_b200._lib import command
    L = 10
    rng = np.random.default_rng(5)
    names = ["identity", "z", "raising", "lowering", "x", "y"]
    coefficients = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    coefficients = coefficients + coefficients.T
    terms = []
    for i_a, a in enumerate(names):
        for i_b, b in enumerate(names):
            c = coefficients[i_a, i_b]
            terms.append({"product": {"local": [a, b]},
                          "couplings": [{"coefficient": [c.real, c.imag], "sites": [i, (i + 3) % L]} for i in range(L)]})
    for up, maps in [(None, []), (None, _quspin_maps(L, 0, 1)), (None, _quspin_maps(L, 3))]:
        request = {"operation": "create_model",
                   "basis": {"kind": "spin", "sites": L, "up": up, "normalization": "pauli", "symmetries": maps,
                             "reverse": True},
                   "terms": terms, "site_permutation": list(range(L))[::-1],
                   "checks": {"hermiticity": False, "particle_conservation": False}}
        h = model_matrix(request)
        model = command(request)
        try:
            x = rng.standard_normal((2, h.shape[0])) + 1j * rng.standard_normal((2, h.shape[0]))
            got = command({"operation": "apply_model", "handle": model["handle"],
                           "vectors": [[[v.real, v.imag] for v in col] for col in x]})
            y = np.array([[complex(*v) for v in col] for col in got["vectors"]])
            assert np.abs(y - x @ h.T).max() <= 1e-12 * max(1.0, np.abs(h).max() * h.shape[0])
        finally:
            command({"operation": "release_model", "handle": model["handle"]})


@pytest.mark.parametrize("kblock,pblock,zblock", [(0, 1, 1), (0, 1, -1), (5, -1, 1), (3, None, -1), (None, None, 1)])
def test_spin_flip_sectors_match_the_oracle(kblock, pblock, zblock):
    """Operators that commute with the spin flip on zblock sectors (full space and up = L/2), reversed order."""
    from frontend_protocol import model_matrix
    from qmbed_b200._lib import command
    L = 10
    rng = np.random.default_rng(11)

    def term(local, coefficient, offset):
        return {"product": {"local": local},
                "couplings": [{"coefficient": [coefficient, 0.0], "sites": [(i + k) % L for k in offset]}
                              for i in range(L)]}

    flip_even = [
        (["x"], (0,)), (["x", "x"], (0, 1)), (["y", "y"], (0, 1)), (["z", "z"], (0, 2)),
        (["raising", "lowering"], (0, 1)),
    ]
    # y z is flip-even; with z y of the same coefficient it is also reflection-even
    c_yz = float(rng.standard_normal())
    for up in (None, 5):
        terms = [term(local, float(rng.standard_normal()), offset) for local, offset in flip_even]
        terms.append(dict(terms[-1], product={"local": ["lowering", "raising"]}))  # S+S- + S-S+, one coefficient
        terms += [term(["y", "z"], c_yz, (0, 3)), term(["z", "y"], c_yz, (0, 3))]
        if up is not None:
            terms = [t for t in terms if t["product"]["local"] not in (["x"],)]
            terms = [t for t in terms if "y" not in t["product"]["local"] and t["product"]["local"] != ["x", "x"]]
        request = {"operation": "create_model",
                   "basis": {"kind": "spin", "sites": L, "up": up, "normalization": "pauli",
                             "symmetries": _quspin_maps(L, kblock, pblock, zblock), "reverse": True},
                   "terms": terms, "site_permutation": list(range(L))[::-1],
                   "checks": {"hermiticity": True, "particle_conservation": up is not None}}
        h = model_matrix(request)
        model = command(request)
        try:
            assert model["dimension"] == h.shape[0]
            x = rng.standard_normal((2, h.shape[0])) + 1j * rng.standard_normal((2, h.shape[0]))
            got = command({"operation": "apply_model", "handle": model["handle"],
                           "vectors": [[[v.real, v.imag] for v in col] for col in x]})
            y = np.array([[complex(*v) for v in col] for col in got["vectors"]])
            assert np.abs(y - x @ h.T).max() <= 1e-12 * max(1.0, np.abs(h).max() * h.shape[0])
        finally:
            command({"operation": "release_model", "handle": model["handle"]})


def _matrix_request(a):
    rows, cols = np.nonzero(a)
    return {"shape": list(a.shape),
            "entries": [{"row": int(r), "column": int(c), "value": [a[r, c].real, a[r, c].imag]}
                        for r, c in zip(rows, cols)]}


@pytest.mark.parametrize("complex_matrix", [False, True])
def test_explicit_matrix_models_apply_solve_and_exponentiate(complex_matrix):
    """create_operator_model with a static matrix: CSR action, eigsh and the Taylor plan against dense numpy."""
    import scipy.linalg
    from qmbed_b200._lib import command
    rng = np.random.default_rng(3)
    n = 300
    a = np.where(rng.random((n, n)) < 0.02, rng.standard_normal((n, n)), 0.0).astype(complex)
    if complex_matrix:
        a += 1j * np.where(rng.random((n, n)) < 0.02, rng.standard_normal((n, n)), 0.0)
    a = a + a.conj().T + np.diag(rng.standard_normal(n))
    model = command({"operation": "create_operator_model", "static_operator": _matrix_request(a)})
    try:
        assert model["dimension"] == n
        x = rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))
        got = command({"operation": "apply_model", "handle": model["handle"],
                       "vectors": [[[v.real, v.imag] for v in col] for col in x]})
        y = np.array([[complex(*v) for v in col] for col in got["vectors"]])
        assert np.abs(y - x @ a.T).max() <= 1e-13 * np.abs(a).sum(axis=1).max()
        solved = command({"operation": "eigsh_model", "handle": model["handle"],
                          "solver": {"eigenpairs": 3, "target": {"kind": "smallest_algebraic"}, "tolerance": 1e-12}})
        np.testing.assert_allclose(solved["eigenvalues"], np.linalg.eigvalsh(a)[:3], atol=1e-9)
        plan = command({"operation": "create_expm_action", "handle": model["handle"], "coefficient": [0.0, -0.3]})
        out = command({"operation": "apply_expm_action", "expm_handle": plan["handle"],
                       "vectors": [[[v.real, v.imag] for v in x[0]]]})
        z = np.array([complex(*v) for v in out["vectors"][0]])
        assert np.linalg.norm(z - scipy.linalg.expm(-0.3j * a) @ x[0]) <= 1e-12 * np.linalg.norm(x[0])
        command({"operation": "release_expm_action", "expm_handle": plan["handle"]})
    finally:
        command({"operation": "release_model", "handle": model["handle"]})


def test_explicit_matrix_models_reject_bad_requests():
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    square = {"shape": [2, 2], "entries": [{"row": 0, "column": 1, "value": [1.0, 0.0]}]}
    cases = [
        ({"static_operator": {"shape": [2, 3], "entries": []}}, "^dimension mismatch"),
        ({"static_operator": {"shape": [2, 2], "entries": [{"row": 2, "column": 0, "value": [1.0, 0.0]}]}},
         "^dimension mismatch"),
        ({"static_operator": square, "components": [{"name": "g", "operator": square}]}, "^unsupported backend"),
        ({}, "^invalid options"),
    ]
    for request, message in cases:
        with pytest.raises(QmbedError, match=message):
            command({"operation": "create_operator_model", **request})


def test_operator_actions_match_the_oracle():
    """Normal, conjugate, adjoint and transpose actions (OperatorActionRequest, bindings/capi/src/lib.rs:937-945)
    of a non-Hermitian, translation-invariant model on a complex momentum sector: apply_model,
    evaluate_operator_expression and apply_operator_expression of model and transform expressions."""
    from frontend_protocol import OracleProtocol
    from qmbed_b200._lib import command
    L = 10
    bonds = [[i, (i + 1) % L] for i in range(L)]
    terms = [{"product": {"local": p}, "couplings": [{"coefficient": list(c), "sites": b} for b in bonds]}
             for p, c in ((["raising", "lowering"], (0.7, 0.2)), (["lowering", "raising"], (0.3, -0.5)),
                          (["z", "z"], (0.4, 0.1)))]
    terms.append({"product": {"local": ["z"]}, "couplings": [{"coefficient": [0.2, 0.3], "sites": [i]} for i in range(L)]})
    request = {"operation": "create_model", "basis": {"kind": "spin", "sites": L, "up": 4, "momentum": 3},
               "terms": terms, "checks": {"hermiticity": False, "particle_conservation": True}}
    oracle = OracleProtocol()
    o_handle = oracle.call("qmbed_command_json", request)["handle"]
    model = command(request)
    try:
        rng = np.random.default_rng(8)
        x = rng.standard_normal((2, model["dimension"])) + 1j * rng.standard_normal((2, model["dimension"]))
        vectors = [[[v.real, v.imag] for v in col] for col in x]
        for action in ("normal", "conjugate", "adjoint", "transpose"):
            for kind in ("model", "transform"):
                expression = ({"kind": "model", "handle": model["handle"], "action": action} if kind == "model" else
                              {"kind": "transform", "action": action,
                               "operand": {"kind": "scale", "coefficient": [0.3, 0.4],
                                           "operand": {"kind": "model", "handle": model["handle"]}}})
                o_expression = json.loads(json.dumps(expression).replace(f'"{model["handle"]}"', f'"{o_handle}"'))
                want = oracle.expression_matrix(o_expression)
                got = _dense(command({"operation": "evaluate_operator_expression", "expression": expression}))
                assert np.abs(got - want).max() <= 1e-13, (action, kind)
                applied = command({"operation": "apply_operator_expression", "expression": expression,
                                   "vectors": vectors})
                y = np.array([[complex(*v) for v in col] for col in applied["vectors"]])
                assert np.abs(y - x @ want.T).max() <= 1e-12, (action, kind)
            applied = command({"operation": "apply_model", "handle": model["handle"], "action": action,
                               "vectors": vectors})
            y = np.array([[complex(*v) for v in col] for col in applied["vectors"]])
            want = oracle.call("qmbed_command_json", {"operation": "apply_model", "handle": o_handle,
                                                      "action": action, "vectors": vectors})
            assert np.abs(y - np.array([[complex(*v) for v in col] for col in want["vectors"]])).max() <= 1e-12
    finally:
        command({"operation": "release_model", "handle": model["handle"]})


def test_spin_flip_sectors_split_the_spectrum_on_the_gpu():
    """eigh_model on QuSpin's zblock = +1 and -1 sectors (kblock=0, pblock=1, reversed order, 12 sites) gives
    together the spectrum of the sector without the spin flip."""
    from qmbed_b200._lib import command
    L = 12
    bonds = [[i, (i + 1) % L] for i in range(L)]
    terms = [{"product": {"local": p}, "couplings": [{"coefficient": [c, 0.0], "sites": b} for b in bonds]}
             for p, c in ((["z", "z"], 0.8), (["raising", "lowering"], 0.5), (["lowering", "raising"], 0.5))]
    spectra = {}
    for z in (None, 1, -1):
        request = {"operation": "create_model",
                   "basis": {"kind": "spin", "sites": L, "up": L // 2, "normalization": "angular_momentum",
                             "symmetries": _quspin_maps(L, 0, 1, z), "reverse": True},
                   "terms": terms, "site_permutation": list(range(L))[::-1]}
        model = command(request)
        try:
            spectra[z] = np.array(command({"operation": "eigh_model", "handle": model["handle"]})["eigenvalues"])
        finally:
            command({"operation": "release_model", "handle": model["handle"]})
    assert len(spectra[1]) > 0 and len(spectra[-1]) > 0
    np.testing.assert_allclose(np.sort(np.concatenate([spectra[1], spectra[-1]])), np.sort(spectra[None]), atol=1e-11)
