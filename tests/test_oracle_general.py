"""The oracle's lattice-map bases and site conventions (no GPU).

``oracle/general.py`` restates the reference's runtime-symmetry spin basis
(GeneralBasis with orbit seeds, src/basis/mod.rs:4163-4306) and
``reverse`` ordering (bindings/capi/src/lib.rs:3412-3423). It is pinned here
by the reference's own known answer (a general translation map equals the
built-in momentum sector, tests/runtime_symmetry.rs:9-38) and by the C++
oracle's built-in sectors, which the reference's anchors pin in
tests/test_oracle_anchors.py. The last tests check the identity the GPU engine
builds reversed bases on: the reversed, maximum-representative sector is the
bitwise complement of the ordinary sector with up' = L - up, and its reduced
operator is that of C H C with C the global spin flip.
"""

import json
from pathlib import Path

import numpy as np
import pytest

L10 = 10


def _translation(sites, step):
    return [(i + step) % sites for i in range(sites)]


def _reflection(sites):
    return [sites - 1 - i for i in range(sites)]


def test_runtime_translation_matches_the_builtin_sector(oracle):
    """tests/runtime_symmetry.rs:9-38: L=6, up=3, map i -> i+1 with sector 1 lists the momentum-1 states."""
    from oracle import general
    g = general.GeneralSpinBasis(6, 3, [{"destinations": _translation(6, 1), "sector": 1}])
    states, _ = oracle.Basis(6, up=3, momentum=1).states()
    assert g.states.tolist() == states.tolist()


@pytest.mark.parametrize("k", range(L10))
def test_translation_maps_reproduce_builtin_momentum_operators(oracle, k):
    """Both translation directions: i -> i+1 with sector k and i -> i-1 with sector -k are momentum k."""
    from oracle import general
    terms = oracle.heisenberg_terms(L10, delta=0.7)
    builtin = oracle.Operator.build(oracle.Basis(L10, up=5, momentum=k), terms).dense()
    for step, sector in ((1, k), (-1, -k)):
        g = general.GeneralSpinBasis(L10, 5, [{"destinations": _translation(L10, step), "sector": sector}])
        assert np.abs(general.reduced_dense(g, terms) - builtin).max() <= 1e-13


@pytest.mark.parametrize("k,p", [(0, 1), (0, -1), (5, 1), (5, -1)])
def test_translation_and_reflection_maps_reproduce_builtin_parity(oracle, k, p):
    from oracle import general
    terms = oracle.heisenberg_terms(L10, delta=1.2)
    maps = [{"destinations": _translation(L10, -1), "sector": k},
            {"destinations": _reflection(L10), "sector": 0 if p == 1 else 1}]
    g = general.GeneralSpinBasis(L10, 5, maps)
    builtin = oracle.Operator.build(oracle.Basis(L10, up=5, momentum=k, parity=p), terms).dense()
    assert np.abs(general.reduced_dense(g, terms) - builtin).max() <= 1e-13


FLIP = {"I": ("I", 1.0), "z": ("z", -1.0), "+": ("-", 1.0), "-": ("+", 1.0), "x": ("x", 1.0), "y": ("y", -1.0)}


def _flip(terms):
    out = []
    for symbols, couplings in terms:
        sign = np.prod([FLIP[c][1] for c in symbols])
        out.append(("".join(FLIP[c][0] for c in symbols), [(sign * c, s) for c, s in couplings]))
    return out


@pytest.mark.parametrize("up,maps,k,p", [
    (4, [], None, None),
    (None, [], None, None),
    (4, [{"destinations": _translation(L10, -1), "sector": 3}], 7, None),
    (5, [{"destinations": _translation(L10, -1), "sector": 0}, {"destinations": _reflection(L10), "sector": 1}], 0, -1),
])
def test_reversed_sectors_are_complemented_ordinary_sectors(oracle, up, maps, k, p):
    from oracle import general
    rng = np.random.default_rng(3)
    symbols = ["I", "z", "+", "-", "x", "y"]
    terms = [(a + b, [(complex(*rng.standard_normal(2)), (i, (i + 2) % L10)) for i in range(L10)])
             for a in symbols for b in symbols]
    permutation = list(range(L10))[::-1]
    reversed_basis = general.GeneralSpinBasis(L10, up, maps, reverse=True)
    ordinary = oracle.Basis(L10, up=None if up is None else L10 - up, momentum=k, parity=p)
    states, _ = ordinary.states()
    mask = (1 << L10) - 1
    assert reversed_basis.states.tolist() == [(~int(s)) & mask for s in states]
    expected = oracle.Operator.build(ordinary, _flip(general.permute_terms(terms, permutation)),
                                     check_hermitian=False, check_particles=False).dense()
    got = general.reduced_dense(reversed_basis, terms, site_permutation=permutation)
    assert np.abs(got - expected).max() <= 1e-13


def test_recorded_frontend_requests_are_answered_by_the_oracle():
    """The fixture of frontend requests is complete: every request has an oracle answer, handles come first."""
    import frontend_protocol
    scenarios = json.loads((Path(__file__).resolve().parent / "golden" / "frontend_requests.json").read_text())
    assert len(scenarios) >= 5
    operations = set()
    for name, scenario in scenarios.items():
        proto = frontend_protocol.OracleProtocol()
        for call in scenario["calls"]:
            proto.call(call["symbol"], call["request"])
            operations.add(call["request"].get("operation", "run"))
    assert {"run", "create_model", "eigsh_model", "apply_model", "measure_model", "matrix_elements_model",
            "eigh_model", "evolve_model", "release_model"} <= operations


def test_reference_frontend_binds_every_symbol_of_the_library():
    """The reference's own ctypes loader (bindings/python/src/qmbed/_ffi.py:154-186) binds all six JSON
    symbols of libqmbed_b200.so; skipped when the frontend is not installed in baseline/_ref."""
    import ctypes
    import importlib.util
    root = Path(__file__).resolve().parents[1]
    ffi_path = root / "baseline" / "_ref" / "qmbed" / "_ffi.py"
    library = root / "qmbed_b200" / "libqmbed_b200.so"
    if not ffi_path.is_file() or not library.is_file():
        pytest.skip("reference frontend or library not present")
    spec = importlib.util.spec_from_file_location("reference_qmbed_ffi", ffi_path)
    ffi = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ffi)
    lib = ffi._load_library(str(library))
    for symbol in ("qmbed_run_json", "qmbed_command_json", "qmbed_string_free", "qmbed_evolve_model_with_drive_json",
                   "qmbed_register_user_basis_32_json", "qmbed_register_user_basis_64_json"):
        assert isinstance(getattr(lib, symbol), ctypes._CFuncPtr)


@pytest.mark.parametrize("k,p", [(0, 1), (0, -1), (5, None), (3, None)])
def test_spin_flip_sectors_split_the_spectrum(oracle, k, p):
    """The global spin flip (identity destinations, local maps [1, 0]) splits a sector at up = L/2 into
    z = +1 and z = -1 blocks whose spectra together are the sector's, like the reference's parity
    anchors (tests/full_api_foundation.rs:159-198)."""
    from oracle import general
    terms = oracle.heisenberg_terms(L10, delta=0.8)
    maps = [{"destinations": _translation(L10, -1), "sector": k}]
    if p is not None:
        maps.append({"destinations": _reflection(L10), "sector": 0 if p == 1 else 1})
    whole = np.linalg.eigvalsh(general.reduced_dense(general.GeneralSpinBasis(L10, 5, maps), terms))
    flip = {"destinations": list(range(L10)), "local_permutations": [[1, 0]] * L10}
    parts = []
    for z in (0, 1):
        b = general.GeneralSpinBasis(L10, 5, maps + [{**flip, "sector": z}], reverse=True)
        parts.append(np.linalg.eigvalsh(general.reduced_dense(b, terms)))
    assert len(parts[0]) + len(parts[1]) == len(whole) and min(len(parts[0]), len(parts[1])) > 0
    np.testing.assert_allclose(np.sort(np.concatenate(parts)), whole, atol=1e-12)
