"""Warp-tile matrix-free H.v against the CPU oracle, one lookup at a time.

The on-the-fly action resolves each target state through the sector's image
table, through the representative search, or (legacy) through the
one-thread-per-row expansion. Every lookup must reproduce the oracle's action
(FP64 relative 2-norm error <= 1e-13, FP32 <= 5e-6), and the image table must
give the same (row, character, orbit size) as the canonical search, bit for
bit in rows and orbit sizes.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _models(sites):
    from oracle import oracle
    from qmbed_b200.engine import heisenberg_terms
    rng = np.random.default_rng(7)
    fields = rng.uniform(-2, 2, size=sites)
    bonds = [(i, (i + 1) % sites) for i in range(sites)]
    return {
        "heisenberg": oracle.heisenberg_terms(sites),
        "xxz": oracle.heisenberg_terms(sites, delta=0.73),
        "j1j2": heisenberg_terms(sites, j2=0.37, delta=0.9),
        "xy_y": [("xx", [(0.4, b) for b in bonds]), ("yy", [(0.4, b) for b in bonds]),
                 ("zz", [(1.1, b) for b in bonds])],
        # Dzyaloshinskii-Moriya exchange: complex hopping amplitudes
        "dm": [("+-", [(0.5 + 0.3j, b) for b in bonds]), ("-+", [(0.5 - 0.3j, b) for b in bonds]),
               ("zz", [(0.8, b) for b in bonds])],
        "tfim_fields": [("zz", [(-1.0, (i, i + 1)) for i in range(sites - 1)]),
                        ("x", [(-1.0, (i,)) for i in range(sites)]),
                        ("z", [(float(h), (i,)) for i, h in enumerate(fields)])],
        # translation- and reflection-invariant: serves the symmetric sectors
        "tfim_uniform": [("zz", [(-1.0, b) for b in bonds]), ("x", [(-0.9, (i,)) for i in range(sites)]),
                         ("z", [(0.3, (i,)) for i in range(sites)])],
    }


# (model, sites, up, momentum, parity, normalization)
CASES = [
    ("heisenberg", 16, 8, 0, 1, "angular_momentum"),
    ("heisenberg", 16, 8, 3, None, "angular_momentum"),
    ("heisenberg", 14, 7, 7, -1, "angular_momentum"),
    ("xxz", 18, 9, 0, None, "angular_momentum"),
    ("j1j2", 16, 8, 5, None, "angular_momentum"),
    ("j1j2", 14, 7, 0, -1, "angular_momentum"),
    ("xy_y", 12, 6, 2, None, "angular_momentum"),
    ("xy_y", 12, 6, 0, 1, "pauli"),
    ("dm", 12, 6, 4, None, "angular_momentum"),
    ("tfim_fields", 12, None, None, None, "pauli_cartesian"),
    ("tfim_uniform", 12, None, 0, None, "pauli_cartesian"),
    ("tfim_uniform", 12, None, 6, 1, "pauli_cartesian"),
    ("heisenberg", 12, 6, None, None, "angular_momentum"),
    ("heisenberg", 12, None, 0, 1, "pauli"),
    ("heisenberg", 13, None, None, -1, "angular_momentum"),
]


def _pair(engine, oracle, model, sites, up, momentum, parity, norm):
    terms = _models(sites)[model]
    checks = dict(check_particles=not model.startswith("tfim"))
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity, normalization=norm),
                              terms, **checks)
    gb = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity, normalization=norm)
    g = engine.GpuOperator(gb, terms, storage="matrix_free", **checks)
    return o, g


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _lookups(case):
    symmetric = case[3] is not None or case[4] is not None
    return ["table", "table_generic", "search", "legacy"] if symmetric else ["auto", "legacy"]


def _expected_in_use(lookup, info):
    """The lookup that lookup_info reports for a requested one: "table" runs the
    nearest-neighbour hop kernel where it applies."""
    if lookup == "table":
        return info["lookup"] in ("table", "table_hop")
    if lookup == "table_generic":
        return info["lookup"] == "table"
    return info["lookup"] == lookup


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(map(str, c)))
def test_tile_hv_fp64_matches_oracle(engine, oracle, case):
    o, g = _pair(engine, oracle, *case)
    n = o.dim
    rng = np.random.default_rng(3)
    xc = rng.normal(size=n) + 1j * rng.normal(size=n)
    xr = rng.normal(size=n)
    expected_c = o.apply(xc)
    expected_r = o.apply(xr).real if o.is_real else None
    for lookup in _lookups(case):
        g.set_lookup(lookup)
        info = g.lookup_info()
        if lookup in ("table", "table_generic", "search", "legacy"):
            assert _expected_in_use(lookup, info), (lookup, info)
        got = g.apply(xc)
        assert np.linalg.norm(got - expected_c) <= 1e-13 * max(np.linalg.norm(expected_c), 1.0), lookup
        if expected_r is not None:
            assert g.is_real
            got_r = g.apply(xr)
            assert np.linalg.norm(got_r - expected_r) <= 1e-13 * max(np.linalg.norm(expected_r), 1.0), lookup


@pytest.mark.parametrize("case", [c for c in CASES if c[0] in ("heisenberg", "j1j2", "dm", "tfim_uniform")],
                         ids=lambda c: "-".join(map(str, c)))
def test_tile_hv_fp32_matches_oracle(engine, oracle, case):
    import torch
    o, g = _pair(engine, oracle, *case)
    n = o.dim
    rng = np.random.default_rng(5)
    cplx = not o.is_real
    x = rng.normal(size=n) + (1j * rng.normal(size=n) if cplx else 0)
    expected = o.apply(x) if cplx else o.apply(x).real
    xin = np.ascontiguousarray(np.stack([x.real, x.imag], -1).reshape(-1)) if cplx else x
    for lookup in _lookups(case):
        g.set_lookup(lookup)
        xd = torch.tensor(xin, dtype=torch.float32, device="cuda")
        yd = torch.full_like(xd, float("nan"))
        g.apply_device(xd, yd, precision=32, complex_vectors=cplx)
        torch.cuda.synchronize()
        y = yd.double().cpu().numpy()
        got = y.reshape(-1, 2) @ np.array([1, 1j]) if cplx else y
        assert np.linalg.norm(got - expected) <= 5e-6 * max(np.linalg.norm(expected), 1.0), lookup


@pytest.mark.parametrize("sites,momentum,parity", [(18, 0, 1), (16, 8, -1), (14, None, 1), (16, 0, None)])
@pytest.mark.parametrize("precision,nb", [(64, 8), (64, 16), (32, 8), (32, 16)])
def test_tile_block_action_matches_packed(engine, sites, momentum, parity, precision, nb):
    import torch
    from qmbed_b200.engine import heisenberg_terms
    terms = heisenberg_terms(sites, j2=0.21, delta=1.1)
    basis = engine.GpuBasis(sites, up=sites // 2, momentum=momentum, parity=parity)
    packed = engine.GpuOperator(basis, terms, storage="packed")
    free = engine.GpuOperator(basis, terms, storage="matrix_free")
    n = packed.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(sites + nb)
    z = torch.randn(n, nb, dtype=dtype, device="cuda", generator=gen)
    p = torch.randn(n, nb, dtype=dtype, device="cuda", generator=gen)
    ref = torch.empty_like(z)
    packed.apply_block_device(z, ref, nb, precision=precision, alpha=0.7, beta=-0.2, gamma=0.4, p=p)
    tol = 1e-13 if precision == 64 else 2e-5
    for lookup in ("table", "table_generic", "search", "legacy"):
        free.set_lookup(lookup)
        out = torch.full_like(z, float("nan"))
        free.apply_block_device(z, out, nb, precision=precision, alpha=0.7, beta=-0.2, gamma=0.4, p=p)
        torch.cuda.synchronize()
        err = float(torch.linalg.vector_norm((out - ref).double()))
        assert err <= tol * float(torch.linalg.vector_norm(ref.double())), (lookup, err)


@pytest.mark.parametrize("sites,up,momentum,parity", [(16, 8, 0, 1), (16, 8, 3, None), (18, 9, 9, -1),
                                                       (14, None, 0, 1), (15, 7, None, 1), (12, None, 5, None)])
def test_table_images_equal_canonical_images(engine, sites, up, momentum, parity):
    basis = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity)
    rng = np.random.default_rng(sites * 7 + (momentum or 0))
    states = rng.integers(0, 1 << sites, size=20000, dtype=np.uint64)
    if up is not None:
        # half of the sample in the fixed-weight space
        states = np.array([s for s in states.tolist() if bin(s).count("1") == up] + states[:5000].tolist(),
                          np.uint64)
    index, phase, orbit = basis.images(states)
    tindex, tphase, torbit = basis.table_images(states)
    assert np.array_equal(index, tindex)
    assert np.array_equal(orbit, torbit)
    assert np.max(np.abs(phase - tphase)) <= 4e-15


def test_repeated_site_products_take_the_legacy_expansion(engine, oracle):
    sites = 12
    terms = oracle.heisenberg_terms(sites) + [("+-", [(0.3, (i, i)) for i in range(sites)])]
    o = oracle.Operator.build(oracle.Basis(sites, up=6, momentum=0, parity=1), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=6, momentum=0, parity=1), terms, storage="matrix_free")
    assert g.lookup_info()["lookup"] == "legacy"
    x = np.random.default_rng(1).normal(size=o.dim)
    expected = o.apply(x).real
    assert np.linalg.norm(g.apply(x) - expected) <= 1e-13 * np.linalg.norm(expected)


@pytest.mark.parametrize("model,chain", [("heisenberg", True), ("j1j2", True), ("xy_y", True), ("dm", True),
                                         ("tfim_uniform", False), ("tfim_fields", False)])
def test_chain_form_detection(engine, model, chain):
    """Uniform bond models take the translation-structured expansion; single-site
    flips and non-uniform couplings keep the per-group expansion."""
    sites = 12
    up = None if model.startswith("tfim") else 6
    norm = "pauli_cartesian" if model.startswith("tfim") else "angular_momentum"
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, normalization=norm), _models(sites)[model],
                           storage="matrix_free", check_particles=not model.startswith("tfim"))
    assert g.lookup_info()["chain_form"] is chain


def test_open_chain_with_uniform_fields_matches_oracle(engine, oracle):
    """Open boundary (a partial bond mask) and a uniform longitudinal field in the chain form."""
    sites = 14
    bonds = [(i, i + 1) for i in range(sites - 1)]
    terms = [("zz", [(0.9, b) for b in bonds]), ("+-", [(0.5, b) for b in bonds]), ("-+", [(0.5, b) for b in bonds]),
             ("z", [(0.37, (i,)) for i in range(sites)])]
    o = oracle.Operator.build(oracle.Basis(sites, up=7), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=7), terms, storage="matrix_free")
    assert g.lookup_info()["chain_form"]
    x = np.random.default_rng(2).normal(size=o.dim)
    expected = o.apply(x).real
    assert np.linalg.norm(g.apply(x) - expected) <= 1e-13 * np.linalg.norm(expected)


def test_matrix_free_defaults_to_the_image_table(engine):
    from qmbed_b200.engine import heisenberg_terms
    g = engine.GpuOperator(engine.GpuBasis(20, up=10, momentum=0, parity=1), heisenberg_terms(20),
                           storage="matrix_free")
    info = g.lookup_info()
    assert info["lookup"] == "table_hop"
    assert info["table_bytes"] == 184756 * 4  # C(20, 10) u32 entries


def test_tile_lookups_agree_at_26_sites(engine):
    """Size-independent cross-check at a scan size: every lookup, and the packed rows."""
    import torch
    from qmbed_b200.engine import heisenberg_terms
    terms = heisenberg_terms(26, j2=0.3, delta=0.95)
    for momentum in (0, 5):
        basis = engine.GpuBasis(26, up=13, momentum=momentum)
        packed = engine.GpuOperator(basis, terms, storage="packed")
        free = engine.GpuOperator(basis, terms, storage="matrix_free")
        n = packed.dim
        width = n if momentum == 0 else 2 * n
        cplx = momentum != 0
        x = torch.randn(width, dtype=torch.float64, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(momentum))
        ref = torch.empty_like(x)
        packed.apply_device(x, ref, precision=64, complex_vectors=cplx)
        for lookup in ("table", "table_generic", "search", "legacy"):
            free.set_lookup(lookup)
            y = torch.full_like(x, float("nan"))
            free.apply_device(x, y, precision=64, complex_vectors=cplx)
            torch.cuda.synchronize()
            assert float(torch.linalg.vector_norm(y - ref)) <= 1e-13 * float(torch.linalg.vector_norm(ref)), lookup


# (sites, up, momentum, parity, delta, periodic): real sectors of nearest-neighbour chains
HOP_CASES = [(16, 8, 0, 1, 1.0, True), (18, 9, 9, -1, 0.73, True), (17, 8, 0, None, 1.2, True),
             (16, 7, 8, 1, 0.5, True), (14, 7, None, 1, 0.9, False), (15, 7, None, -1, 1.0, False),
             (20, 10, 0, -1, 1.35, True)]


def _hop_terms(sites, delta, periodic):
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]
    return [("zz", [(delta, b) for b in bonds]), ("+-", [(0.5, b) for b in bonds]), ("-+", [(0.5, b) for b in bonds])]


@pytest.mark.parametrize("case", HOP_CASES, ids=lambda c: "-".join(map(str, c)))
def test_hop_kernel_matches_oracle(engine, oracle, case):
    """The nearest-neighbour hop kernel (rank steps by one binomial, the wrapping
    bond from the chunk tables) against the oracle: FP64 1e-13, FP32 5e-6."""
    import torch
    sites, up, momentum, parity, delta, periodic = case
    terms = _hop_terms(sites, delta, periodic)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms,
                           storage="matrix_free")
    assert g.lookup_info()["lookup"] == "table_hop"
    x = np.random.default_rng(sites).normal(size=o.dim)
    expected = o.apply(x).real
    assert np.linalg.norm(g.apply(x) - expected) <= 1e-13 * np.linalg.norm(expected)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.full_like(xd, float("nan"))
    g.apply_device(xd, yd, precision=32)
    torch.cuda.synchronize()
    assert np.linalg.norm(yd.double().cpu().numpy() - expected) <= 5e-6 * np.linalg.norm(expected)


@pytest.mark.parametrize("case", HOP_CASES[:4], ids=lambda c: "-".join(map(str, c)))
@pytest.mark.parametrize("precision,nb", [(64, 8), (64, 16), (32, 8), (32, 16)])
def test_hop_block_action_matches_generic_tile(engine, case, precision, nb):
    """Block action of the hop kernel against the general tile kernel on the same table."""
    import torch
    sites, up, momentum, parity, delta, periodic = case
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity),
                           _hop_terms(sites, delta, periodic), storage="matrix_free")
    n = g.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(nb + sites)
    z = torch.randn(n, nb, dtype=dtype, device="cuda", generator=gen)
    p = torch.randn(n, nb, dtype=dtype, device="cuda", generator=gen)
    g.set_lookup("table_generic")
    ref = torch.full_like(z, float("nan"))
    g.apply_block_device(z, ref, nb, precision=precision, alpha=0.6, beta=0.3, gamma=-0.5, p=p)
    g.set_lookup("table")
    out = torch.full_like(z, float("nan"))
    g.apply_block_device(z, out, nb, precision=precision, alpha=0.6, beta=0.3, gamma=-0.5, p=p)
    torch.cuda.synchronize()
    tol = 1e-13 if precision == 64 else 2e-6
    err = float(torch.linalg.vector_norm((out - ref).double()))
    assert err <= tol * float(torch.linalg.vector_norm(ref.double())), err


def test_hop_kernel_agrees_with_packed_rows_at_28_sites(engine):
    """Size-independent check at the XXZ benchmark size: hop kernel against the
    packed rows in FP64 (L=28, k=0, p=+1, D = 718,146)."""
    import torch
    terms = _hop_terms(28, 1.35, True)
    basis = engine.GpuBasis(28, up=14, momentum=0, parity=1)
    packed = engine.GpuOperator(basis, terms, storage="packed")
    free = engine.GpuOperator(basis, terms, storage="matrix_free")
    assert free.lookup_info()["lookup"] == "table_hop"
    x = torch.randn(packed.dim, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    ref, y = torch.empty_like(x), torch.full_like(x, float("nan"))
    packed.apply_device(x, ref, precision=64)
    free.apply_device(x, y, precision=64)
    torch.cuda.synchronize()
    assert float(torch.linalg.vector_norm(y - ref)) <= 1e-13 * float(torch.linalg.vector_norm(ref))


@pytest.mark.parametrize("sites,up,momentum,parity", [(16, 1, 0, 1), (16, 15, 0, None), (18, 2, 9, -1),
                                                       (5, 2, 0, 1), (6, 3, 3, None), (22, 11, 0, 1)])
def test_hop_kernel_extreme_fillings_match_oracle(engine, oracle, sites, up, momentum, parity):
    """One or two up spins (few hops), one down spin, the smallest chains, and a
    half-filled 22-site sector, through the hop kernel against the oracle."""
    terms = _hop_terms(sites, 0.8, True)
    o = oracle.Operator.build(oracle.Basis(sites, up=up, momentum=momentum, parity=parity), terms)
    g = engine.GpuOperator(engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity), terms,
                           storage="matrix_free")
    assert g.lookup_info()["lookup"] == "table_hop"
    x = np.random.default_rng(up).normal(size=o.dim)
    expected = o.apply(x).real
    assert np.linalg.norm(g.apply(x) - expected) <= 1e-13 * max(np.linalg.norm(expected), 1e-300)
