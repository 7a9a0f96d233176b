"""Record the JSON requests the reference's unmodified Python frontend sends.

The reference's Python packages (``qmbed`` and its QuSpin-compatible
``quspin``) are pure Python over ``qmbed._ffi._call_json``
(bindings/python/src/qmbed/_ffi.py:189-207). This script imports them from a
reference checkout, replaces that one function by a recorder whose answers
come from the oracle (``tests/frontend_protocol.py``), runs a few ordinary user
scripts, and writes every request, in order, to
``tests/golden/frontend_requests.json``. ``tests/test_gpu_frontend_requests.py``
replays the file through ``libqmbed_b200.so`` and checks each answer against
the oracle, so the GPU tests need neither the reference nor its frontend.

    python tests/golden/make_frontend_requests.py <reference checkout>

The checkout may instead be given as ``$QMBED_REFERENCE``; one of the two is
required.
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from frontend_protocol import OracleProtocol  # noqa: E402

OUT = Path(__file__).resolve().parent / "frontend_requests.json"


def reference_frontend(checkout: Path):
    sys.path.insert(0, str(checkout / "bindings" / "python" / "src"))
    import qmbed
    import qmbed._ffi as ffi
    return qmbed, ffi


class Recorder:
    def __init__(self):
        self.protocol = OracleProtocol()
        self.calls = []

    def __call__(self, symbol, request, *, library_path=None):
        request = json.loads(json.dumps(request))  # the bytes the library would receive
        self.calls.append({"symbol": symbol, "request": request})
        return self.protocol.call(symbol, request)


def heisenberg_static(sites, delta):
    bonds = [[1.0, i, (i + 1) % sites] for i in range(sites)]
    return [["xx", bonds], ["yy", bonds], ["zz", [[delta, i, j] for _, i, j in bonds]]]


def scenarios(qmbed):
    from quspin.basis import spin_basis_1d
    from quspin.operators import hamiltonian

    rng = np.random.default_rng(20261204)

    def native_eigsh():
        """qmbed.eigsh on a built-in momentum/parity sector (model.py:311-358)."""
        L = 12
        bonds = [(i, (i + 1) % L) for i in range(L)]
        terms = [
            qmbed.OperatorSpec(qmbed.OpProduct(("z", "z")), tuple(qmbed.Coupling(0.9, b) for b in bonds)),
            qmbed.OperatorSpec(qmbed.OpProduct(("raising", "lowering")), tuple(qmbed.Coupling(0.5, b) for b in bonds)),
            qmbed.OperatorSpec(qmbed.OpProduct(("lowering", "raising")), tuple(qmbed.Coupling(0.5, b) for b in bonds)),
        ]
        basis = qmbed.SpinBasis(L, up=6, momentum=0, parity=1)
        qmbed.eigsh(basis, terms, qmbed.EigshOptions(3, tolerance=1e-12, seed=4, eigenvectors=True))

    def quspin_real_sector():
        """hamiltonian on spin_basis_1d(L, Nup, kblock=0, pblock=1): QuSpin's lattice maps, reversed order."""
        L = 12
        basis = spin_basis_1d(L, Nup=L // 2, kblock=0, pblock=1, pauli=False)
        H = hamiltonian(heisenberg_static(L, 1.3), [], basis=basis, dtype=np.float64)
        H.eigsh(k=4, which="SA")
        H.eigsh(k=2, which="LA", return_eigenvectors=False)
        v = rng.standard_normal(H.Ns)
        w = rng.standard_normal(H.Ns)
        H.dot(v)
        H.expt_value(v / np.linalg.norm(v))
        H.quant_fluct(v / np.linalg.norm(v))
        H.matrix_ele(v.astype(complex), w.astype(complex))
        H.eigvalsh()

    def quspin_complex_sector():
        """kblock=1 on 12 sites: a complex momentum sector through the reversed translation map."""
        L = 12
        basis = spin_basis_1d(L, Nup=5, kblock=1, pauli=False)
        H = hamiltonian(heisenberg_static(L, 0.8), [], basis=basis, dtype=np.complex128)
        H.eigsh(k=3, which="SA")
        z = rng.standard_normal(H.Ns) + 1j * rng.standard_normal(H.Ns)
        H.dot(z)
        H.expt_value(z / np.linalg.norm(z))

    def quspin_transverse_field():
        """A transverse-field Ising chain on the full space in Pauli normalisation, with the Krylov evolve."""
        L = 10
        fields = rng.uniform(-1.0, 1.0, L)
        static = [["zz", [[-1.0, i, i + 1] for i in range(L - 1)]],
                  ["x", [[-0.9, i] for i in range(L)]],
                  ["z", [[float(h), i] for i, h in enumerate(fields)]]]
        basis = spin_basis_1d(L)
        H = hamiltonian(static, [], basis=basis, dtype=np.float64)
        H.eigsh(k=2, which="SA")
        psi = np.zeros(H.Ns, dtype=np.complex128)
        psi[0] = 1.0
        H.dot(psi)
        H.evolve(psi, 0.0, [0.5, 1.0], solver_name="qmbed")

    def quspin_density_matrix():
        """Expectation and fluctuation of a density matrix on a small reflection-even sector."""
        L = 6
        basis = spin_basis_1d(L, Nup=3, pblock=1, pauli=False)
        H = hamiltonian(heisenberg_static(L, 0.6), [], basis=basis, dtype=np.float64)
        a = rng.standard_normal((H.Ns, H.Ns)) + 1j * rng.standard_normal((H.Ns, H.Ns))
        rho = a @ a.conj().T
        rho /= np.trace(rho)
        H.expt_value(rho)
        H.quant_fluct(rho)

    def quspin_lanczos_tools():
        """QuSpin's Lanczos tools on -H in a kblock=0, pblock=1, zblock=1 sector (the compat test_Lanczos flow)."""
        from quspin.tools.lanczos import expm_lanczos, lanczos_full, lanczos_iter, lin_comb_Q_T
        L = 16
        basis = spin_basis_1d(L, m=0, kblock=0, pblock=1, zblock=1)
        J = [[1.0, i, (i + 1) % L] for i in range(L)]
        H = -hamiltonian([[op, J] for op in ["xx", "yy", "zz"]], [], basis=basis, dtype=np.float64)
        v0 = rng.normal(0, 1, size=basis.Ns)
        v0 /= np.linalg.norm(v0)
        E1, V1, lv1 = lanczos_full(H, v0, 20)
        E2, V2, lv2 = lanczos_iter(H, v0, 20)
        expm_lanczos(E1, V1, lv1, a=-0.1j)
        expm_lanczos(E2, V2, lv2, a=-0.1j)
        H.eigsh(k=1, which="LA")
        E, V, Q = lanczos_full(H, v0, 30, full_ortho=False)
        lin_comb_Q_T(V[:, -1], Q)
        H.static

    def quspin_expm_multiply_parallel():
        """expm_multiply_parallel on -(H - E) of a zblock sector (the compat test_imag_time flow) and on a
        random complex sparse matrix: explicit-matrix operator models and their exponential-action plans."""
        import scipy.sparse as sp
        from quspin.tools.evolution import expm_multiply_parallel
        L = 12
        basis = spin_basis_1d(L, m=0, kblock=0, pblock=1, zblock=1)
        J = [[1.0, i, (i + 1) % L] for i in range(L)]
        H = hamiltonian([["xx", J], ["yy", J], ["zz", J]], [], basis=basis, dtype=np.float64)
        (E,), _ = H.eigsh(k=1, which="SA")
        A = -(H.tocsr() - E * sp.eye(H.Ns, format="csr", dtype=np.float64))
        U = expm_multiply_parallel(A)
        v = rng.uniform(-1, 1, size=H.Ns)
        v /= np.linalg.norm(v)
        for _ in range(3):
            v = U.dot(v)
            v /= np.linalg.norm(v)
        n = 120
        B = (sp.random(n, n, density=np.log(n) / n, random_state=1)
             + 1j * sp.random(n, n, density=np.log(n) / n, random_state=2)).tocsr()
        w = rng.normal(0, 1, size=n) + 1j * rng.normal(0, 1, size=n)
        w /= np.linalg.norm(w)
        expm_multiply_parallel(B).dot(w)
        expm_multiply_parallel(B, a=-0.01j, dtype=np.complex128).dot(w)

    def quspin_driven_hamiltonian():
        """A driven chain: the dynamic term becomes a named component; dot, eigsh and the matrix at given times."""
        L = 10
        basis = spin_basis_1d(L, Nup=5, kblock=0, pblock=1, pauli=False)

        def drive(t, omega):
            return np.cos(omega * t)

        dynamic = [["zz", [[0.4, i, (i + 2) % L] for i in range(L)], drive, [2.0]]]
        H = hamiltonian(heisenberg_static(L, 1.0), dynamic, basis=basis, dtype=np.float64)
        H.dot(rng.standard_normal(H.Ns), time=0.3)
        H.eigsh(k=2, which="SA", time=0.7)
        H.tocsr(time=1.1)

    def quspin_fixed_magnetisation():
        """spin_basis_1d(L, Nup) without lattice maps: reversed order and site permutation only."""
        L = 10
        basis = spin_basis_1d(L, Nup=3, pauli=False)
        static = heisenberg_static(L, 1.0)[:2] + [["z", [[0.3 * i, i] for i in range(L)]]]
        H = hamiltonian(static, [], basis=basis, dtype=np.float64)
        H.eigsh(k=2, which="SA")
        H.dot(rng.standard_normal(H.Ns))

    return {f.__name__: f for f in (native_eigsh, quspin_real_sector, quspin_complex_sector,
                                     quspin_transverse_field, quspin_density_matrix, quspin_lanczos_tools,
                                     quspin_expm_multiply_parallel, quspin_driven_hamiltonian,
                                     quspin_fixed_magnetisation)}


def main() -> None:
    location = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QMBED_REFERENCE")
    if not location:
        sys.exit("usage: make_frontend_requests.py <reference checkout>  (or set QMBED_REFERENCE)")
    checkout = Path(location)
    qmbed, ffi = reference_frontend(checkout)
    out = {}
    for name, scenario in scenarios(qmbed).items():
        recorder = Recorder()
        ffi._call_json = recorder
        ffi._library_path = lambda: Path("/nonexistent/libqmbed_capi.so")
        scenario()
        out[name] = {"doc": scenario.__doc__, "calls": recorder.calls}
    OUT.write_text(json.dumps(out, separators=(",", ":")) + "\n")
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {sum(len(v['calls']) for v in out.values())} requests)")


if __name__ == "__main__":
    main()
