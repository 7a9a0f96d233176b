"""ctypes binding of the CPU oracle (test infrastructure only).

Only the tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` import this module. It loads ``oracle/libqmbed_oracle.so`` (built
by ``oracle/Makefile``) and exposes the reference algorithms restated in
``oracle/qmbed_oracle.cpp``: spin-sector enumeration, column-streaming
assembly, COO/CSR apply, restarted Lanczos ``eigsh`` and the Taylor
exponential-action plan.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libqmbed_oracle.so"

TARGETS = {
    "smallest_algebraic": 0,
    "largest_algebraic": 1,
    "smallest_magnitude": 2,
    "largest_magnitude": 3,
    "both_ends": 4,
    "shift": 5,
}

NORMALIZATIONS = {"angular_momentum": 0, "pauli": 1, "pauli_cartesian": 2}


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def build() -> Path:
    """Compile the oracle library in place (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, i, ll, d, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_uint64
        P = ctypes.POINTER
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_basis_create.argtypes = [i, i, i, i, i, i, P(vp)]
        L.oracle_basis_free.argtypes = [vp]
        L.oracle_basis_dim.argtypes = [vp]
        L.oracle_basis_dim.restype = ll
        L.oracle_basis_states.argtypes = [vp, vp, vp, vp]
        L.oracle_basis_image.argtypes = [vp, u64, u64, P(u64), P(u64), P(d), P(u64)]
        L.oracle_orbit_images.argtypes = [i, i, i, i, ctypes.c_longlong, vp, vp, vp, vp, vp, vp]
        L.oracle_operator_build.argtypes = [vp, i, vp, ctypes.c_char_p, vp, vp, vp, i, i, P(vp)]
        L.oracle_operator_from_triplets.argtypes = [ll, ll, vp, vp, vp, P(vp)]
        L.oracle_operator_free.argtypes = [vp]
        L.oracle_operator_dim.argtypes = [vp]
        L.oracle_operator_dim.restype = ll
        L.oracle_operator_nnz.argtypes = [vp]
        L.oracle_operator_nnz.restype = ll
        L.oracle_operator_is_real.argtypes = [vp]
        L.oracle_operator_csr.argtypes = [vp, vp, vp, vp]
        L.oracle_operator_apply.argtypes = [vp, vp, vp]
        L.oracle_deterministic_start.argtypes = [ll, u64, vp]
        L.oracle_eigsh.argtypes = [vp, ll, i, d, ll, d, ll, u64, vp, i, vp, vp, vp, P(ll)]
        L.oracle_expm_plan.argtypes = [vp, d, d, ll, d, ll, P(ll), P(ll), P(d), P(d)]
        L.oracle_expm_apply.argtypes = [vp, d, d, ll, d, ll, vp, vp]
        L.oracle_hermitian_eigen.argtypes = [ll, vp, vp, vp]
        L.oracle_tridiagonal_eigen.argtypes = [ll, vp, vp, vp, vp]
        L.oracle_evolve.argtypes = [vp, vp, ll, vp, ll, d, ll, vp, vp]
        L.oracle_expm_lanczos.argtypes = [vp, vp, d, ll, vp]
        L.oracle_sector_shift.argtypes = [vp, vp, i, vp, ctypes.c_char_p, vp, vp, vp, ll, vp, ll, vp]
        L.oracle_spectral_function.argtypes = [vp, vp, ll, vp, d, d, ll, d, vp]
        L.oracle_lanczos_ritz.argtypes = [vp, vp, ll, d, P(ll), P(d), vp, vp, vp, vp, vp]
        L.oracle_thermal_iteration.argtypes = [vp, vp, ll, vp, ll, d, vp, vp, P(ll)]
        L.oracle_thermal_observables.argtypes = [vp, vp, ll, d, i, ll, vp, ll, vp, vp, vp]
        _LIB = L
    return _LIB


def _check(code: int) -> None:
    if code != 0:
        raise OracleError(code, lib().oracle_last_error().decode())


def _ptr(array: np.ndarray | None):
    return None if array is None else array.ctypes.data_as(ctypes.c_void_p)


class Basis:
    """Spin-1/2 chain sector built by the reference's orbit-hashing rules."""

    def __init__(self, sites: int, up: int | None = None, momentum: int | None = None,
                 parity: int | None = None, normalization: str = "angular_momentum"):
        handle = ctypes.c_void_p()
        _check(lib().oracle_basis_create(
            sites, -1 if up is None else up, 0 if momentum is None else 1,
            0 if momentum is None else momentum, 0 if parity is None else parity,
            NORMALIZATIONS[normalization], ctypes.byref(handle)))
        self.handle = handle
        self._free = lib().oracle_basis_free  # held so the destructor works during interpreter shutdown
        self.sites = sites
        self.up = up
        self.momentum = momentum
        self.parity = parity
        self.normalization = normalization

    def __del__(self):
        if getattr(self, "handle", None):
            self._free(self.handle)
            self.handle = None

    def __len__(self) -> int:
        return int(lib().oracle_basis_dim(self.handle))

    def states(self) -> tuple[np.ndarray, np.ndarray]:
        n = len(self)
        lo = np.zeros(n, np.uint64)
        hi = np.zeros(n, np.uint64)
        orbit = np.zeros(n, np.uint64)
        _check(lib().oracle_basis_states(self.handle, _ptr(lo), _ptr(hi), _ptr(orbit)))
        if self.sites <= 64:
            return lo, orbit
        return lo + (hi.astype(object) << 64), orbit

    def image(self, state: int):
        lo = ctypes.c_uint64(state & ((1 << 64) - 1))
        hi = ctypes.c_uint64(state >> 64)
        rep_lo, rep_hi, orbit = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        phase = (ctypes.c_double * 2)()
        found = lib().oracle_basis_image(self.handle, lo, hi, ctypes.byref(rep_lo), ctypes.byref(rep_hi),
                                         phase, ctypes.byref(orbit))
        if not found:
            return None
        return (rep_hi.value << 64) | rep_lo.value, complex(phase[0], phase[1]), orbit.value


def orbit_images(sites: int, states, momentum: int | None = None, parity: int | None = None):
    """Reduction images of physical states by the reference's per-orbit rule
    (spin_symmetry_sector, src/basis/mod.rs:760-841, one orbit at a time):
    (representative, phase, orbit size); orbit size 0 when the state's orbit
    is not in the sector. For sectors too large for the full lookup."""
    states = np.ascontiguousarray(states, np.uint64)
    n = len(states)
    rep_lo = np.zeros(n, np.uint64)
    rep_hi = np.zeros(n, np.uint64)
    phase = np.zeros(n, np.complex128)
    orbit = np.zeros(n, np.uint64)
    _check(lib().oracle_orbit_images(sites, 0 if momentum is None else 1, 0 if momentum is None else momentum,
                                     0 if parity is None else parity, n, _ptr(states), None, _ptr(rep_lo),
                                     _ptr(rep_hi), _ptr(phase), _ptr(orbit)))
    return rep_lo, phase, orbit


def _fixed_weight_count(cycles, weight):
    """States of the given weight fixed by a site permutation with these cycle lengths."""
    poly = [1] + [0] * weight
    for c in cycles:
        nxt = poly[:]
        for w in range(weight - c + 1):
            nxt[w + c] += poly[w]
        poly = nxt
    return poly[weight]


def _cycles(perm):
    seen, out = set(), []
    for start in range(len(perm)):
        if start in seen:
            continue
        n, i = 0, start
        while i not in seen:
            seen.add(i)
            i = perm[i]
            n += 1
        out.append(n)
    return out


def sector_dimension(sites: int, up: int, momentum: int, parity: int | None) -> int:
    """Dimension of a momentum (and parity) sector without enumerating it:
    the multiplicity of the sector's character in the permutation action on
    weight-`up` states: (1/|G|) sum_g conj(chi(g)) fix(g), over translations T^a
    (chi = exp(-2 pi i k a / L)) and, with parity p, reflections R T^a (chi = p
    exp(-2 pi i k a / L))."""
    total = 0j
    for a in range(sites):
        chi = complex(math.cos(2 * math.pi * momentum * a / sites), -math.sin(2 * math.pi * momentum * a / sites))
        rot = [(i + a) % sites for i in range(sites)]
        total += chi.conjugate() * _fixed_weight_count(_cycles(rot), up)
        if parity:
            refl = [sites - 1 - rot[i] for i in range(sites)]
            total += parity * chi.conjugate() * _fixed_weight_count(_cycles(refl), up)
    order = sites * (2 if parity else 1)
    value = total / order
    assert abs(value.imag) < 1e-6
    return int(round(value.real))



def encode_terms(terms):
    """Flatten ``[(label, [(coefficient, sites), ...]), ...]`` for the C ABI."""
    arity, symbols, n_couplings, coefficients, sites = [], [], [], [], []
    for label, couplings in terms:
        label = label.replace("|", "")
        arity.append(len(label))
        symbols.append(label)
        n_couplings.append(len(couplings))
        for coefficient, coupling_sites in couplings:
            coefficient = complex(coefficient)
            coefficients += [coefficient.real, coefficient.imag]
            sites += list(coupling_sites)
    return (np.asarray(arity, np.int32), "".join(symbols).encode(), np.asarray(n_couplings, np.int32),
            np.asarray(coefficients, np.float64), np.asarray(sites, np.int32))


@dataclass
class EigshResult:
    eigenvalues: np.ndarray
    residuals: np.ndarray
    eigenvectors: np.ndarray | None
    iterations: int
    reorthogonalization_passes: int
    conditional_second_passes: int


class Operator:
    """Assembled operator (row-sorted triplets, all formats act identically)."""

    def __init__(self, handle):
        self.handle = handle
        self._free = lib().oracle_operator_free  # held so the destructor works during interpreter shutdown

    @classmethod
    def build(cls, basis: Basis, terms, check_hermitian=True, check_particles=True) -> "Operator":
        arity, symbols, n_couplings, coefficients, sites = encode_terms(terms)
        handle = ctypes.c_void_p()
        _check(lib().oracle_operator_build(basis.handle, len(arity), _ptr(arity), symbols, _ptr(n_couplings),
                                           _ptr(coefficients), _ptr(sites), int(check_hermitian),
                                           int(check_particles), ctypes.byref(handle)))
        return cls(handle)

    @classmethod
    def from_triplets(cls, n: int, rows, cols, values) -> "Operator":
        rows = np.ascontiguousarray(rows, np.int64)
        cols = np.ascontiguousarray(cols, np.int64)
        values = np.ascontiguousarray(np.asarray(values, np.complex128))
        handle = ctypes.c_void_p()
        _check(lib().oracle_operator_from_triplets(n, len(rows), _ptr(rows), _ptr(cols), _ptr(values),
                                                   ctypes.byref(handle)))
        return cls(handle)

    @classmethod
    def diagonal(cls, values) -> "Operator":
        values = np.asarray(values, np.float64)
        n = len(values)
        idx = np.arange(n)
        return cls.from_triplets(n, idx, idx, values.astype(np.complex128))

    def __del__(self):
        if getattr(self, "handle", None):
            self._free(self.handle)
            self.handle = None

    @property
    def dim(self) -> int:
        return int(lib().oracle_operator_dim(self.handle))

    @property
    def nnz(self) -> int:
        return int(lib().oracle_operator_nnz(self.handle))

    @property
    def is_real(self) -> bool:
        return bool(lib().oracle_operator_is_real(self.handle))

    def csr(self):
        n, nnz = self.dim, self.nnz
        row_ptr = np.zeros(n + 1, np.int64)
        cols = np.zeros(nnz, np.int64)
        values = np.zeros(nnz, np.complex128)
        _check(lib().oracle_operator_csr(self.handle, _ptr(row_ptr), _ptr(cols), _ptr(values)))
        return row_ptr, cols, values

    def to_scipy(self):
        import scipy.sparse as sp
        row_ptr, cols, values = self.csr()
        return sp.csr_matrix((values, cols, row_ptr), shape=(self.dim, self.dim))

    def dense(self) -> np.ndarray:
        return self.to_scipy().toarray()

    def apply(self, x) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(x, np.complex128))
        y = np.zeros(self.dim, np.complex128)
        _check(lib().oracle_operator_apply(self.handle, _ptr(x), _ptr(y)))
        return y

    def eigsh(self, eigenpairs: int, target: str = "smallest_algebraic", shift: float = 0.0,
              krylov_dimension: int | None = None, tolerance: float = 1e-10, max_iterations: int = 1000,
              seed: int = 0, initial=None, eigenvectors: bool = False) -> EigshResult:
        n = self.dim
        if initial is not None:
            initial = np.ascontiguousarray(np.atleast_2d(np.asarray(initial, np.complex128)))
            n_initial = initial.shape[0]
        else:
            n_initial = 0
        values = np.zeros(eigenpairs)
        residuals = np.zeros(eigenpairs)
        vectors = np.zeros((eigenpairs, n), np.complex128) if eigenvectors else None
        counters = (ctypes.c_longlong * 3)()
        _check(lib().oracle_eigsh(self.handle, eigenpairs, TARGETS[target], shift, krylov_dimension or 0,
                                  tolerance, max_iterations, seed, _ptr(initial), n_initial, _ptr(values),
                                  _ptr(residuals), _ptr(vectors), counters))
        return EigshResult(values, residuals, vectors, counters[0], counters[1], counters[2])

    def expm_plan(self, coefficient: complex, max_degree: int = 55, tolerance: float = 0.5 * np.finfo(float).eps,
                  max_substeps: int = 10_000):
        degree, scaling = ctypes.c_longlong(), ctypes.c_longlong()
        shift = (ctypes.c_double * 2)()
        one_norm = ctypes.c_double()
        coefficient = complex(coefficient)
        _check(lib().oracle_expm_plan(self.handle, coefficient.real, coefficient.imag, max_degree, tolerance,
                                      max_substeps, ctypes.byref(degree), ctypes.byref(scaling), shift,
                                      ctypes.byref(one_norm)))
        return degree.value, scaling.value, complex(shift[0], shift[1]), one_norm.value

    def expm_apply(self, coefficient: complex, vector, max_degree: int = 55,
                   tolerance: float = 0.5 * np.finfo(float).eps, max_substeps: int = 10_000) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(vector, np.complex128))
        y = np.zeros(self.dim, np.complex128)
        coefficient = complex(coefficient)
        _check(lib().oracle_expm_apply(self.handle, coefficient.real, coefficient.imag, max_degree, tolerance,
                                       max_substeps, _ptr(x), _ptr(y)))
        return y

    def evolve(self, initial, times, krylov_dimension: int = 30, tolerance: float = 1e-10,
               max_substeps: int = 10_000):
        """Adaptive Hermitian Krylov evolution exp(-i H t) v on a time grid.

        Returns (states[n_times, dim], diagnostics dict) like
        evolve_with_diagnostics (src/solve/mod.rs:3374-3406)."""
        x = np.ascontiguousarray(np.asarray(initial, np.complex128))
        t = np.ascontiguousarray(np.asarray(times, np.float64))
        states = np.zeros((len(t), self.dim), np.complex128)
        diag = np.zeros(7)
        _check(lib().oracle_evolve(self.handle, _ptr(x), len(t), _ptr(t), krylov_dimension, tolerance, max_substeps,
                                   _ptr(states), _ptr(diag)))
        return states, dict(zip(EVOLUTION_DIAGNOSTICS, [int(v) for v in diag[:6]] + [float(diag[6])]))

    def expm_lanczos(self, initial, time: float, krylov_dimension: int = 30) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(initial, np.complex128))
        y = np.zeros(self.dim, np.complex128)
        _check(lib().oracle_expm_lanczos(self.handle, _ptr(x), time, krylov_dimension, _ptr(y)))
        return y


    def lanczos_ritz(self, initial, krylov_dimension: int, tolerance: float = 1e-12):
        """Full reorthogonalised Lanczos decomposition and its sorted Ritz system
        (lanczos_ritz, src/solve/mod.rs:2818-2857). Returns a dict with basis
        [m, dim], diagonal, off_diagonal, initial_norm, values and vectors
        (vectors[:, c] is the eigenvector of values[c])."""
        x = np.ascontiguousarray(np.asarray(initial, np.complex128))
        k = max(int(krylov_dimension), 0)
        basis = np.zeros((max(k, 1), self.dim), np.complex128)
        diag, off, values = np.zeros(max(k, 1)), np.zeros(max(k, 1)), np.zeros(max(k, 1))
        vectors = np.zeros(max(k, 1) ** 2)
        size, norm = ctypes.c_longlong(), ctypes.c_double()
        _check(lib().oracle_lanczos_ritz(self.handle, _ptr(x), krylov_dimension, tolerance, ctypes.byref(size),
                                         ctypes.byref(norm), _ptr(basis), _ptr(diag), _ptr(off), _ptr(values),
                                         _ptr(vectors)))
        m = size.value
        return {"basis": basis[:m], "diagonal": diag[:m], "off_diagonal": off[:max(m - 1, 0)],
                "initial_norm": norm.value, "values": values[:m],
                "vectors": vectors[:m * m].reshape(m, m).T.copy()}

    def thermal_iteration(self, initial, inverse_temperatures, krylov_dimension: int, tolerance: float = 1e-12):
        """ftlm_static_iteration (src/solve/mod.rs:3543-3554): (log_partition, mean_energy, krylov_dimension)."""
        x = np.ascontiguousarray(np.asarray(initial, np.complex128))
        b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)))
        lz, e = np.zeros(max(len(b), 1)), np.zeros(max(len(b), 1))
        size = ctypes.c_longlong()
        _check(lib().oracle_thermal_iteration(self.handle, _ptr(x), len(b), _ptr(b), krylov_dimension, tolerance,
                                              _ptr(lz), _ptr(e), ctypes.byref(size)))
        return lz[:len(b)], e[:len(b)], size.value

    def thermal_observables(self, initial, observables, inverse_temperatures, krylov_dimension: int,
                            tolerance: float = 1e-12, method: str = "ftlm"):
        """ftlm_/ltlm_observable_iteration (src/solve/mod.rs:3858-3898):
        (values[n_observables, n_betas] complex, identity[n_betas])."""
        x = np.ascontiguousarray(np.asarray(initial, np.complex128))
        b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)))
        handles = (ctypes.c_void_p * max(len(observables), 1))(*[o.handle for o in observables])
        values = np.zeros((max(len(observables), 1), max(len(b), 1)), np.complex128)
        identity = np.zeros(max(len(b), 1))
        _check(lib().oracle_thermal_observables(self.handle, _ptr(x), krylov_dimension, tolerance,
                                                {"ftlm": 0, "ltlm": 1}[method], len(observables), handles, len(b),
                                                _ptr(b), _ptr(values), _ptr(identity)))
        return values[:len(observables), :len(b)], identity[:len(b)]


    def spectral_function(self, created, frequencies, reference_energy: float, broadening: float,
                          krylov_dimension: int = 64, tolerance: float = 1e-10) -> np.ndarray:
        """spectral_function (src/dynamics/mod.rs:964-1021) of the probed vector
        `created` (= probe applied to the source state) on this target Hamiltonian."""
        x = np.ascontiguousarray(np.asarray(created, np.complex128))
        f = np.ascontiguousarray(np.atleast_1d(np.asarray(frequencies, np.float64)))
        out = np.zeros(max(f.size, 1))
        _check(lib().oracle_spectral_function(self.handle, _ptr(x), f.size, _ptr(f), reference_energy, broadening,
                                              krylov_dimension, tolerance, _ptr(out)))
        return out[:f.size]


def sector_shift(source: "Basis", target: "Basis", terms, vector) -> np.ndarray:
    """apply_sector_shift (src/operator/mod.rs:2305-2351): `terms` applied to a
    vector of `source`, reduced into `target`."""
    arity, symbols, n_couplings, coefficients, sites = encode_terms(terms)
    x = np.ascontiguousarray(np.asarray(vector, np.complex128))
    y = np.zeros(len(target), np.complex128)
    _check(lib().oracle_sector_shift(source.handle, target.handle, len(arity), _ptr(arity), symbols,
                                     _ptr(n_couplings), _ptr(coefficients), _ptr(sites), x.size, _ptr(x), y.size,
                                     _ptr(y)))
    return y


EVOLUTION_DIAGNOSTICS = ("lanczos_projections", "matrix_vector_products", "real_lanczos_projections",
                         "real_matrix_vector_products", "accepted_substeps", "rejected_trial_intervals",
                         "maximum_estimated_error")


def deterministic_start(n: int, seed: int) -> np.ndarray:
    out = np.zeros(n)
    _check(lib().oracle_deterministic_start(n, seed, _ptr(out)))
    return out


def hermitian_eigen(matrix: np.ndarray):
    a = np.ascontiguousarray(np.asarray(matrix, np.complex128))
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros(n * n, np.complex128)
    _check(lib().oracle_hermitian_eigen(n, _ptr(a), _ptr(w), _ptr(v)))
    return w, v.reshape(n, n).T  # columns are eigenvectors


def tridiagonal_eigen(diag, off):
    d = np.ascontiguousarray(diag, np.float64)
    e = np.ascontiguousarray(off, np.float64)
    n = len(d)
    w = np.zeros(n)
    z = np.zeros(n * n)
    _check(lib().oracle_tridiagonal_eigen(n, _ptr(d), _ptr(e), _ptr(w), _ptr(z)))
    return w, z.reshape(n, n).T


def heisenberg_terms(sites: int, j: float = 1.0, delta: float = 1.0, periodic: bool = True):
    """H = J sum (S+S- + S-S+)/2 + J*Delta sum SzSz, as in the reference tests."""
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]
    return [
        ("zz", [(j * delta, b) for b in bonds]),
        ("+-", [(0.5 * j, b) for b in bonds]),
        ("-+", [(0.5 * j, b) for b in bonds]),
    ]


def cpu_threads() -> int:
    return os.cpu_count() or 1
