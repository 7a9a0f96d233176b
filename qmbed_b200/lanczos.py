"""Full Lanczos decompositions and thermal Lanczos (FTLM / LTLM) on the GPU.

The functions mirror the reference's QuSpin-compatible Lanczos tools
(bindings/python/src/quspin/tools/lanczos.py: lanczos_full, lanczos_iter,
lin_comb_Q_T, expm_lanczos, FTLM_static_iteration, LTLM_static_iteration)
over the typed C-ABI: the Krylov basis Q_T stays in HBM behind a
``LanczosBasis`` handle, observables that are ``GpuOperator`` objects are
projected on the GPU, and other observables (anything with ``.dot``) are
projected on the host from the exported basis, as the reference does for
observables it cannot express natively. The recurrence and the thermal
formulas are the reference's (src/solve/mod.rs:2694-2857, 3457-3940).

``thermal_iteration`` is ftlm_static_iteration / ltlm_static_iteration
(log Z and the mean energy from one start vector); ``ftlm_sample`` runs many
random start vectors generated on the GPU and ``ftlm_average`` combines them.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .engine import GpuOperator, _ptr, _sector_vectors

METHODS = {"ftlm": 0, "ltlm": 1}


class LanczosBasis:
    """Device-resident Lanczos decomposition (the reference's LanczosRitzDecomposition)."""

    def __init__(self, op: GpuOperator, v0, m: int, eps: float = 1e-13):
        x = _sector_vectors(v0, op.dim, np.complex128, "v0")
        handle = ctypes.c_void_p()
        check(lib().qmbed_gpu_lanczos_create(op.handle, _ptr(x), int(m), float(eps), ctypes.byref(handle)))
        self._handle = handle
        dim, size, second = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        norm, real = ctypes.c_double(), ctypes.c_int()
        check(lib().qmbed_gpu_lanczos_info(handle, ctypes.byref(dim), ctypes.byref(size), ctypes.byref(norm),
                                           ctypes.byref(real), ctypes.byref(second)))
        self.dimension, self.krylov_dimension = dim.value, size.value
        self.initial_norm, self.is_real, self.second_passes = norm.value, bool(real.value), second.value
        m_ = self.krylov_dimension
        self.eigenvalues = np.zeros(m_)
        vectors = np.zeros(m_ * m_)
        self.diagonal = np.zeros(m_)
        self.off_diagonal = np.zeros(max(m_ - 1, 0) + 1)
        check(lib().qmbed_gpu_lanczos_ritz(handle, _ptr(self.eigenvalues), _ptr(vectors), _ptr(self.diagonal),
                                           _ptr(self.off_diagonal)))
        self.off_diagonal = self.off_diagonal[:max(m_ - 1, 0)]
        # vectors[c * m + r] is row r of eigenvector c; V[:, c] is eigenvector c
        self.eigenvectors = vectors.reshape(m_, m_).T.copy()

    @property
    def handle(self):
        if self._handle is None:
            raise RuntimeError("Lanczos decomposition is closed")
        return self._handle

    def close(self):
        if getattr(self, "_handle", None):
            lib().qmbed_gpu_lanczos_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def __len__(self) -> int:
        return self.krylov_dimension

    def to_numpy(self) -> np.ndarray:
        """The basis as rows, [krylov_dimension, dimension] complex."""
        out = np.zeros((self.krylov_dimension, self.dimension), np.complex128)
        check(lib().qmbed_gpu_lanczos_basis(self.handle, _ptr(out)))
        return out

    def __array__(self, dtype=None, copy=None):
        values = self.to_numpy()
        return values.astype(dtype, copy=False) if dtype is not None else values

    def __iter__(self):
        return iter(self.to_numpy())

    def linear_combination(self, coefficients) -> np.ndarray:
        c = np.ascontiguousarray(np.asarray(coefficients, np.complex128).reshape(-1))
        if c.size != self.krylov_dimension:
            raise ValueError("coefficient and Lanczos-vector counts differ")
        out = np.zeros(self.dimension, np.complex128)
        check(lib().qmbed_gpu_lanczos_combine(self.handle, _ptr(c), _ptr(out)))
        return out

    def exponential_action(self, coefficient: complex) -> np.ndarray:
        """|v| Q exp(c T) e_1 (exponential_action, src/solve/mod.rs:2642-2671)."""
        c = complex(coefficient)
        out = np.zeros(self.dimension, np.complex128)
        check(lib().qmbed_gpu_lanczos_exponential(self.handle, c.real, c.imag, _ptr(out)))
        return out

    def project(self, observable: GpuOperator, method: str = "ftlm") -> np.ndarray:
        """FTLM: <q_i|A|q_0> (m values); LTLM: <q_j|A|q_i> at [i, j] (m x m)."""
        m = self.krylov_dimension
        out = np.zeros(m * m if method == "ltlm" else m, np.complex128)
        check(lib().qmbed_gpu_lanczos_project(self.handle, METHODS[method], observable.handle, _ptr(out)))
        return out.reshape(m, m) if method == "ltlm" else out

    def thermal(self, observables: dict, inverse_temperatures, method: str = "ftlm"):
        """thermal_observable_iteration (src/solve/mod.rs:3858-3872) with this
        decomposition's Ritz system: ({name: values[n_betas]}, identity[n_betas])."""
        items = list(observables.items())
        b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)).reshape(-1))
        if all(isinstance(o, GpuOperator) for _, o in items):
            handles = (ctypes.c_void_p * max(len(items), 1))(*[o.handle for _, o in items])
            values = np.zeros((max(len(items), 1), max(b.size, 1)), np.complex128)
            identity = np.zeros(max(b.size, 1))
            check(lib().qmbed_gpu_lanczos_thermal(self.handle, METHODS[method], b.size, _ptr(b), len(items), handles,
                                                  _ptr(values), _ptr(identity)))
            return {k: values[i, :b.size] for i, (k, _) in enumerate(items)}, identity[:b.size]
        projected = [self.project(o, method) if isinstance(o, GpuOperator) else _host_projection(o, self, method)
                     for _, o in items]
        values, identity = thermal_contraction(method, self.eigenvalues, self.eigenvectors, projected, b)
        return {k: values[i] for i, (k, _) in enumerate(items)}, identity


def _host_projection(observable, basis, method: str) -> np.ndarray:
    q = basis.to_numpy() if isinstance(basis, LanczosBasis) else np.asarray(basis)
    if method == "ftlm":
        return q.conj() @ np.asarray(observable.dot(q[0]))
    applied = np.column_stack([np.asarray(observable.dot(v)) for v in q])
    return (q.conj() @ applied).T


def thermal_contraction(method: str, eigenvalues, eigenvectors, projected, inverse_temperatures):
    """thermal_observable_contraction (src/solve/mod.rs:3785-3806); V[:, c] is
    the eigenvector of eigenvalues[c]. Returns (values[n_observables, n_betas], identity)."""
    e = np.ascontiguousarray(np.asarray(eigenvalues, np.float64).reshape(-1))
    v = np.ascontiguousarray(np.asarray(eigenvectors, np.float64))
    m = e.size
    if v.shape != (m, m):
        raise ValueError("V must be a square Ritz eigenvector matrix")
    elements = np.ascontiguousarray(np.concatenate([np.asarray(p, np.complex128).reshape(-1) for p in projected])
                                    if projected else np.zeros(1, np.complex128))
    b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)).reshape(-1))
    values = np.zeros((max(len(projected), 1), max(b.size, 1)), np.complex128)
    identity = np.zeros(max(b.size, 1))
    check(lib().qmbed_gpu_thermal_contraction(METHODS[method], m, _ptr(e), _ptr(v), len(projected), _ptr(elements),
                                              b.size, _ptr(b), _ptr(values), _ptr(identity)))
    return values[:len(projected), :b.size], identity[:b.size]


# ---- QuSpin-compatible names (bindings/python/src/quspin/tools/lanczos.py) ----

def lanczos_full(A: GpuOperator, v0, m: int, full_ortho=False, out=None, eps=None):
    """(E, V, Q_T): ascending Ritz values, Ritz vectors as columns, device basis."""
    del full_ortho, out
    q = LanczosBasis(A, v0, m, 1e-13 if eps is None else float(eps))
    return q.eigenvalues, q.eigenvectors, q


def lanczos_iter(A: GpuOperator, v0, m: int, return_vec_iter=True, copy_v0=True, copy_A=False, eps=None):
    del copy_v0, copy_A
    e, v, q = lanczos_full(A, v0, m, eps=eps)
    if return_vec_iter:
        return e, v, q
    q.close()
    return e, v


def lin_comb_Q_T(coeff, Q_T, out=None):
    c = np.asarray(coeff)
    if isinstance(Q_T, LanczosBasis):
        values = Q_T.linear_combination(c)
    else:
        values = c @ np.asarray(list(Q_T) if not isinstance(Q_T, np.ndarray) else Q_T)
    if out is not None:
        out[...] = values
        return out
    return values


def expm_lanczos(E, V, Q_T, a=1.0, out=None):
    e = np.asarray(E, np.float64)
    v = np.asarray(V)
    if v.shape != (e.size, e.size):
        raise ValueError("V must be a square Ritz eigenvector matrix")
    coefficients = v @ (np.exp(complex(a) * e) * v[0, :].conj())
    if isinstance(Q_T, LanczosBasis):
        coefficients = coefficients * Q_T.initial_norm
    return lin_comb_Q_T(coefficients, Q_T, out=out)


def _static_iteration(method, O_dict, E, V, Q_T, beta):
    if not hasattr(O_dict, "items") or not O_dict:
        raise ValueError("O_dict must be a nonempty mapping")
    b = np.asarray(beta, np.float64)
    items = list(O_dict.items())
    projected = [Q_T.project(o, method) if isinstance(Q_T, LanczosBasis) and isinstance(o, GpuOperator)
                 else _host_projection(o, Q_T, method) for _, o in items]
    values, identity = thermal_contraction(method, E, np.real(np.asarray(V)), projected, b.reshape(-1))
    out = {k: np.real_if_close(values[i].reshape(b.shape)).squeeze() for i, (k, _) in enumerate(items)}
    return out, identity.reshape(b.shape).squeeze()


def FTLM_static_iteration(O_dict, E, V, Q_T, beta=0):
    """One finite-temperature Lanczos observable iteration."""
    return _static_iteration("ftlm", O_dict, E, V, Q_T, beta)


def LTLM_static_iteration(O_dict, E, V, Q_T, beta=0):
    """One low-temperature Lanczos observable iteration."""
    return _static_iteration("ltlm", O_dict, E, V, Q_T, beta)


# ---- partition-function estimates -------------------------------------------

def thermal_iteration(op: GpuOperator, initial, inverse_temperatures, krylov_dimension: int,
                      tolerance: float = 1e-12):
    """ftlm_static_iteration (src/solve/mod.rs:3543-3554): (log_partition, mean_energy, krylov_dimension)."""
    x = _sector_vectors(initial, op.dim, np.complex128, "the initial vector")
    b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)))
    lz, e = np.zeros(max(b.size, 1)), np.zeros(max(b.size, 1))
    size = ctypes.c_uint64()
    check(lib().qmbed_gpu_thermal_iteration(op.handle, _ptr(x), b.size, _ptr(b), int(krylov_dimension), tolerance,
                                            _ptr(lz), _ptr(e), ctypes.byref(size)))
    return lz[:b.size], e[:b.size], size.value


def ftlm_sample(op: GpuOperator, vectors: int, inverse_temperatures, krylov_dimension: int, seed: int = 0,
                tolerance: float = 1e-12):
    """FTLM estimates from `vectors` random start vectors generated on the GPU:
    (log_partition[vectors, n_betas], mean_energy[vectors, n_betas], lengths[vectors])."""
    b = np.ascontiguousarray(np.atleast_1d(np.asarray(inverse_temperatures, np.float64)))
    lz = np.zeros((vectors, max(b.size, 1)))
    e = np.zeros((vectors, max(b.size, 1)))
    lengths = np.zeros(vectors, np.int32)
    check(lib().qmbed_gpu_ftlm_sample(op.handle, int(vectors), int(seed), b.size, _ptr(b), int(krylov_dimension),
                                      tolerance, _ptr(lz), _ptr(e), _ptr(lengths)))
    return lz[:, :b.size], e[:, :b.size], lengths


def ftlm_start(op: GpuOperator, index: int, seed: int = 0) -> np.ndarray:
    """Start vector `index` of ftlm_sample(op, ..., seed) (complex, as generated on the GPU)."""
    out = np.zeros(op.dim, np.complex128)
    check(lib().qmbed_gpu_ftlm_start(op.handle, int(seed), int(index), _ptr(out)))
    return out


def ftlm_average(log_partition, mean_energy):
    """Combine per-vector estimates: Z = mean_r Z_r and E = sum_r Z_r E_r / sum_r Z_r,
    evaluated in log space. Returns (log Z[n_betas], E[n_betas])."""
    lz = np.atleast_2d(np.asarray(log_partition, np.float64))
    e = np.atleast_2d(np.asarray(mean_energy, np.float64))
    top = lz.max(axis=0)
    w = np.exp(lz - top)
    return top + np.log(w.mean(axis=0)), (w * e).sum(axis=0) / w.sum(axis=0)
