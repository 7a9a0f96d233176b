"""Typed handles over the GPU engine: sector bases and operators.

These wrap the ``qmbed_gpu_*`` C ABI. Host arrays are numpy arrays; device
entry points take any object exposing ``data_ptr()`` (a torch CUDA tensor).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import STATUS, EigshHintC, EigshInfoC, EigshOptionsC, QmbedError, check, lib

NORMALIZATIONS = {"angular_momentum": 0, "pauli": 1, "pauli_cartesian": 2}
TARGETS = {
    "smallest_algebraic": 0,
    "largest_algebraic": 1,
    "smallest_magnitude": 2,
    "largest_magnitude": 3,
    "both_ends": 4,
    "shift": 5,
}
MODES = {"fp64": 0, "mixed": 1, "filtered": 2}
EVOLUTION_DIAGNOSTICS = ("lanczos_projections", "matrix_vector_products", "real_lanczos_projections",
                         "real_matrix_vector_products", "accepted_substeps", "rejected_trial_intervals",
                         "maximum_estimated_error")
STORAGE = {"matrix_free": 0, "packed": 1, "explicit": 2}
LOOKUPS = {"auto": 0, "table": 1, "search": 2, "legacy": 3, "table_generic": 4}
LOOKUPS_IN_USE = {1: "table", 2: "search", 3: "legacy", 4: "index", 5: "table_hop"}


def _sector_vectors(x, dim: int, dtype, what: str, batch: bool = False) -> np.ndarray:
    """x as contiguous `dtype` vectors of the sector's length (one vector, or rows
    of vectors with `batch`). The host entries read `dim` values per vector from
    the buffer they are given, so another length is refused here with the
    library's dimension-mismatch error instead of being read past its end."""
    arr = np.ascontiguousarray(np.atleast_2d(x) if batch else np.asarray(x), dtype)
    if arr.ndim != (2 if batch else 1) or arr.shape[-1] != dim:
        raise QmbedError(f"dimension mismatch: {what} has shape {tuple(np.shape(x))}, the sector dimension is {dim}",
                         STATUS["dimension_mismatch"])
    return arr


def _device_operands(*operands, device: int | None = None) -> None:
    """Refuses torch tensors that the kernels cannot use: one smaller than the
    bytes the action reads or writes through it, one that is not contiguous
    (the kernels use the dense span from data_ptr()), one off the GPU, or one
    on another GPU than `device` (the operator's). `operands` are
    (description, tensor, bytes) triples; sizes and layouts are checked for
    all of them before devices. Objects without these attributes (any other
    holder of a device pointer) are the caller's to size."""
    tensors = [(what, t, need) for what, t, need in operands
               if t is not None and hasattr(t, "numel") and hasattr(t, "element_size")]
    for what, t, need in tensors:
        have = int(t.numel()) * int(t.element_size())
        if have < need:
            raise QmbedError(f"dimension mismatch: {what} holds {have} bytes, the action needs {need}",
                             STATUS["dimension_mismatch"])
        if hasattr(t, "is_contiguous") and not t.is_contiguous():
            raise QmbedError(f"invalid options: {what} must be contiguous", STATUS["invalid_options"])
    for what, t, _ in tensors:
        if getattr(t, "is_cuda", True) is False:
            raise QmbedError(f"invalid options: {what} must be a CUDA tensor", STATUS["invalid_options"])
        index = getattr(getattr(t, "device", None), "index", None)
        if device is not None and index is not None and index != device:
            raise QmbedError(f"invalid options: {what} is on cuda:{index}, the operator on cuda:{device}",
                             STATUS["invalid_options"])


def _ptr(array):
    if array is None:
        return None
    if hasattr(array, "data_ptr"):
        return ctypes.c_void_p(array.data_ptr())
    return array.ctypes.data_as(ctypes.c_void_p)


class GpuBasis:
    """Spin-1/2 chain sector enumerated on the GPU (SpinBasis1D)."""

    def __init__(self, sites: int, up: int | None = None, momentum: int | None = None, parity: int | None = None,
                 normalization: str = "angular_momentum", device: int = 0):
        handle = ctypes.c_void_p()
        check(lib().qmbed_gpu_spin_basis_create(
            device, sites, -1 if up is None else up, 0 if momentum is None else 1,
            0 if momentum is None else momentum, 0 if parity is None else parity,
            NORMALIZATIONS[normalization], ctypes.byref(handle)))
        self.handle = handle
        self.sites, self.up, self.momentum, self.parity = sites, up, momentum, parity
        self.normalization = normalization
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            lib().qmbed_gpu_basis_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        dim = ctypes.c_uint64()
        check(lib().qmbed_gpu_basis_dimension(self.handle, ctypes.byref(dim)))
        return dim.value

    @property
    def build_seconds(self) -> float:
        value = ctypes.c_double()
        check(lib().qmbed_gpu_basis_build_seconds(self.handle, ctypes.byref(value)))
        return value.value

    def states(self, offset: int = 0, count: int | None = None):
        """Return (lo, hi, orbit) arrays for basis rows [offset, offset+count)."""
        n = len(self) - offset if count is None else count
        lo = np.zeros(n, np.uint64)
        hi = np.zeros(n, np.uint64)
        orbit = np.zeros(n, np.uint16)
        check(lib().qmbed_gpu_basis_states(self.handle, offset, n, _ptr(lo), _ptr(hi), _ptr(orbit)))
        return lo, hi, orbit

    def images(self, lo, hi=None):
        lo = np.ascontiguousarray(np.atleast_1d(lo), np.uint64)
        hi = None if hi is None else np.ascontiguousarray(np.atleast_1d(hi), np.uint64)
        n = len(lo)
        if lo.ndim != 1 or (hi is not None and hi.shape != lo.shape):
            raise QmbedError("dimension mismatch: the high state words must match the low ones one to one",
                             STATUS["dimension_mismatch"])
        index = np.zeros(n, np.int64)
        phase = np.zeros(n, np.complex128)
        orbit = np.zeros(n, np.uint16)
        check(lib().qmbed_gpu_basis_images(self.handle, _ptr(lo), _ptr(hi), n, _ptr(index), _ptr(phase), _ptr(orbit)))
        return index, phase, orbit

    def table_images(self, lo):
        """images() resolved through the sector's image table (u64 symmetry sectors)."""
        lo = np.ascontiguousarray(lo, np.uint64)
        n = len(lo)
        index = np.zeros(n, np.int64)
        phase = np.zeros(n, np.complex128)
        orbit = np.zeros(n, np.uint16)
        check(lib().qmbed_gpu_basis_table_images(self.handle, _ptr(lo), n, _ptr(index), _ptr(phase), _ptr(orbit)))
        return index, phase, orbit


def encode_terms(terms):
    """Flatten ``[(label, [(coefficient, sites), ...]), ...]`` for the C ABI."""
    arity, symbols, n_couplings, coefficients, sites = [], [], [], [], []
    for label, couplings in terms:
        label = label.replace("|", "")
        if not label:
            raise QmbedError("invalid or unregistered operator: operator products cannot be empty", 1)
        arity.append(len(label))
        symbols.append(label)
        n_couplings.append(len(couplings))
        for coefficient, coupling_sites in couplings:
            if len(coupling_sites) != len(label):
                # OperatorSpec::from_product (src/operator/mod.rs:226-247)
                raise QmbedError(f'invalid coupling: operator "{label}" has arity {len(label)}, but a coupling has '
                                 f"{len(coupling_sites)} sites", 2)
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
    fp32_iterations: int
    fp64_iterations: int
    operator_applications: int
    converged: bool
    hint_used: bool = False
    bound_applications: int = 0


class GpuOperator:
    """Hamiltonian assembled from local terms on a GPU basis (OperatorBuilder)."""

    def __init__(self, basis: GpuBasis, terms, storage: str = "packed", check_hermitian: bool = True,
                 check_particles: bool = True):
        arity, symbols, n_couplings, coefficients, sites = encode_terms(terms)
        handle = ctypes.c_void_p()
        check(lib().qmbed_gpu_operator_create(basis.handle, len(arity), _ptr(arity), symbols, _ptr(n_couplings),
                                              _ptr(coefficients), _ptr(sites), int(check_hermitian),
                                              int(check_particles), STORAGE[storage], ctypes.byref(handle)))
        self.handle = handle
        self.basis = basis

    def close(self):
        if getattr(self, "handle", None):
            lib().qmbed_gpu_operator_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        dim, real, storage, nnz, codes, seconds = (ctypes.c_uint64(), ctypes.c_int(), ctypes.c_int(),
                                                   ctypes.c_uint64(), ctypes.c_int(), ctypes.c_double())
        check(lib().qmbed_gpu_operator_info(self.handle, ctypes.byref(dim), ctypes.byref(real), ctypes.byref(storage),
                                            ctypes.byref(nnz), ctypes.byref(codes), ctypes.byref(seconds)))
        return {"dimension": dim.value, "is_real": bool(real.value), "storage": storage.value,
                "nnz_offdiag": nnz.value, "value_codes": codes.value, "assembly_seconds": seconds.value}

    @property
    def dim(self) -> int:
        return self.info()["dimension"]

    def _rows(self) -> int:
        """The sector dimension, read once (it never changes for an operator)."""
        n = self.__dict__.get("_rows_cache")
        if n is None:
            n = self._rows_cache = int(self.dim)
        return n

    def _device(self) -> int | None:
        return getattr(getattr(self, "basis", None), "device", None)

    def _vector_bytes(self, precision: int, complex_vectors: bool, columns: int = 1) -> int:
        return self._rows() * columns * (8 if precision == 64 else 4) * (2 if complex_vectors else 1)

    @property
    def is_real(self) -> bool:
        return self.info()["is_real"]

    def apply(self, x, force_matrix_free: bool = False) -> np.ndarray:
        """y = H x on host vectors (FP64). Real input uses the real action when possible."""
        x = np.asarray(x)
        complex_vectors = np.iscomplexobj(x) or not self.is_real
        xin = _sector_vectors(x, self.dim, np.complex128 if complex_vectors else np.float64, "the input vector")
        y = np.zeros_like(xin)
        check(lib().qmbed_gpu_operator_apply_host(self.handle, int(complex_vectors), _ptr(xin), _ptr(y),
                                                  int(force_matrix_free)))
        return y

    def apply_device(self, x, y, precision: int = 64, complex_vectors: bool = False, stream=None,
                     force_matrix_free: bool = False) -> None:
        """y = H x on device tensors (``data_ptr()``), FP64 or FP32."""
        need = self._vector_bytes(precision, complex_vectors)
        _device_operands(("the input vector", x, need), ("the output vector", y, need), device=self._device())
        check(lib().qmbed_gpu_operator_apply_device(self.handle, precision, int(complex_vectors), _ptr(x), _ptr(y),
                                                    None if stream is None else ctypes.c_void_p(stream),
                                                    int(force_matrix_free)))

    def apply_block_device(self, z, out, nb: int, precision: int = 64, alpha: float = 1.0, beta: float = 0.0,
                           gamma: float = 0.0, p=None, stream=None) -> None:
        """out = alpha (S^-1 H S) z + beta z + gamma p on row-major n x nb device blocks.

        Coordinates are orbit-scaled (z = x / sqrt(R) in symmetry sectors); real
        operators with packed or matrix-free storage.
        """
        need = self._vector_bytes(precision, False, nb)
        _device_operands(("the input block", z, need), ("the output block", out, need), ("the third block", p, need),
                         device=self._device())
        check(lib().qmbed_gpu_operator_apply_block_device(self.handle, precision, nb, _ptr(z), _ptr(p), _ptr(out),
                                                          alpha, beta, gamma,
                                                          None if stream is None else ctypes.c_void_p(stream)))

    def apply_device_noalloc(self, x, y, precision: int = 64, complex_vectors: bool = False, stream=None) -> None:
        """y = H x on device tensors without any device allocation by the library.

        For callers that manage all GPU memory themselves: the scaled input of
        symmetry sectors goes to a fixed 32 MiB device array shared by all
        calls, so vectors are limited to 32 MiB and concurrent calls race.
        """
        need = self._vector_bytes(precision, complex_vectors)
        _device_operands(("the input vector", x, need), ("the output vector", y, need), device=self._device())
        check(lib().qmbed_gpu_operator_apply_device_noalloc(self.handle, precision, int(complex_vectors), _ptr(x),
                                                            _ptr(y), None if stream is None else ctypes.c_void_p(stream)))

    def set_lookup(self, mode: str) -> None:
        """Lookup of the matrix-free action: "auto", "table", "search", "legacy" or "table_generic"."""
        check(lib().qmbed_gpu_operator_set_lookup(self.handle, LOOKUPS[mode]))

    def lookup_info(self) -> dict:
        in_use, chain, nbytes, seconds = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint64(), ctypes.c_double()
        check(lib().qmbed_gpu_operator_lookup_info(self.handle, ctypes.byref(in_use), ctypes.byref(chain),
                                                   ctypes.byref(nbytes), ctypes.byref(seconds)))
        return {"lookup": LOOKUPS_IN_USE.get(in_use.value, "none"), "chain_form": bool(chain.value),
                "table_bytes": nbytes.value, "table_seconds": seconds.value}

    def operand_bytes(self, precision: int = 64, complex_vectors: bool = False) -> float:
        value = ctypes.c_double()
        check(lib().qmbed_gpu_operator_operand_bytes(self.handle, precision, int(complex_vectors), ctypes.byref(value)))
        return value.value

    def csr(self):
        """Assembled rows (diagonal included) as (row_ptr, cols, values)."""
        nnz = ctypes.c_uint64()
        check(lib().qmbed_gpu_operator_export_csr(self.handle, ctypes.byref(nnz), None, None, None))
        n = self.dim
        row_ptr = np.zeros(n + 1, np.uint64)
        cols = np.zeros(nnz.value, np.uint32)
        values = np.zeros(nnz.value, np.complex128)
        check(lib().qmbed_gpu_operator_export_csr(self.handle, ctypes.byref(nnz), _ptr(row_ptr), _ptr(cols),
                                                  _ptr(values)))
        return row_ptr, cols, values

    def to_scipy(self):
        import scipy.sparse as sp
        row_ptr, cols, values = self.csr()
        return sp.csr_matrix((values, cols.astype(np.int64), row_ptr.astype(np.int64)), shape=(self.dim, self.dim))

    def eigsh(self, eigenpairs: int, target: str = "smallest_algebraic", shift: float = 0.0,
              krylov_dimension: int | None = None, tolerance: float = 1e-10, max_iterations: int = 1000,
              seed: int = 0, initial=None, eigenvectors: bool = False, mode: str = "fp64",
              hint: dict | None = None) -> EigshResult:
        """Reference eigsh (mode "fp64") or the mixed / filtered GPU modes.

        `hint` (optional): {"lower", "upper", "gap", "restart_keep", "check_steps"}, a
        predicted spectral interval and gap (qmbed_gpu_eigsh_hinted); the result
        then says whether the interval passed its Lanczos check."""
        n = self.dim
        options = EigshOptionsC(eigenpairs, TARGETS[target], shift, krylov_dimension or 0, tolerance, max_iterations,
                                seed, MODES[mode])
        if initial is not None:
            initial = _sector_vectors(initial, n, np.complex128, "the initial vectors", batch=True)
            n_initial = initial.shape[0]
        else:
            n_initial = 0
        values = np.zeros(eigenpairs)
        residuals = np.zeros(eigenpairs)
        vectors = np.zeros((eigenpairs, n), np.complex128) if eigenvectors else None
        info = EigshInfoC()
        # an empty hint (upper <= lower, restart_keep 0) changes nothing and reports the bound work
        hint = hint or {}
        h = EigshHintC(float(hint.get("lower", 0.0)), float(hint.get("upper", 0.0)), float(hint.get("gap", 0.0)),
                       int(hint.get("restart_keep", 0)), int(hint.get("check_steps", 8)), 0, 0)
        check(lib().qmbed_gpu_eigsh_hinted(self.handle, ctypes.byref(options), ctypes.byref(h), _ptr(initial),
                                           n_initial, _ptr(values), _ptr(residuals), _ptr(vectors),
                                           ctypes.byref(info)))
        used, bound = bool(h.used), int(h.bound_applications)
        return EigshResult(values, residuals, vectors, info.iterations, info.reorthogonalization_passes,
                           info.conditional_second_passes, info.fp32_iterations, info.fp64_iterations,
                           info.operator_applications, bool(info.converged), used, bound)

    def evolve(self, initial, times, krylov_dimension: int = 30, tolerance: float = 1e-10,
               max_substeps: int = 10_000):
        """exp(-i H t) initial on a nondecreasing time grid (reference evolve).

        Returns (states[n_times, dim], diagnostics dict)."""
        x = _sector_vectors(initial, self.dim, np.complex128, "the initial state")
        t = np.ascontiguousarray(np.asarray(times, np.float64))
        states = np.zeros((len(t), self.dim), np.complex128)
        diag = np.zeros(7)
        check(lib().qmbed_gpu_evolve(self.handle, _ptr(x), len(t), _ptr(t), krylov_dimension, tolerance,
                                     max_substeps, _ptr(states), _ptr(diag)))
        return states, dict(zip(EVOLUTION_DIAGNOSTICS, [int(v) for v in diag[:6]] + [float(diag[6])]))

    def expm_lanczos(self, initial, time: float, krylov_dimension: int = 30) -> np.ndarray:
        """exp(-i H time) initial from one Lanczos projection (reference expm_lanczos)."""
        x = _sector_vectors(initial, self.dim, np.complex128, "the initial state")
        y = np.zeros(self.dim, np.complex128)
        check(lib().qmbed_gpu_expm_lanczos(self.handle, _ptr(x), time, krylov_dimension, _ptr(y)))
        return y

    def chebyshev_evolve(self, initial, times, e_min: float = float("nan"), e_max: float = float("nan"),
                         tolerance: float = 1e-10, precision: int = 64, final_only: bool = False):
        """exp(-i H t) initial on a time grid by Chebyshev expansions (flip-chain operators).

        [e_min, e_max] must contain the spectrum; NaN uses the guaranteed
        +-sum|coefficients| bound. Returns (states[n_times or 1, dim], info dict)."""
        x = _sector_vectors(initial, self.dim, np.complex128, "the initial state")
        t = np.ascontiguousarray(np.asarray(times, np.float64))
        states = np.zeros((1 if final_only else len(t), self.dim), np.complex128)
        info = np.zeros(5)
        check(lib().qmbed_gpu_chebyshev_evolve(self.handle, _ptr(x), len(t), _ptr(t), e_min, e_max, tolerance,
                                               precision, int(final_only), _ptr(states), _ptr(info)))
        return states, {"applications": int(info[0]), "intervals": int(info[1]), "e_min": float(info[2]),
                        "e_max": float(info[3]), "max_norm_drift": float(info[4])}

    def chebyshev_evolve_device(self, state, times, e_min: float = float("nan"), e_max: float = float("nan"),
                                tolerance: float = 1e-10, precision: int = 64) -> dict:
        """In place on a device complex128 tensor (``data_ptr()``): state <- exp(-i H t_last) state,
        stepping through `times`. Returns the info dict of chebyshev_evolve."""
        _device_operands(("the state", state, self._vector_bytes(64, True)), device=self._device())
        t = np.ascontiguousarray(np.asarray(times, np.float64))
        info = np.zeros(5)
        check(lib().qmbed_gpu_chebyshev_evolve_device(self.handle, _ptr(state), len(t), _ptr(t), e_min, e_max,
                                                      tolerance, precision, _ptr(info)))
        return {"applications": int(info[0]), "intervals": int(info[1]), "e_min": float(info[2]),
                "e_max": float(info[3]), "max_norm_drift": float(info[4])}

    def expm_plan(self, coefficient: complex, max_degree: int = 55, tolerance: float = 0.5 * np.finfo(float).eps,
                  max_substeps: int = 10_000):
        degree, scaling, one_norm = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double()
        shift = (ctypes.c_double * 2)()
        coefficient = complex(coefficient)
        check(lib().qmbed_gpu_expm_plan(self.handle, coefficient.real, coefficient.imag, max_degree, tolerance,
                                        max_substeps, ctypes.byref(degree), ctypes.byref(scaling), shift,
                                        ctypes.byref(one_norm)))
        return degree.value, scaling.value, complex(shift[0], shift[1]), one_norm.value

    def expm_apply(self, coefficient: complex, vectors, max_degree: int = 55,
                   tolerance: float = 0.5 * np.finfo(float).eps, max_substeps: int = 10_000,
                   precision: int = 64) -> np.ndarray:
        x = _sector_vectors(vectors, self.dim, np.complex128, "the input vectors", batch=True)
        y = np.zeros_like(x)
        coefficient = complex(coefficient)
        check(lib().qmbed_gpu_expm_apply_host(self.handle, coefficient.real, coefficient.imag, max_degree, tolerance,
                                              max_substeps, precision, _ptr(x), _ptr(y), x.shape[0]))
        return y if np.ndim(vectors) > 1 else y[0]


def deterministic_start(n: int, seed: int, device: int = 0) -> np.ndarray:
    out = np.zeros(n)
    check(lib().qmbed_gpu_deterministic_start(device, n, seed, _ptr(out)))
    return out


def launch_count() -> int:
    """Kernels launched by libqmbed_b200.so in this process so far."""
    count = ctypes.c_uint64()
    check(lib().qmbed_gpu_launch_count(ctypes.byref(count)))
    return count.value


def device_count() -> int:
    count = ctypes.c_int()
    check(lib().qmbed_gpu_device_count(ctypes.byref(count)))
    return count.value


def heisenberg_terms(sites: int, j: float = 1.0, delta: float = 1.0, periodic: bool = True, j2: float = 0.0):
    """H = J sum_<ij> [ (S+S- + S-S+)/2 + Delta SzSz ] (+ J2 next-nearest), the reference test model."""
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]
    terms = [
        ("zz", [(j * delta, b) for b in bonds]),
        ("+-", [(0.5 * j, b) for b in bonds]),
        ("-+", [(0.5 * j, b) for b in bonds]),
    ]
    if j2:
        bonds2 = [(i, (i + 2) % sites) for i in range(sites if periodic else sites - 2)]
        terms += [
            ("zz", [(j2 * delta, b) for b in bonds2]),
            ("+-", [(0.5 * j2, b) for b in bonds2]),
            ("-+", [(0.5 * j2, b) for b in bonds2]),
        ]
    return terms


def tfim_terms(sites: int, j: float = 1.0, g: float = 1.0, fields=None, periodic: bool = False):
    """Transverse-field Ising chain with optional longitudinal fields (Pauli normalisation)."""
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]
    terms = [("zz", [(-j, b) for b in bonds]), ("x", [(-g, (i,)) for i in range(sites)])]
    if fields is not None:
        terms.append(("z", [(float(h), (i,)) for i, h in enumerate(fields)]))
    return terms


__all__ = ["GpuBasis", "GpuOperator", "EigshResult", "QmbedError", "deterministic_start", "device_count",
           "heisenberg_terms", "tfim_terms", "encode_terms"]
