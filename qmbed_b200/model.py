"""Request types and model handles with the names of the reference Python API.

Mirrors ``bindings/python/src/qmbed/model.py`` and the ``NativeModel`` /
``NativeExpmAction`` classes of ``bindings/python/src/qmbed/_ffi.py``
(matrixlab-research/QMBED): the same dataclasses serialise to the same JSON
requests, which ``libqmbed_b200.so`` executes on the GPU. ``EigshOptions``
adds one optional field, ``precision`` ("fp64" runs the reference
algorithms; "mixed" uses FP32 vectors with FP64 refinement).
"""

from __future__ import annotations

import weakref
from dataclasses import dataclass
from enum import Enum
from typing import Any, Iterable, Sequence

import numpy as np

from ._lib import QmbedError, command, run


class LocalOperator(str, Enum):
    IDENTITY = "identity"
    NUMBER = "number"
    Z = "z"
    RAISING = "raising"
    LOWERING = "lowering"
    X = "x"
    Y = "y"


@dataclass(frozen=True)
class OpProduct:
    local: tuple[LocalOperator | str, ...]
    split: int | None = None
    splits: tuple[int, ...] = ()

    def request(self) -> dict:
        local = [op.value if isinstance(op, LocalOperator) else op for op in self.local]
        result: dict[str, Any] = {"local": local}
        if self.splits:
            if self.split is not None:
                raise ValueError("OpProduct cannot define both split and splits")
            result["splits"] = list(self.splits)
        elif self.split is not None:
            result["split"] = self.split
        return result


@dataclass(frozen=True)
class Coupling:
    coefficient: complex
    sites: tuple[int, ...]

    def request(self) -> dict:
        c = complex(self.coefficient)
        return {"coefficient": [c.real, c.imag], "sites": list(self.sites)}


@dataclass(frozen=True)
class OperatorSpec:
    product: OpProduct
    couplings: tuple[Coupling, ...]

    def request(self) -> dict:
        return {"product": self.product.request(), "couplings": [c.request() for c in self.couplings]}


@dataclass(frozen=True)
class SpinBasis:
    sites: int
    spin_twice: int = 1
    up: int | None = None
    momentum: int | None = None
    parity: int | None = None
    pauli: bool = False

    def request(self) -> dict:
        return {"kind": "spin", "sites": self.sites, "spin_twice": self.spin_twice, "up": self.up,
                "momentum": self.momentum, "parity": self.parity, "pauli": self.pauli}


@dataclass(frozen=True)
class EigshOptions:
    eigenpairs: int
    target: str = "smallest_algebraic"
    shift: float | None = None
    krylov_dimension: int | None = None
    tolerance: float = 1.0e-10
    max_iterations: int = 1_000
    seed: int = 0
    eigenvectors: bool = False
    precision: str = "fp64"

    def request(self) -> dict:
        target = {"kind": "shift", "value": self.shift} if self.target == "shift" else {"kind": self.target}
        return {"eigenpairs": self.eigenpairs, "target": target, "krylov_dimension": self.krylov_dimension,
                "tolerance": self.tolerance, "max_iterations": self.max_iterations, "seed": self.seed,
                "eigenvectors": self.eigenvectors, "precision": self.precision}


@dataclass(frozen=True)
class Eigensystem:
    dimension: int
    eigenvalues: tuple[float, ...]
    residuals: tuple[float, ...]
    iterations: int
    converged: bool
    eigenvectors: tuple[tuple[complex, ...], ...] | None = None


def _eigensystem(result: dict) -> Eigensystem:
    vectors = result.get("eigenvectors")
    return Eigensystem(
        dimension=result["dimension"], eigenvalues=tuple(result["eigenvalues"]),
        residuals=tuple(result["residuals"]), iterations=result["iterations"], converged=result["converged"],
        eigenvectors=None if vectors is None else tuple(tuple(complex(r, i) for r, i in v) for v in vectors))


def eigsh(basis: SpinBasis, terms: Sequence[OperatorSpec], options: EigshOptions, *, format: str = "csc") -> Eigensystem:
    """Selected eigenpairs of the Hamiltonian assembled from ``terms`` (reference ``qmbed.eigsh``)."""
    return _eigensystem(run({"basis": basis.request(), "terms": [t.request() for t in terms], "format": format,
                             "solver": options.request()}))


def _vectors_request(vectors) -> list:
    array = np.atleast_2d(np.asarray(vectors, np.complex128))
    return [[[float(v.real), float(v.imag)] for v in row] for row in array]


def _vectors_result(result: dict) -> np.ndarray:
    return np.asarray([[complex(r, i) for r, i in v] for v in result["vectors"]], np.complex128)


def _release(kind: str, key: str, handle: str) -> None:
    try:
        command({"operation": kind, key: handle})
    except Exception:
        pass


class NativeModel:
    """Owned reference to one persistent model held by the engine (create_model)."""

    def __init__(self, request: dict[str, Any]):
        result = command({"operation": "create_model", **request})
        self._handle: str | None = str(result["handle"])
        self.dimension = int(result["dimension"])
        self._finalizer = weakref.finalize(self, _release, "release_model", "handle", self._handle)

    @property
    def handle(self) -> str:
        if self._handle is None:
            raise QmbedError("QMBED model is closed")
        return self._handle

    @property
    def closed(self) -> bool:
        return self._handle is None

    def execute(self, operation: str, **options: Any) -> dict[str, Any]:
        return command({"operation": operation, "handle": self.handle, **options})

    def eigsh(self, options: EigshOptions, parameters: dict[str, complex] | None = None,
              format: str = "csc") -> Eigensystem:
        params = {k: [complex(v).real, complex(v).imag] for k, v in (parameters or {}).items()}
        return _eigensystem(self.execute("eigsh_model", solver=options.request(), parameters=params, format=format))

    def eigh(self, eigenvectors: bool = False, parameters: dict[str, complex] | None = None) -> Eigensystem:
        """Every eigenpair (the eigh_model command, bindings/capi/src/lib.rs:5290-5300)."""
        params = {k: [complex(v).real, complex(v).imag] for k, v in (parameters or {}).items()}
        return _eigensystem(self.execute("eigh_model", eigenvectors=eigenvectors, parameters=params))

    def apply(self, vectors, parameters: dict[str, complex] | None = None) -> np.ndarray:
        params = {k: [complex(v).real, complex(v).imag] for k, v in (parameters or {}).items()}
        return _vectors_result(self.execute("apply_model", vectors=_vectors_request(vectors), parameters=params))

    def evolve(self, vectors, times, *, krylov_dimension: int = 64, tolerance: float = 1e-10,
               max_substeps: int = 10_000, parameters: dict[str, complex] | None = None) -> np.ndarray:
        """exp(-i H t) applied to each column at each time: the evolve_model
        command (bindings/capi/src/lib.rs:4673-4694). Returns [time][column][component]."""
        params = {k: [complex(v).real, complex(v).imag] for k, v in (parameters or {}).items()}
        result = self.execute("evolve_model", vectors=_vectors_request(vectors), parameters=params,
                              evolution={"times": [float(t) for t in times], "krylov_dimension": krylov_dimension,
                                         "tolerance": tolerance, "max_substeps": max_substeps})
        return np.array([[[complex(re, im) for re, im in column] for column in columns]
                         for columns in result["states"]])

    def close(self) -> None:
        if self._handle is None:
            return
        command({"operation": "release_model", "handle": self._handle})
        self._handle = None
        self._finalizer.detach()

    def __enter__(self) -> "NativeModel":
        return self

    def __exit__(self, *_exc: object) -> None:
        self.close()


class NativeExpmAction:
    """Owned reusable exponential-action plan (create_expm_action / apply_expm_action)."""

    def __init__(self, model: NativeModel, coefficient: complex, *, max_degree: int = 55,
                 tolerance: float = 0.5 * np.finfo(np.float64).eps, max_substeps: int = 10_000,
                 parameters: dict[str, complex] | None = None):
        result = command({
            "operation": "create_expm_action", "handle": model.handle,
            "parameters": {str(k): [complex(v).real, complex(v).imag] for k, v in (parameters or {}).items()},
            "coefficient": [complex(coefficient).real, complex(coefficient).imag],
            "max_degree": int(max_degree), "tolerance": float(tolerance), "max_substeps": int(max_substeps)})
        self._handle: str | None = str(result["handle"])
        self.dimension = int(result["dimension"])
        self._model = model
        self._finalizer = weakref.finalize(self, _release, "release_expm_action", "expm_handle", self._handle)

    @property
    def handle(self) -> str:
        if self._handle is None:
            raise QmbedError("QMBED exponential-action plan is closed")
        return self._handle

    def apply(self, vectors, *, threads: int | None = None) -> np.ndarray:
        request: dict[str, Any] = {"operation": "apply_expm_action", "expm_handle": self.handle,
                                   "vectors": _vectors_request(vectors)}
        if threads is not None:
            request["threads"] = int(threads)
        return _vectors_result(command(request))

    def close(self) -> None:
        if self._handle is None:
            return
        command({"operation": "release_expm_action", "expm_handle": self._handle})
        self._handle = None
        self._finalizer.detach()

    def __enter__(self) -> "NativeExpmAction":
        return self

    def __exit__(self, *_exc: object) -> None:
        self.close()


def heisenberg_specs(sites: int, j: float = 1.0, delta: float = 1.0, periodic: bool = True) -> list[OperatorSpec]:
    """Heisenberg/XXZ terms zz(J Delta) + (+-)(J/2) + (-+)(J/2) as OperatorSpecs."""
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]

    def spec(local, coefficient):
        return OperatorSpec(OpProduct(tuple(local)), tuple(Coupling(coefficient, b) for b in bonds))

    return [spec(("z", "z"), j * delta), spec(("raising", "lowering"), 0.5 * j), spec(("lowering", "raising"), 0.5 * j)]


__all__ = ["LocalOperator", "OpProduct", "Coupling", "OperatorSpec", "SpinBasis", "EigshOptions", "Eigensystem",
           "eigsh", "NativeModel", "NativeExpmAction", "heisenberg_specs", "QmbedError"]
