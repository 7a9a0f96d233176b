"""Oracle answers to the reference's JSON protocol for spin chains (test infrastructure).

``tests/golden/make_frontend_requests.py`` uses this interpreter as the
stand-in native library while it records the requests that the reference's
unmodified Python frontend sends (``qmbed._ffi._call_json``,
bindings/python/src/qmbed/_ffi.py:189-207), and
``tests/test_gpu_frontend_requests.py`` uses it for the expected answers when
the same requests are replayed through ``libqmbed_b200.so``.

Every operator is the dense reduced matrix of ``oracle.general.reduced_dense``
(the reference's transition rule on lattice-map bases, with the model's site
permutation), so the answers cover the request forms the frontend sends:
``run`` (SolveRequest, bindings/capi/src/lib.rs:55-61) and the commands
``describe_basis``, ``create_model``, ``eigsh_model``, ``apply_model``,
``eigh_model``, ``measure_model``, ``matrix_elements_model``,
``evolve_model``, ``release_model`` and the Lanczos resource commands on
linear model expressions (lib.rs:64-410, 4046-4212, 4362-4432, 5513-5990).
"""

from __future__ import annotations

import numpy as np
import scipy.linalg

from oracle import general

def _oracle_module():
    from oracle import oracle
    oracle.build()
    return oracle


LOCAL = {"identity": "I", "z": "z", "raising": "+", "lowering": "-", "x": "x", "y": "y"}


def oracle_terms(terms):
    out = []
    for t in terms:
        symbols = "".join(LOCAL[name] for name in t["product"]["local"])
        couplings = [(complex(*c["coefficient"]), tuple(c["sites"])) for c in t["couplings"]]
        out.append((symbols, couplings))
    return out


def normalization(basis) -> str:
    if basis.get("normalization"):
        return basis["normalization"]
    return "pauli_cartesian" if basis.get("pauli") else "angular_momentum"


def oracle_basis(basis) -> general.GeneralSpinBasis:
    """A spin basis request as lattice maps (built-in momentum k: i -> i+1 with sector k; parity p: i -> L-1-i)."""
    sites = basis["sites"]
    up = basis.get("up")
    if basis.get("up_sectors") is not None:
        (up,) = basis["up_sectors"]
    maps = list(basis.get("symmetries") or [])
    if basis.get("momentum") is not None:
        maps.append({"destinations": [(i + 1) % sites for i in range(sites)], "sector": basis["momentum"]})
    if basis.get("parity") is not None:
        maps.append({"destinations": [sites - 1 - i for i in range(sites)], "sector": 0 if basis["parity"] == 1 else 1})
    return general.GeneralSpinBasis(sites, up, maps, reverse=bool(basis.get("reverse")))


def model_parts(request):
    """(static matrix, {component name: (matrix with coefficient 1, default or None)}) of a model request."""
    b = oracle_basis(request["basis"])
    norm, perm = normalization(request["basis"]), request.get("site_permutation")
    static = general.reduced_dense(b, oracle_terms(request["terms"]), norm, perm)
    components = {}
    for c in request.get("components") or []:
        default = complex(*c["default"]) if c.get("default") is not None else None
        components[c["name"]] = (general.reduced_dense(b, oracle_terms(c["terms"]), norm, perm), default)
    return static, components


def evaluate(parts, parameters=None) -> np.ndarray:
    """The model at the given parameter values (defaults for the rest), like EdModel::materialize."""
    static, components = parts
    h = static.copy()
    for name, (matrix, default) in components.items():
        value = complex(*parameters[name]) if parameters and name in parameters else default
        if value is None:
            raise ValueError(f"operator parameter {name!r} has no default and was not supplied")
        h = h + value * matrix
    return h


def model_matrix(request) -> np.ndarray:
    return evaluate(model_parts(request))


def act(h, action):
    """OperatorActionRequest (bindings/capi/src/lib.rs:937-945) on a dense matrix."""
    return {"normal": h, "conjugate": h.conj(), "adjoint": h.conj().T, "transpose": h.T}[action]


def complex_vectors(vectors):
    return [np.array([complex(*v) for v in vec]) for vec in vectors]


def pairs(vector):
    return [[float(v.real), float(v.imag)] for v in np.asarray(vector, dtype=complex)]


def selected(values, k, target):
    kind = target["kind"]
    order = {
        "smallest_algebraic": np.argsort(values),
        "largest_algebraic": np.argsort(-values),
        "smallest_magnitude": np.argsort(np.abs(values)),
        "largest_magnitude": np.argsort(-np.abs(values)),
    }.get(kind)
    if kind == "shift":
        order = np.argsort(np.abs(values - target["value"]))
    if order is None:
        raise NotImplementedError(kind)
    return order[:k]


class OracleProtocol:
    """Answers requests the way the reference library does, from dense oracle matrices."""

    def __init__(self):
        self.models = {}
        self.lanczos = {}
        self.plans = {}
        self.next_handle = 1

    def expression_matrix(self, e) -> np.ndarray:
        """OperatorExpressionRequest (bindings/capi/src/lib.rs:789-818) for models without parameters."""
        kind = e["kind"]
        if kind == "model":
            return act(self.matrix(e["handle"], e.get("parameters")), e.get("action", "normal"))
        if kind == "transform":
            return act(self.expression_matrix(e["operand"]), e.get("action", "normal"))
        if kind == "scale":
            return complex(*e["coefficient"]) * self.expression_matrix(e["operand"])
        if kind == "binary":
            left, right = self.expression_matrix(e["left"]), self.expression_matrix(e["right"])
            return {"add": left + right, "subtract": left - right, "product": left @ right}[e["operation"]]
        raise NotImplementedError(kind)

    def lanczos_command(self, op, request):
        """command_lanczos_* (bindings/capi/src/lib.rs:4046-4212) with the C++ oracle's lanczos_ritz."""
        if op == "lanczos_operator":
            h = self.expression_matrix(request["expression"])
            rows, cols = np.nonzero(h)
            operator = _oracle_module().Operator.from_triplets(h.shape[0], rows, cols, h[rows, cols])
            d = operator.lanczos_ritz(np.array([complex(*v) for v in request["initial"]]),
                                      request["krylov_dimension"], request.get("tolerance", 1e-13))
            handle = f"oracle-lanczos-{self.next_handle}"
            self.next_handle += 1
            self.lanczos[handle] = d
            return {"kind": "lanczos", "handle": handle, "dimension": h.shape[0],
                    "krylov_dimension": len(d["values"]), "initial_norm": d["initial_norm"],
                    "eigenvalues": d["values"].tolist(), "eigenvectors": d["vectors"].T.tolist()}
        d = self.lanczos[request["lanczos_handle"]]
        if op == "lanczos_combine":
            c = np.array([complex(*v) for v in request["coefficients"]])
        elif op == "lanczos_exponential":
            a = complex(*request["coefficient"])
            v = d["vectors"]
            c = v @ (v[0, :] * np.exp(a * d["values"]) * d["initial_norm"])
        elif op == "release_lanczos":
            self.lanczos.pop(request["lanczos_handle"])
            return {"kind": "released"}
        else:
            raise NotImplementedError(op)
        return {"kind": "vectors", "dimension": d["basis"].shape[1], "vectors": [pairs(c @ d["basis"])]}

    def matrix(self, handle, parameters=None) -> np.ndarray:
        model = self.models[handle]
        return evaluate(model, parameters) if isinstance(model, tuple) else model

    @staticmethod
    def entries(h, format):
        rows, cols = np.nonzero(h)
        return {"kind": "operator", "shape": list(h.shape), "format": format,
                "entries": [{"row": int(r), "column": int(c), "value": pairs([h[r, c]])[0]}
                            for r, c in zip(rows, cols)]}

    def eigensystem(self, h, solver):
        values, vectors = np.linalg.eigh(h)
        idx = selected(values, solver["eigenpairs"], solver["target"])
        idx = sorted(idx, key=lambda i: values[i])
        result = {"dimension": h.shape[0], "eigenvalues": [float(values[i]) for i in idx],
                  "residuals": [0.0 for _ in idx], "iterations": 0, "converged": True}
        if solver.get("eigenvectors"):
            result["eigenvectors"] = [pairs(vectors[:, i]) for i in idx]
        return result

    def run(self, request):
        return self.eigensystem(model_matrix(request), request["solver"])

    def command(self, request):
        op = request["operation"]
        if op == "create_model":
            handle = f"oracle-model-{self.next_handle}"
            self.next_handle += 1
            self.models[handle] = model_parts(request)
            return {"kind": "model", "handle": handle, "dimension": self.models[handle][0].shape[0]}
        if op == "describe_basis":
            b = oracle_basis(request["basis"])
            return {"kind": "basis", "dimension": len(b), "states": [str(int(x)) for x in b.states]}
        if op == "create_operator_model":
            m = request["static_operator"]
            h = np.zeros(m["shape"], dtype=complex)
            for e in m["entries"]:
                h[e["row"], e["column"]] += complex(*e["value"])
            handle = f"oracle-model-{self.next_handle}"
            self.next_handle += 1
            self.models[handle] = h
            return {"kind": "model", "handle": handle, "dimension": h.shape[0]}
        if op == "create_expm_action":
            # ExpmActionPlan (src/solve/mod.rs:116-248) as restated by the C++ oracle
            h = self.matrix(request["handle"])
            rows, cols = np.nonzero(h)
            operator = _oracle_module().Operator.from_triplets(h.shape[0], rows, cols, h[rows, cols])
            handle = f"oracle-expm-{self.next_handle}"
            self.next_handle += 1
            self.plans[handle] = (operator, complex(*request["coefficient"]), request.get("max_degree", 55),
                                  request.get("tolerance", 0.5 * np.finfo(float).eps))
            return {"kind": "expm_plan", "handle": handle, "dimension": h.shape[0]}
        if op == "apply_expm_action":
            operator, c, degree, tolerance = self.plans[request["expm_handle"]]
            return {"kind": "vectors", "dimension": operator.dim,
                    "vectors": [pairs(operator.expm_apply(c, v, max_degree=degree, tolerance=tolerance))
                                for v in complex_vectors(request["vectors"])]}
        if op == "release_expm_action":
            self.plans.pop(request["expm_handle"], None)
            return {"kind": "released"}
        if op == "release_model":
            self.models.pop(request["handle"], None)
            return {"kind": "released"}
        if op.startswith("lanczos_") or op == "release_lanczos":
            return self.lanczos_command(op, request)
        if op == "eigsh_operator_expression":
            return {"kind": "eigensystem", **self.eigensystem(self.expression_matrix(request["expression"]),
                                                              request["solver"])}
        if op == "apply_operator_expression":
            h = self.expression_matrix(request["expression"])
            return {"kind": "vectors", "dimension": h.shape[0],
                    "vectors": [pairs(h @ v) for v in complex_vectors(request["vectors"])]}
        if op in ("materialize_model", "evaluate_operator_expression"):
            h = self.matrix(request["handle"], request.get("parameters")) if op == "materialize_model" else \
                self.expression_matrix(request["expression"])
            return self.entries(h, request.get("format", "csc"))
        if op == "materialize_component_model":
            matrix, _ = self.models[request["handle"]][1][request["name"]]
            return self.entries(matrix, request.get("format", "csc"))
        h = self.matrix(request["handle"], request.get("parameters"))
        if op == "eigsh_model":
            return {"kind": "eigensystem", **self.eigensystem(h, request["solver"])}
        if op == "apply_model":
            a = act(h, request.get("action", "normal"))
            return {"kind": "vectors", "dimension": h.shape[0],
                    "vectors": [pairs(a @ v) for v in complex_vectors(request["vectors"])]}
        if op == "eigh_model":
            values, vectors = np.linalg.eigh(h)
            out = {"kind": "eigensystem", "dimension": h.shape[0], "eigenvalues": values.tolist()}
            if request.get("eigenvectors"):
                out["eigenvectors"] = [pairs(vectors[:, i]) for i in range(h.shape[0])]
            return out
        if op == "matrix_elements_model":
            left = complex_vectors(request["left_vectors"])
            right = complex_vectors(request["right_vectors"])
            if request.get("diagonal"):
                values = [np.vdot(a, h @ b) for a, b in zip(left, right)]
                shape = [len(left)]
            else:
                values = [np.vdot(a, h @ b) for a in left for b in right]
                shape = [len(left), len(right)]
            return {"kind": "measurements", "shape": shape, "values": pairs(values)}
        if op == "measure_model":
            fluct = request["measurement"] == "quantum_fluctuation"
            values = []
            for sample in request["samples"]:
                s = np.array([complex(*v) for v in sample["values"]])
                if sample["kind"] == "pure":
                    mean = np.vdot(s, h @ s)
                    values.append(np.vdot(s, h @ (h @ s)) - mean * mean if fluct else mean)
                else:
                    rho = s.reshape(h.shape)
                    mean = np.trace(h @ rho)
                    values.append(np.trace(h @ h @ rho) - mean * mean if fluct else mean)
            return {"kind": "measurements", "shape": [len(values)], "values": pairs(values)}
        if op == "evolve_model":
            ev = request["evolution"]
            times = ev["times"]
            states = []
            for t in times:
                u = scipy.linalg.expm(-1j * t * h)
                states.append([pairs(u @ v) for v in complex_vectors(request["vectors"])])
            return {"kind": "evolution", "times": times, "states": states}
        raise NotImplementedError(op)

    def call(self, symbol, request):
        if symbol == "qmbed_run_json":
            return self.run(request)
        if symbol == "qmbed_command_json":
            return self.command(request)
        raise NotImplementedError(symbol)
