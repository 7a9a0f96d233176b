"""qmbed_evolve_model_with_drive_json: callback-driven evolution against the oracle.

The reference evolves H(t) = H_0 + sum_j c_j(t) H_j, the c_j from the caller's
callback at every internal time, with adaptive RK4 step doubling
(bindings/capi/src/lib.rs:4695-4746; src/solve/mod.rs:3941-4138). The GPU
trajectory must match a tight SciPy integration of the oracle's dense
matrices (model parts from tests/frontend_protocol.py) to 1e-8, in real and
imaginary time, and the errors must follow the reference's texts.
"""

import ctypes
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Complex(ctypes.Structure):
    _fields_ = [("real", ctypes.c_double), ("imaginary", ctypes.c_double)]


Callback = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(Complex), ctypes.c_size_t)


def _drive(request, function, status=0):
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import lib
    library = lib()
    entry = library.qmbed_evolve_model_with_drive_json
    entry.argtypes = [ctypes.c_char_p, Callback, ctypes.c_void_p]
    entry.restype = ctypes.c_void_p
    seen = []

    @Callback
    def bridge(_context, time, coefficients, count):
        seen.append(time)
        for i, value in enumerate(function(time)[:count]):
            coefficients[i].real = value.real
            coefficients[i].imaginary = value.imag
        return status

    pointer = entry(json.dumps(request).encode(), bridge, None)
    try:
        response = json.loads(ctypes.string_at(pointer))
    finally:
        library.qmbed_string_free(ctypes.c_void_p(pointer))
    if response["status"] != "ok":
        raise QmbedError(response["error"])
    return response["result"], seen


def _model(command):
    L = 10
    bonds = [[i, (i + 1) % L] for i in range(L)]
    terms = [{"product": {"local": p}, "couplings": [{"coefficient": [c, 0.0], "sites": b} for b in bonds]}
             for p, c in ((["z", "z"], 1.0), (["raising", "lowering"], 0.5), (["lowering", "raising"], 0.5))]
    drive = [{"product": {"local": ["z", "z"]},
              "couplings": [{"coefficient": [0.4, 0.0], "sites": [i, (i + 2) % L]} for i in range(L)]}]
    request = {"basis": {"kind": "spin", "sites": L, "up": 5, "momentum": 0, "parity": 1}, "terms": terms,
               "components": [{"name": "drive", "terms": drive, "default": [1.0, 0.0]}]}
    return request, command({"operation": "create_model", **request})


@pytest.mark.parametrize("imaginary", [False, True])
def test_driven_trajectory_matches_a_tight_integration(imaginary):
    from scipy.integrate import solve_ivp
    from frontend_protocol import model_parts
    from qmbed_b200._lib import command
    request, model = _model(command)
    try:
        h0, components = model_parts(request)
        h1 = components["drive"][0]
        n = h0.shape[0]
        rng = np.random.default_rng(4)
        psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        psi /= np.linalg.norm(psi)
        times = [0.4, 1.0, 1.3]
        coefficient = lambda t: np.cos(2.0 * t)  # noqa: E731
        result, seen = _drive({"handle": model["handle"], "component_names": ["drive"], "initial_time": 0.1,
                               "vectors": [[[v.real, v.imag] for v in psi]],
                               "evolution": {"times": times, "tolerance": 1e-10, "imaginary_time": imaginary}},
                              lambda t: [complex(coefficient(t))])
        assert result["kind"] == "trajectory" and result["dimension"] == n and len(seen) > 0
        factor = -1.0 if imaginary else -1.0j
        reference = solve_ivp(lambda t, y: factor * ((h0 + coefficient(t) * h1) @ y), (0.1, times[-1]), psi,
                              method="DOP853", t_eval=times, rtol=1e-13, atol=1e-13)
        for k, states in enumerate(result["states"]):
            got = np.array([complex(*v) for v in states[0]])
            want = reference.y[:, k]
            want = want / np.linalg.norm(want)  # the reference rescales to the initial norm at every output
            assert abs(np.linalg.norm(got) - 1.0) <= 1e-12
            assert np.linalg.norm(got - want) <= 1e-8
    finally:
        command({"operation": "release_model", "handle": model["handle"]})


def test_drive_errors_follow_the_reference():
    from qmbed_b200 import QmbedError
    from qmbed_b200._lib import command
    request, model = _model(command)
    try:
        base = {"handle": model["handle"], "component_names": ["drive"], "initial_time": 0.0,
                "vectors": [[[1.0, 0.0]] + [[0.0, 0.0]] * (model["dimension"] - 1)],
                "evolution": {"times": [0.5]}}
        with pytest.raises(QmbedError, match=r'^invalid options: drive component order mismatch: expected \["drive"\]'):
            _drive({**base, "component_names": ["other"]}, lambda t: [1.0])
        with pytest.raises(QmbedError, match="^invalid options: drive callback returned status 1 at time 0"):
            _drive(base, lambda t: [1.0], status=1)
        with pytest.raises(QmbedError, match="^invalid options: time-dependent coefficient callback did not return 1"):
            _drive(base, lambda t: [complex(float("nan"), 0.0)])
        with pytest.raises(QmbedError, match="^invalid options: initial time must be finite"):
            _drive({**base, "initial_time": 1.0}, lambda t: [1.0])
    finally:
        command({"operation": "release_model", "handle": model["handle"]})
