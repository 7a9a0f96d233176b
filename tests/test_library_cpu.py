"""Host-side checks of libqmbed_b200.so that need no GPU: the library loads,
exports every symbol its header declares, and the JSON boundary rejects
malformed requests with the reference's error texts before touching CUDA."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def library():
    from qmbed_b200 import build
    build.build()
    from qmbed_b200._lib import lib
    return lib()


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        names |= set(re.findall(r"QMBED_API\s+[\w\s\*]+?\b(qmbed_\w+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported(library):
    names = declared_symbols()
    assert {"qmbed_run_json", "qmbed_command_json", "qmbed_string_free", "qmbed_evolve_model_with_drive_json",
            "qmbed_register_user_basis_32_json", "qmbed_register_user_basis_64_json"} <= names
    for name in names:
        assert hasattr(library, name), name
    exported = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "qmbed_b200" / "libqmbed_b200.so")],
                              capture_output=True, text=True, check=True).stdout
    public = {line.split()[-1] for line in exported.splitlines() if " T " in line}
    assert public == names, public ^ names


def _json(library, symbol, payload: bytes) -> dict:
    import json
    pointer = getattr(library, symbol)(payload)
    try:
        return json.loads(ctypes.string_at(pointer))
    finally:
        library.qmbed_string_free(pointer)


def test_malformed_requests_are_errors_not_crashes(library):
    r = _json(library, "qmbed_run_json", b"{not json")
    assert r["status"] == "error" and r["error"].startswith("invalid options: invalid binding request")
    r = _json(library, "qmbed_command_json", b'{"operation":"no_such_operation"}')
    assert r["status"] == "error" and "no_such_operation" in r["error"]
    r = _json(library, "qmbed_run_json", b'{"basis":{"kind":"boson","sites":3,"states_per_site":2},'
                                         b'"terms":[],"solver":{"eigenpairs":1,"target":{"kind":"smallest_algebraic"}}}')
    assert r["status"] == "error" and r["error"].startswith("unsupported backend")
    r = _json(library, "qmbed_command_json", b'{"operation":"release_model","handle":"abc"}')
    assert r["status"] == "error" and "is not a positive integer" in r["error"]
    pointer = library.qmbed_run_json(None)
    assert b"request pointer is null" in ctypes.string_at(pointer)
    library.qmbed_string_free(pointer)


def test_callback_exports_validate_their_arguments(library):
    """Null pointers give the reference's fixed errors (bindings/capi/src/lib.rs:6159-6165); user bases are
    outside the engine."""
    library.qmbed_evolve_model_with_drive_json.restype = ctypes.c_void_p
    pointer = library.qmbed_evolve_model_with_drive_json(b"{}", None, None)
    assert b"drive callback is null" in ctypes.string_at(pointer)
    library.qmbed_string_free(pointer)
    pointer = library.qmbed_evolve_model_with_drive_json(None, None, None)
    assert b"request pointer is null" in ctypes.string_at(pointer)
    library.qmbed_string_free(pointer)
    library.qmbed_register_user_basis_32_json.restype = ctypes.c_void_p
    pointer = library.qmbed_register_user_basis_32_json(b"{}", None, None, None, None, 0)
    assert b"unsupported backend" in ctypes.string_at(pointer)
    library.qmbed_string_free(pointer)


def test_typed_entries_reject_null_arguments_before_cuda(library):
    """Null handles, components and output pointers are argument errors
    (QMBED_STATUS_INVALID_OPTIONS = 8), raised before any device work."""
    import numpy as np
    from qmbed_b200._lib import EigshOptionsC
    invalid = 8

    def ptr(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    values, residuals = np.zeros(4), np.zeros(4)
    options = EigshOptionsC()
    assert library.qmbed_gpu_eigsh_hinted(None, ctypes.byref(options), None, None, 0, ptr(values), ptr(residuals),
                                          None, None) == invalid
    assert b"null operator" in library.qmbed_gpu_last_error()
    components = (ctypes.c_void_p * 1)(None)
    coefficients, steps = np.ones(1), np.zeros(1, np.int32)
    assert library.qmbed_gpu_scan_solve(1, 1, components, 1, ptr(coefficients), 1, 1e-10, 10, 0, ptr(values), None,
                                        None, ptr(steps), None) == invalid
    assert b"null scan component" in library.qmbed_gpu_last_error()
    assert library.qmbed_gpu_scan_solve(0, 1, components, 1, ptr(coefficients), 1, 1e-10, 10, 0, ptr(values), None,
                                        None, ptr(steps), None) == invalid
    assert library.qmbed_gpu_scan_barrier_selftest(0, None) == invalid
    assert library.qmbed_gpu_flip_wait_selftest(0, None) == invalid
    assert library.qmbed_gpu_lanczos_extremes(None, 8, 0, None) == invalid
    assert b"null operator" in library.qmbed_gpu_last_error()


def test_struct_layouts_match_the_header(library):
    from qmbed_b200._lib import EigshHintC, EigshInfoC, EigshOptionsC
    assert ctypes.sizeof(EigshOptionsC) == 64
    assert ctypes.sizeof(EigshInfoC) == 56
    assert ctypes.sizeof(EigshHintC) == 48  # qmbed_eigsh_hint: 3 doubles, u64, 2 ints, u64


def test_missing_library_fails_loudly(tmp_path):
    code = ("import os, sys; os.environ['QMBED_B200_LIBRARY']=sys.argv[1];"
            "from qmbed_b200._lib import lib, QmbedError\n"
            "try:\n lib()\nexcept QmbedError as e:\n print('raised', e)\n")
    out = subprocess.run(["python", "-c", code, str(tmp_path / "missing.so")], capture_output=True, text=True,
                         cwd=ROOT)
    assert "raised" in out.stdout and "not found" in out.stdout


def test_ctypes_bindings_match_the_header(library):
    """Every function the header declares is bound in qmbed_b200._lib with as
    many argument types as the declaration has parameters (a drifted binding
    would pass arguments in the wrong slots). The three callback exports are
    bound by the reference's own frontend, not by this package."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "qmbed_b200.h").read_text(), flags=re.S)
    declared = {}
    for m in re.finditer(r"QMBED_API\s+[\w\s\*]+?\b(qmbed_\w+)\s*\((.*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        declared[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    assert len(declared) == len(declared_symbols())
    frontend_only = {"qmbed_evolve_model_with_drive_json", "qmbed_register_user_basis_32_json",
                     "qmbed_register_user_basis_64_json"}
    for name, count in declared.items():
        argtypes = getattr(getattr(library, name), "argtypes", None)
        if name in frontend_only or (argtypes is None and count == 0):
            continue
        assert argtypes is not None, f"{name} has no argtypes"
        assert len(argtypes) == count, (name, len(argtypes), count)


def test_header_is_plain_c_with_the_binding_layouts(tmp_path):
    """The boundary header compiles as strict C99, and its structs have the
    sizes and field offsets the ctypes binding uses."""
    from qmbed_b200._lib import EigshHintC, EigshInfoC, EigshOptionsC
    fields = {"qmbed_eigsh_options": EigshOptionsC, "qmbed_eigsh_info": EigshInfoC, "qmbed_eigsh_hint": EigshHintC}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "qmbed_b200.h"', "int main(void) {"]
    for struct, binding in fields.items():
        lines.append(f'  printf("{struct} %zu\\n", sizeof({struct}));')
        for name, _ in binding._fields_:
            lines.append(f'  printf("{struct}.{name} %zu\\n", offsetof({struct}, {name}));')
    lines += ["  return 0;", "}"]
    source = tmp_path / "layout.c"
    source.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"),
                    "-o", str(exe), str(source)], check=True, capture_output=True, text=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                              text=True).stdout.split("\n") if line)
    for struct, binding in fields.items():
        assert int(out[struct]) == ctypes.sizeof(binding), struct
        for name, _ in binding._fields_:
            assert int(out[f"{struct}.{name}"]) == getattr(binding, name).offset, (struct, name)
