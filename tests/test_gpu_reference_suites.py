"""The reference's own Python test files, unmodified, against libqmbed_b200.so.

baseline/install_reference.sh installs the reference's pure-Python frontends
into baseline/_ref and copies these files beside them:

* compat/test_Lanczos.py, compat/test_expm_multiply_parallel.py — the QuSpin
  1.0.1 compatibility tests of the eigsh / Lanczos / exponential-action path
  (bindings/python/compat_tests/quspin-1.0.1/test);
* native/test_qmbed.py — the native frontend's suite (bindings/python/tests).

Each file runs in its own pytest process with QMBED_LIBRARY_PATH naming this
library, so every numeric call of the reference frontend goes through the
GPU engine. The compatibility files must pass whole. test_qmbed.py also
covers families this library leaves to the reference (fermion and photon
bases, archives, Floquet and density workflows), which answer "unsupported
backend"; the tests of the eigsh / expm / evolution / sector-shift path
listed in NATIVE_IN_SCOPE must pass, and the outcome and failure reason of
every test is printed. The tests skip when baseline/_ref is absent.
"""

import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
FRONTEND = ROOT / "baseline" / "_ref"
SUITES = FRONTEND / "reference_tests"
LIBRARY = ROOT / "qmbed_b200" / "libqmbed_b200.so"

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not SUITES.is_dir(), reason="reference suites not installed (baseline/install_reference.sh)"),
]

# test_qmbed.py tests on this library's path (eigsh, exponential action,
# evolution, thermal Lanczos, sector shifts on spin chains)
NATIVE_IN_SCOPE = [
    "test_native_and_compatibility_paths_share_the_rust_solver",
    "test_quspin_static_adapter",
    "test_quspin_hamiltonian_reuses_and_releases_one_native_model",
    "test_reusable_nonnormal_exponential_action_supports_column_batches",
    "test_sector_shift_runs_directly_between_persistent_models",
    "test_static_hamiltonian_evolution_uses_the_registered_rust_model",
    "test_basis_dynamic_hamiltonian_groups_equal_drives_in_rust",
]


def _run(path: Path):
    env = dict(os.environ)
    env["QMBED_LIBRARY_PATH"] = str(LIBRARY)
    env["PYTHONPATH"] = os.pathsep.join([str(FRONTEND), env.get("PYTHONPATH", "")])
    proc = subprocess.run([sys.executable, "-m", "pytest", str(path), "-q", "-rA", "-p", "no:cacheprovider",
                           "--rootdir", str(path.parent)],
                          cwd=path.parent, env=env, capture_output=True, text=True, timeout=1800)
    outcomes = {}
    for line in proc.stdout.splitlines():
        m = re.match(r"^(PASSED|FAILED|ERROR|SKIPPED)\s+\S*::(?:\S+::)?(\S+)", line)
        if m:
            outcomes[m.group(2)] = m.group(1)
    return proc, outcomes


@pytest.mark.parametrize("name", ["test_Lanczos.py", "test_expm_multiply_parallel.py"])
def test_compat_suite_passes_verbatim(name):
    proc, outcomes = _run(SUITES / "compat" / name)
    print(proc.stdout[-3000:])
    assert proc.returncode == 0, proc.stdout[-3000:] + proc.stderr[-2000:]
    assert outcomes and all(v == "PASSED" for v in outcomes.values())


def test_native_suite_in_scope_tests_pass_verbatim():
    proc, outcomes = _run(SUITES / "native" / "test_qmbed.py")
    for name, outcome in sorted(outcomes.items()):
        print(f"{outcome:7s} {name}")
    # the reason of every failure, as pytest's short summary gives it
    for line in proc.stdout.splitlines():
        if line.startswith("FAILED"):
            print(line[:400])
    assert outcomes, proc.stdout[-3000:] + proc.stderr[-2000:]
    missing = [t for t in NATIVE_IN_SCOPE if outcomes.get(t) != "PASSED"]
    assert not missing, (missing, proc.stdout[-4000:])
