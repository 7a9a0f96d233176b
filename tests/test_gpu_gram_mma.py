"""The dense contractions on the FP64 tensor cores (m8n8k4 DMMA): the filtered
solver's block Gram and the Krylov Ritz combinations, against the CUDA-core
kernels they replaced (QMBED_DENSE=scalar), on the same solves: eigenvalues within 1e-12 relative of each other, and both within
1e-10 of the oracle where the oracle runs (L=18)."""

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
from qmbed_b200 import GpuBasis, GpuOperator
from qmbed_b200.engine import heisenberg_terms
out = {{}}
for sites, k, storage, mode, krylov in ((18, 4, "packed", "filtered", None), (24, 6, "packed", "filtered", None),
                                        (22, 12, "matrix_free", "filtered", None), (18, 4, "packed", "fp64", 40),
                                        (22, 3, "packed", "mixed", 24)):
    op = GpuOperator(GpuBasis(sites, up=sites // 2, momentum=0, parity=1), heisenberg_terms(sites, delta=1.1),
                     storage=storage)
    r = op.eigsh(k, tolerance=1e-10, seed=5, mode=mode, krylov_dimension=krylov)
    out[f"{{sites}}-{{k}}-{{mode}}"] = {{"values": r.eigenvalues.tolist(), "iterations": r.iterations,
                                        "residuals": r.residuals.tolist()}}
print(json.dumps(out))
"""


def _solve(gram):
    env = dict(os.environ)
    if gram:
        env["QMBED_DENSE"] = gram
    else:
        env.pop("QMBED_DENSE", None)
    proc = subprocess.run([sys.executable, "-c", SCRIPT.format(root=str(ROOT))], env=env, capture_output=True,
                          text=True, timeout=900)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return json.loads(proc.stdout.strip().splitlines()[-1])


def test_tensor_core_gram_matches_the_cuda_core_gram(oracle):
    mma, scalar = _solve(None), _solve("scalar")
    for key in mma:
        a, b = np.asarray(mma[key]["values"]), np.asarray(scalar[key]["values"])
        assert np.max(np.abs(a - b) / np.abs(b)) <= 1e-12, key
        assert np.all(np.asarray(mma[key]["residuals"]) <= 1e-10 * np.maximum(np.abs(a), 1.0))
    ref = oracle.Operator.build(oracle.Basis(18, up=9, momentum=0, parity=1),
                                oracle.heisenberg_terms(18, delta=1.1)).eigsh(4, tolerance=1e-12, seed=5)
    for key in ("18-4-filtered", "18-4-fp64"):
        got = np.asarray(mma[key]["values"])
        assert np.max(np.abs(got - ref.eigenvalues) / np.abs(ref.eigenvalues)) <= 1e-10, key
