#!/bin/sh
# Offline install of the reference's pure-Python frontends (qmbed and its
# QuSpin-compatible quspin package) into baseline/_ref, plus copies of the
# reference's own Python test files that tests/test_gpu_reference_suites.py
# runs unmodified against libqmbed_b200.so. baseline/_ref is git-ignored and
# travels with the working tree to the GPU box. The Rust extension of the
# reference is not built (no cargo here); the frontend loads the library
# named by QMBED_LIBRARY_PATH instead.
#
#   sh baseline/install_reference.sh <reference checkout>
set -e
REF=${1:?usage: sh baseline/install_reference.sh <reference checkout>}
HERE=$(cd "$(dirname "$0")" && pwd)
TMP=$(mktemp -d)
cp -r "$REF/bindings/python" "$TMP/python"
python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
    --target "$HERE/_ref" "$TMP/python"
mkdir -p "$HERE/_ref/reference_tests/compat" "$HERE/_ref/reference_tests/native"
cp "$REF/bindings/python/compat_tests/quspin-1.0.1/test/test_Lanczos.py" \
   "$REF/bindings/python/compat_tests/quspin-1.0.1/test/test_expm_multiply_parallel.py" \
   "$HERE/_ref/reference_tests/compat/"
cp "$REF/bindings/python/tests/test_qmbed.py" "$HERE/_ref/reference_tests/native/"
rm -rf "$TMP"
