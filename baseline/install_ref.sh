#!/usr/bin/env bash
# Installs the reference's Python package (warpsymbolic, unmodified) into baseline/_ref, which is
# git-ignored but travels to the GPU box with the rest of the working tree.  The engine tests and
# `bench.py --config c1` import the reference's estimator and engine from there and resolve its
# native module `rpn_cuda_native` to this library's drop-in (or to the reference extension built
# by oracle/build_ref.sh).
#
# Offline: the wheelhouse holds the build backend; the package's own dependencies (numpy, pandas,
# scipy, scikit-learn, sympy, torch) are already installed in the interpreter, hence --no-deps.
# The build writes into its source tree, so it runs on a copy.
#
# Usage: baseline/install_ref.sh REFERENCE_ROOT      (the reference checkout)
set -euo pipefail
REF_ROOT="${1:?usage: baseline/install_ref.sh REFERENCE_ROOT}"
HERE="$(cd "$(dirname "$0")" && pwd)"
PY=${PYTHON:-python}
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
cp -r "$REF_ROOT" "$TMP/src"
rm -rf "$HERE/_ref"
"$PY" -m pip install --no-index --no-build-isolation --find-links /opt/wheelhouse --no-deps \
    --target "$HERE/_ref" "$TMP/src"
echo "[install_ref] reference package installed in $HERE/_ref"
