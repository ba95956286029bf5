#!/usr/bin/env bash
# Install the reference NFGS package (nfgs_solver + nfgs) into baseline/_ref,
# the location bench.py's reference arm and its reference_torch_cuda leg
# import it from.  Offline: no index, no build isolation, no dependency
# resolution (numpy, torch and scipy of this image serve it).  The build
# writes into its source tree, so it runs from a copy under /tmp.
set -euo pipefail
REF="${NFGS_REFERENCE:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
TMP="$(mktemp -d /tmp/nfgs_ref_src.XXXXXX)"
cp -r "$REF/nfgs" "$REF/nfgs_solver.py" "$REF/pyproject.toml" "$REF/README.md" "$REF/LICENSE" "$TMP/"
python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
    --target "$HERE/_ref" "$TMP"
rm -rf "$TMP"
echo "installed into $HERE/_ref"
