#!/bin/sh
# Build the reference omi_physics (Python + its two Cython accelerators) from
# its own sources into oracle/_ref, for the golden-fixture generator and the
# CPU reference arm of bench.py. pip writes build files into the source tree,
# so it installs from a scratch copy; outputs land only in oracle/_ref.
#   usage: sh oracle/build_ref.sh [/path/to/reference]
# Without an argument: $OMI_REFERENCE_SRC, else a 'reference' folder beside the repository.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
SRC=${1:-${OMI_REFERENCE_SRC:-$(cd "$HERE/../.." && pwd)/reference}}
TMP=$(mktemp -d /tmp/omi_ref_src.XXXXXX)
cp -r "$SRC"/. "$TMP"/
chmod -R u+w "$TMP"
rm -rf "$HERE/_ref"
python -m pip install --no-index --no-build-isolation --no-deps --target "$HERE/_ref" "$TMP"
rm -rf "$TMP"
python -c "import sys; sys.path.insert(0, '$HERE/_ref'); import omi_physics._solver_native, omi_physics._collide_native; print('reference accelerators built')"
