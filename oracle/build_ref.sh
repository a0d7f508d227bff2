#!/bin/sh
# Compiles the reference's own Hogbom CLEAN sources (hclean.cpp + bindings.cpp,
# read in place from the reference tree) into oracle/_ref/, as the reference's
# CMake build would (-O3, C++17, pybind11 module _hogbom_ext).  Used only as a
# checker and as the CPU baseline for CLEAN.  Needs the reference tree, so it
# runs in the build container; the built module travels with the repository.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: $AV_REFERENCE_ROOT, else reference/ beside this repository
REF=${AV_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}
HB=$REF/src/astroviper/core/imaging/deconvolvers/hogbom
[ -f "$HB/src/hclean.cpp" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$HERE/_ref"
EXT=$(python3 -c "import sysconfig; print(sysconfig.get_config_var('EXT_SUFFIX'))")
EXTRA=""
case "$(uname -m)" in aarch64|arm64) EXTRA="-ffp-contract=off";; esac
g++ -O3 -pipe -fPIC -DNDEBUG -shared -std=c++17 $EXTRA $(python3 -m pybind11 --includes) \
    -I"$HB/include" "$HB/src/hclean.cpp" "$HB/python/bindings.cpp" \
    -o "$HERE/_ref/_hogbom_ext$EXT"
echo "built $HERE/_ref/_hogbom_ext$EXT"
