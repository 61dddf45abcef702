#!/usr/bin/env bash
# Builds the UNMODIFIED reference CPU hot path into oracle/_ref/libptref.so (test infrastructure only).
#
# Compiles the reference sources where they lie (nothing is copied into this repository) with the
# reference's strict floating-point setting (-ffp-contract=off, CMakeLists.txt:7-12), plus oracle/ref_shim.cpp.
# Output goes only to oracle/_ref/ (git-ignored; it still travels with the working tree to a GPU host).
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default: $PTB_REFERENCE_ROOT, else /root/reference)
# The root it built from is recorded in oracle/_ref/reference_root.txt for the tests that read reference fixtures.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${PTB_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/lib" ]; then
	echo "reference tree not found at $REF; keeping any prebuilt $OUT/libptref.so" >&2
	exit 0
fi
mkdir -p "$OUT"
SRCS=(
	"$REF/lib/Palm.cpp"
	"$REF/lib/localization/ATrous.cpp"
	"$REF/lib/localization/FrameProcessor.cpp"
	"$REF/lib/localization/Segmentation2D.cpp"
	"$REF/lib/fit/Fitting.cpp"
	"$REF/lib/fit/GaussianFit.cpp"
	"$REF/lib/fit/GaussianModel.cpp"
	"$REF/lib/fit/SplineFit.cpp"
	"$REF/lib/fit/AstigFit.cpp"
	"$REF/lib/signal_processing/Matrix.cpp"
	"$REF/lib/tracking/Tracks.cpp"
	"$HERE/ref_shim.cpp"
)
g++ -std=c++20 -O2 -fopenmp -ffp-contract=off -fPIC -shared \
	-I"$REF/lib" -I"$REF/lib/localization" -I"$REF/lib/fit" -I"$REF/lib/signal_processing" -I"$REF/lib/tracking" \
	"${SRCS[@]}" -o "$OUT/libptref.so.tmp"
mv "$OUT/libptref.so.tmp" "$OUT/libptref.so"
(cd "$REF" && pwd) > "$OUT/reference_root.txt"
echo "built $OUT/libptref.so"
