#!/usr/bin/env bash
# Builds the oracle restatement (oracle/pt_oracle.cpp) into oracle/liboracle.so (test infrastructure only).
# Same strict floating-point setting as the reference (-ffp-contract=off): every FP64 step stays unfused.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
g++ -std=c++20 -O2 -fopenmp -ffp-contract=off -fPIC -shared -Wall -Wextra \
	"$HERE/pt_oracle.cpp" -o "$HERE/liboracle.so.tmp"
mv "$HERE/liboracle.so.tmp" "$HERE/liboracle.so"
echo "built $HERE/liboracle.so"
