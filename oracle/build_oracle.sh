#!/usr/bin/env bash
# Builds the C restatement oracle (test infrastructure) into oracle/_lib/liblbfs_oracle.so.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$HERE/_lib"
gcc -std=c11 -O2 -ffp-contract=off -fPIC -shared -Wall -Wno-unused-function -I"$HERE/../include" \
    "$HERE/lbfs_oracle.c" -o "$HERE/_lib/liblbfs_oracle.so" -lm
echo "built $HERE/_lib/liblbfs_oracle.so"
