#!/usr/bin/env bash
# Builds the C restatement oracle (test infrastructure) into oracle/_lib/liblbfs_oracle.so.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$HERE/_lib"
# build under a private name, then rename: processes that build at the same time never load a half-written file
TMP="$HERE/_lib/liblbfs_oracle.so.$$"
gcc -std=c11 -O2 -ffp-contract=off -fPIC -shared -Wall -Wno-unused-function -I"$HERE/../include" \
    "$HERE/lbfs_oracle.c" -o "$TMP" -lm
mv -f "$TMP" "$HERE/_lib/liblbfs_oracle.so"
echo "built $HERE/_lib/liblbfs_oracle.so"
