#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure) as oracle/libsamos_oracle.so.
# Strict IEEE: no fast-math and no FMA contraction, so the oracle's arithmetic
# follows the reference's source order term by term.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
gcc -std=c11 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math \
    -o "$here/libsamos_oracle.so" "$here/samos_oracle.c" -lm
