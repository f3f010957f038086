#!/usr/bin/env bash
# Builds the CPU oracle restatement (oracle/shape_oracle.c) into
# oracle/liboracle.so. Test infrastructure only. -ffp-contract=off and no
# -march: FP64 results must not depend on FMA contraction.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
${CC:-gcc} -O2 -ffp-contract=off -fPIC -shared -Wall -Wextra -Wno-unused-parameter \
    -o "$HERE/liboracle.so" "$HERE/shape_oracle.c" -lm
echo "built $HERE/liboracle.so"
