#!/usr/bin/env bash
# Test infrastructure only: builds oracle/_ref/libbfam_ref_ops.so, the
# reference's own setup numerics compiled from its source where it lies.
#
# The reference is one amalgamated C file whose full build needs p4est's
# autotools build, MPI and generated config headers, so the whole library is
# not built here.  The hot path's setup numerics are self-contained static
# functions, so this recipe takes exactly these line ranges of
# src/bfam.c, concatenated behind oracle/ref_prelude.h (stand-ins for the
# base layer) and in front of oracle/ref_ops_driver.c (exported wrappers):
#   1074-1306  dense linear algebra (transpose, mmmult, LU, back/forwardslash)
#   2681-3135  Jacobi polynomials, Gauss / Gauss-Lobatto quadrature, V, D, M
#   3835-3868  bfam_subdomain_dgx_interpolator_t
#   5424-5691  init_interpolator .. create_interpolators (mortar operators)
#   8334-8386  PCG32
# Each range is checked against its first line before use.  Output goes only
# to oracle/_ref/ (git-ignored); nothing from the reference is committed.
set -euo pipefail
REF=${BFAM_REFERENCE_DIR:-/root/reference}
SRC="$REF/src/bfam.c"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
  echo "build_ref.sh: $SRC not found; skipping (prebuilt oracle/_ref is used if present)" >&2
  exit 0
fi
mkdir -p "$OUT"

check() { # line expected-prefix
  local got
  got=$(sed -n "${1}p" "$SRC")
  case "$got" in
    "$2"*) ;;
    *) echo "build_ref.sh: line $1 of $SRC is '$got', expected '$2...'" >&2; exit 1 ;;
  esac
}
check 1074 "// {{{ utilities"
check 1306 "}"
check 2681 "// {{{ jacobi"
check 3135 "// }}}"
check 3835 "typedef struct"
check 3868 "} bfam_subdomain_dgx_interpolator_t;"
check 5424 "static void init_interpolator"
check 5691 "}"
check 8334 "static uint32_t bfam_pcg32_random_r"
check 8386 "}"

TU="$OUT/ref_ops_tu.c"
{
  echo '#include "ref_prelude.h"'
  for r in 1074,1306 2681,3135 3835,3868 5424,5691 8334,8386; do
    echo "#line ${r%,*} \"$SRC\""
    sed -n "${r}p" "$SRC"
  done
  echo "#line 1 \"$HERE/ref_ops_driver.c\""
  cat "$HERE/ref_ops_driver.c"
} > "$TU"

gcc -std=gnu99 -O2 -fPIC -shared -I"$HERE" -Wno-unused-function \
  -o "$OUT/libbfam_ref_ops.so" "$TU" -lm
echo "built $OUT/libbfam_ref_ops.so"
