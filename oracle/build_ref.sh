#!/usr/bin/env bash
# Test infrastructure only.  Compiles the reference from its own sources, with
# gcc directly (the reference's Makefile and p4est's autotools build are not
# run), into oracle/_ref/ (git-ignored; nothing from the reference is
# committed).  Set BFAM_REFERENCE_DIR to the reference checkout (the
# directory holding src/bfam.c and third_party/p4est-1.1.tar.gz).
#
# 1. libbfam_ref_ops.so: the hot path's setup numerics, which are
#    self-contained static functions, taken as these line ranges of
#    src/bfam.c, concatenated behind oracle/ref_prelude.h (stand-ins for the
#    base layer) and in front of oracle/ref_ops_driver.c (exported wrappers):
#      1074-1306  dense linear algebra (transpose, mmmult, LU, back/forwardslash)
#      2681-3135  Jacobi polynomials, Gauss / Gauss-Lobatto quadrature, V, D, M
#      3835-3868  bfam_subdomain_dgx_interpolator_t
#      5424-5691  init_interpolator .. create_interpolators (mortar operators)
#      8334-8386  PCG32
#    Each range is checked against its first line before use.
# 2. libbfam_ref2d.so / libbfam_ref3d.so: the whole of src/bfam.c (once per
#    dimension) with the vendored p4est-1.1 and libsc built serially from
#    third_party/p4est-1.1.tar.gz (config headers oracle/ref_cfg/*.h written
#    for this recipe; <mpi.h> mapped to libsc's serial sc_MPI_* by
#    oracle/ref_cfg/mpi.h), plus oracle/bfam_split_driver.c, which runs
#    bfam's brick -> refine -> balance -> split front end and returns the
#    arrays bfam holds.
# 3. bfam_adapter_test{2,3}d: tests/c/bfam_adapter_test.c, a C program
#    compiled against the reference's src/bfam.h and include/bfam_gpu_bfam.h
#    (the adapter from bfam's objects to the bfam_gpu C-ABI), linked with
#    libbfam_ref{2,3}d.so and bfam_b200/libbfam_b200.so.  Built only when the
#    product library exists.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/.." && pwd)"
OUT="$HERE/_ref"
if [ -z "${BFAM_REFERENCE_DIR:-}" ]; then
  echo "build_ref.sh: set BFAM_REFERENCE_DIR to the reference checkout" \
       "(src/bfam.c, third_party/p4est-1.1.tar.gz)" >&2
  exit 2
fi
REF="$BFAM_REFERENCE_DIR"
SRC="$REF/src/bfam.c"
if [ ! -f "$SRC" ]; then
  echo "build_ref.sh: $SRC not found" >&2
  exit 2
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

# ---------------------------------------------------------------- 1. ops
if [ ! -f "$OUT/libbfam_ref_ops.so" ] || [ "$SRC" -nt "$OUT/libbfam_ref_ops.so" ] ||
   [ "$HERE/ref_ops_driver.c" -nt "$OUT/libbfam_ref_ops.so" ] ||
   [ "$HERE/ref_prelude.h" -nt "$OUT/libbfam_ref_ops.so" ]; then
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
fi

# ------------------------------------------------- 2. p4est + whole bfam.c
TAR="$REF/third_party/p4est-1.1.tar.gz"
P4="$OUT/build/p4est-1.1"
P4LIB="$OUT/build/libp4est_serial.a"
if [ ! -f "$P4LIB" ]; then
  rm -rf "$OUT/build"
  mkdir -p "$OUT/build/obj"
  tar xzf "$TAR" -C "$OUT/build"
  INC=(-I"$HERE/ref_cfg" -I"$P4/sc/src" -I"$P4/sc/src/sc_builtin"
       -I"$P4/sc/libb64" -I"$P4/sc/iniparser" -I"$P4/src")
  pids=()
  for f in "$P4"/sc/src/*.c "$P4"/sc/libb64/*.c "$P4"/sc/iniparser/*.c "$P4"/src/*.c; do
    b=$(basename "$f" .c)
    gcc -std=gnu99 -O2 -fPIC -w "${INC[@]}" -c "$f" -o "$OUT/build/obj/$b.o" &
    pids+=($!)
  done
  for p in "${pids[@]}"; do wait "$p"; done
  ar rcs "$P4LIB" "$OUT"/build/obj/*.o
  echo "built $P4LIB"
fi
INC=(-I"$HERE/ref_cfg" -I"$P4/sc/src" -I"$P4/sc/src/sc_builtin" -I"$P4/src"
     -I"$REF/src")
for d in 2 3; do
  LIBD="$OUT/libbfam_ref${d}d.so"
  if [ ! -f "$LIBD" ] || [ "$SRC" -nt "$LIBD" ] ||
     [ "$HERE/bfam_split_driver.c" -nt "$LIBD" ] ||
     [ "$HERE/bfam_split_driver.h" -nt "$LIBD" ]; then
    gcc -std=gnu99 -O2 -fPIC -w -DBFAM_DEBUG -DBFAM_DGX_DIMENSION=$d "${INC[@]}" \
      -c "$SRC" -o "$OUT/build/bfam${d}d.o"
    gcc -std=gnu99 -O2 -fPIC -Wall -Wno-unused-function -DBFAM_DEBUG \
      -DBFAM_DGX_DIMENSION=$d "${INC[@]}" \
      -I"$HERE" -c "$HERE/bfam_split_driver.c" -o "$OUT/build/driver${d}d.o"
    gcc -shared -Wl,-Bsymbolic -o "$LIBD" "$OUT/build/bfam${d}d.o" \
      "$OUT/build/driver${d}d.o" "$P4LIB" -lm
    echo "built $LIBD"
  fi
done

# ------------------------------------------------ 3. the C adapter test
PROD="$ROOT/bfam_b200/libbfam_b200.so"
TEST_SRC="$ROOT/tests/c/bfam_adapter_test.c"
if [ -f "$PROD" ] && [ -f "$TEST_SRC" ]; then
  for d in 2 3; do
    EXE="$OUT/bfam_adapter_test${d}d"
    if [ ! -f "$EXE" ] || [ "$TEST_SRC" -nt "$EXE" ] ||
       [ "$ROOT/include/bfam_gpu_bfam.h" -nt "$EXE" ] ||
       [ "$ROOT/include/bfam_gpu.h" -nt "$EXE" ] ||
       [ "$OUT/libbfam_ref${d}d.so" -nt "$EXE" ] ||
       [ "$PROD" -nt "$EXE" ]; then
      gcc -std=gnu99 -O2 -Wall -Wno-unused-function -DBFAM_DGX_DIMENSION=$d \
        "${INC[@]}" -I"$ROOT/include" -I"$HERE" -o "$EXE" "$TEST_SRC" \
        -L"$OUT" -L"$ROOT/bfam_b200" -lbfam_ref${d}d -lbfam_b200 -lm \
        -Wl,-rpath,'$ORIGIN' -Wl,-rpath,'$ORIGIN/../../bfam_b200'
      echo "built $EXE"
    fi
  done
fi
