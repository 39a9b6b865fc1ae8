/*
 * Test infrastructure only (part of the oracle's checker, never the product).
 *
 * Minimal stand-ins for the parts of bfam's base layer (bfam.h:13-326) that
 * the reference's setup-numerics code needs, so that the reference's own
 * Jacobi/LGL (src/bfam.c:2681-3135), dense linear algebra
 * (src/bfam.c:1074-1306), interpolator (src/bfam.c:3835-3868,
 * src/bfam.c:5424-5691) and PCG32 (src/bfam.c:8334-8386) functions can be
 * compiled where they lie, without p4est, MPI or the rest of bfam.
 *
 * oracle/build_ref.sh concatenates this prelude, those line ranges of the
 * reference (extracted into oracle/_ref/, which is never committed) and
 * oracle/ref_ops_driver.c into one translation unit.
 */
#ifndef BFAM_REF_PRELUDE_H
#define BFAM_REF_PRELUDE_H

#include <float.h>
#include <inttypes.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BFAM_APPEND(x, y) x##y
#define BFAM_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define BFAM_MAX(a, b) (((a) > (b)) ? (a) : (b))
#define BFAM_NOOP()                                                            \
  do                                                                           \
  {                                                                            \
  } while (0)

static void ref_abort(const char *file, int line, const char *msg)
{
  fprintf(stderr, "reference-ops abort at %s:%d: %s\n", file, line, msg);
  abort();
}
#define BFAM_ABORT(...) ref_abort(__FILE__, __LINE__, "abort")
#define BFAM_ABORT_IF(q, ...) ((q) ? BFAM_ABORT(__VA_ARGS__) : (void)0)
#define BFAM_ABORT_IF_NOT(q, ...) BFAM_ABORT_IF(!(q), __VA_ARGS__)
#define BFAM_ASSERT(expression) BFAM_ABORT_IF_NOT((expression), "assert")
#define BFAM_ASSUME_ALIGNED(lvalueptr, align) BFAM_NOOP()
#define BFAM_VERBOSE(...) BFAM_NOOP()
#define BFAM_INFO(...) BFAM_NOOP()
#define BFAM_BUFSIZ 256

/* setup type: plain double (BFAM_USE_LONG_DOUBLE off, the reference default) */
typedef double bfam_long_real_t;
#define BFAM_LONG_REAL(x) x
#define BFAM_LONG_REAL_ABS fabs
#define BFAM_LONG_REAL_ATAN atan
#define BFAM_LONG_REAL_COS cos
#define BFAM_LONG_REAL_LGAMMA lgamma
#define BFAM_LONG_REAL_LOG log
#define BFAM_LONG_REAL_EXP exp
#define BFAM_LONG_REAL_SQRT sqrt
#define BFAM_LONG_REAL_SIN sin
#define BFAM_LONG_REAL_TAN tan
#define BFAM_LONG_REAL_EPS DBL_EPSILON
#define BFAM_LONG_REAL_PI (4 * BFAM_LONG_REAL_ATAN(1))
#define BFAM_APPROX_EQ(x, y, K, abs, eps, min)                                 \
  ((abs)((x) - (y)) < (min) + (K) * (eps)*BFAM_MAX((abs)((x)), (abs)((y))))
#define BFAM_LONG_REAL_APPROX_EQ(x, y, K)                                      \
  BFAM_APPROX_EQ((x), (y), (K), BFAM_LONG_REAL_ABS, BFAM_LONG_REAL_EPS,        \
                 BFAM_LONG_REAL_EPS *BFAM_LONG_REAL_EPS)

typedef double bfam_real_t;
typedef int32_t bfam_locidx_t;

typedef struct
{
  uint64_t state;
  uint64_t inc;
} bfam_pcg32_random_t;

static void *bfam_malloc(size_t size)
{
  void *p = malloc(size ? size : 1);
  if (!p)
    abort();
  return p;
}
static void *bfam_malloc_aligned(size_t size)
{
  void *p = NULL;
  if (posix_memalign(&p, 64, size ? size : 64))
    abort();
  return p;
}
static void bfam_free_aligned(void *p) { free(p); }

#endif
