/*
 * Host setup numerics: PCG32, Legendre-Gauss-Lobatto operators, mortar
 * interpolation / L2-projection operators and LSRK coefficient tables.
 *
 * The LGL construction follows the reference's steps so that the operators
 * agree with bfam's bit for bit (checked by the test-suite against the
 * reference compiled from source):
 *  - orthonormal Jacobi polynomials by the three-term recurrence of Szego
 *    (4.5.1) and the normalisation h_N^{-1/2} (src/bfam.c:2700-2829);
 *  - Gauss-Jacobi nodes by Newton's method in theta = acos(x) started from
 *    the Gatteschi-Pittaluga approximation (Hale & Townsend, SISC 35 (2013)
 *    eq. 3.19), weights from p'_{N+1} (src/bfam.c:2832-3011);
 *  - Gauss-Lobatto = {-1, interior Gauss-Jacobi(alpha+1, beta+1), +1}
 *    (src/bfam.c:3013-3040);
 *  - V, D = Vr V^{-1} via LU with complete pivoting (Golub & van Loan,
 *    Algorithms 3.4.2, 3.1.3, 3.1.4; src/bfam.c:1117-1306, 3042-3108);
 *  - exact mass M = V^{-T} V^{-1} (src/bfam.c:3110-3133).
 */
#include "bfam_b200_host.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ PCG32 */

uint32_t bfam_b200_pcg32_next(bfam_b200_pcg32_t *rng)
{
  const uint64_t old = rng->state;
  rng->state = old * 6364136223846793005ULL + (rng->inc | 1u);
  const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = (uint32_t)(old >> 59u);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

void bfam_b200_pcg32_seed(bfam_b200_pcg32_t *rng, uint64_t initstate,
                          uint64_t initseq)
{
  rng->state = 0u;
  rng->inc = (initseq << 1u) | 1u;
  (void)bfam_b200_pcg32_next(rng);
  rng->state += initstate;
  (void)bfam_b200_pcg32_next(rng);
}

uint32_t bfam_b200_pcg32_bounded(bfam_b200_pcg32_t *rng, uint32_t bound)
{
  const uint32_t threshold = (uint32_t)(0u - bound) % bound;
  for (;;)
  {
    const uint32_t v = bfam_b200_pcg32_next(rng);
    if (v >= threshold)
      return v % bound;
  }
}

double bfam_b200_pcg32_uniform(bfam_b200_pcg32_t *rng)
{
  return (double)bfam_b200_pcg32_next(rng) * (1.0 / 4294967296.0);
}

/* ----------------------------------------------------- small dense algebra */

/* column-major helpers; C += op(A) op(B) with the loop order i, j, p so the
 * rounding matches the reference */
static void mat_transpose(size_t m, size_t n, const double *A, size_t lda,
                          double *B, size_t ldb)
{
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < n; ++j)
      B[i * ldb + j] = A[j * lda + i];
}

/* C (m x n) += A^T B, A is k x m, B is k x n */
static void mat_tmul(size_t m, size_t n, size_t k, const double *A, size_t lda,
                     const double *B, size_t ldb, double *C, size_t ldc)
{
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < n; ++j)
      for (size_t p = 0; p < k; ++p)
        C[j * ldc + i] += A[i * lda + p] * B[j * ldb + p];
}

/* C (m x n) += A B, A is m x k, B is k x n */
static void mat_mul(size_t m, size_t n, size_t k, const double *A, size_t lda,
                    const double *B, size_t ldb, double *C, size_t ldc)
{
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < n; ++j)
      for (size_t p = 0; p < k; ++p)
        C[j * ldc + i] += A[p * lda + i] * B[j * ldb + p];
}

/* LU with complete pivoting, in place, A is n x n column-major */
static void lu_complete(size_t n, double *A, size_t *p, size_t *q)
{
  for (size_t k = 0; k < n; ++k)
    p[k] = q[k] = k;
  for (size_t k = 0; k + 1 < n; ++k)
  {
    size_t mu = k, la = k;
    double amax = 0.0;
    for (size_t j = k; j < n; ++j)
      for (size_t i = k; i < n; ++i)
      {
        const double a = fabs(A[i + n * j]);
        if (a > amax)
        {
          amax = a;
          mu = i;
          la = j;
        }
      }
    size_t t = p[k];
    p[k] = p[mu];
    p[mu] = t;
    for (size_t j = 0; j < n; ++j)
    {
      const double r = A[k + n * j];
      A[k + n * j] = A[mu + n * j];
      A[mu + n * j] = r;
    }
    t = q[k];
    q[k] = q[la];
    q[la] = t;
    for (size_t i = 0; i < n; ++i)
    {
      const double r = A[i + n * k];
      A[i + n * k] = A[i + n * la];
      A[i + n * la] = r;
    }
    if (fabs(A[k + n * k]) > DBL_EPSILON * DBL_EPSILON)
    {
      for (size_t i = k + 1; i < n; ++i)
        A[i + n * k] = A[i + n * k] / A[k + n * k];
      for (size_t i = k + 1; i < n; ++i)
        for (size_t j = k + 1; j < n; ++j)
          A[i + n * j] = A[i + n * j] - A[i + n * k] * A[k + n * j];
    }
  }
}

static void lu_apply(size_t n, const double *LU, double *x, const size_t *p,
                     const size_t *q, double *work)
{
  for (size_t k = 0; k < n; ++k)
    work[k] = x[p[k]];
  for (size_t j = 0; j + 1 < n; ++j)
    for (size_t i = j + 1; i < n; ++i)
      work[i] = work[i] - work[j] * LU[i + n * j];
  for (size_t j = n - 1; j > 0; --j)
  {
    work[j] = work[j] / LU[j + n * j];
    for (size_t i = 0; i < j; ++i)
      work[i] = work[i] - work[j] * LU[i + n * j];
  }
  work[0] = work[0] / LU[0];
  for (size_t k = 0; k < n; ++k)
    x[q[k]] = work[k];
}

/* C = A \ B, A m x m, B m x n */
static void mat_backslash(size_t m, size_t n, const double *A, const double *B,
                          double *C)
{
  double *LU = malloc(m * m * sizeof(double));
  double *work = malloc(m * sizeof(double));
  size_t *p = malloc(m * sizeof(size_t)), *q = malloc(m * sizeof(size_t));
  memcpy(LU, A, m * m * sizeof(double));
  memcpy(C, B, m * n * sizeof(double));
  lu_complete(m, LU, p, q);
  for (size_t j = 0; j < n; ++j)
    lu_apply(m, LU, C + j * m, p, q, work);
  free(q);
  free(p);
  free(work);
  free(LU);
}

/* C = A / B (C B = A), A m x n, B n x n */
static void mat_forwardslash(size_t m, size_t n, const double *A,
                             const double *B, double *C)
{
  double *AT = malloc(n * m * sizeof(double));
  double *BT = malloc(n * n * sizeof(double));
  double *CT = malloc(n * m * sizeof(double));
  mat_transpose(m, n, A, m, AT, n);
  mat_transpose(n, n, B, n, BT, n);
  mat_backslash(n, m, BT, AT, CT);
  mat_transpose(n, m, CT, n, C, m);
  free(CT);
  free(BT);
  free(AT);
}

/* ------------------------------------------------------ Jacobi polynomials */

static double jac_norm(double a, double b, int N)
{
  const double lg = -(a + b + 1) * log(2) - lgamma(N + a + 1) -
                    lgamma(N + b + 1) + log(2 * N + a + b + 1) +
                    lgamma(N + 1) + lgamma(N + a + b + 1);
  return sqrt(exp(lg));
}

/* orthonormal p_N^{(a,b)} at nx points */
static void jac_p(double a, double b, int N, size_t nx, const double *x,
                  double *P)
{
  for (size_t i = 0; i < nx; ++i)
  {
    double pm2, pm1 = 1, p0 = ((a + b + 2) / 2) * x[i] + (a - b) / 2;
    if (N == 0)
      P[i] = pm1;
    else if (N == 1)
      P[i] = p0;
    else
    {
      for (int n = 2; n < N + 1; ++n)
      {
        const double ca = (2 * n + a + b - 1) * (2 * n + a + b) /
                          (2 * n * (n + a + b));
        const double cb = (b * b - a * a) * (2 * n + a + b - 1) /
                          (2 * n * (n + a + b) * (2 * n + a + b - 2));
        const double cc = (n + a - 1) * (n + b - 1) * (2 * n + a + b) /
                          (n * (n + a + b) * (2 * n + a + b - 2));
        pm2 = pm1;
        pm1 = p0;
        p0 = (ca * x[i] - cb) * pm1 - cc * pm2;
      }
      P[i] = p0;
    }
  }
  const double s = jac_norm(a, b, N);
  for (size_t i = 0; i < nx; ++i)
    P[i] *= s;
}

static void jac_dp(double a, double b, int N, size_t nx, const double *x,
                   double *dP)
{
  if (N == 0)
  {
    for (size_t i = 0; i < nx; ++i)
      dP[i] = 0.0;
    return;
  }
  jac_p(a + 1, b + 1, N - 1, nx, x, dP);
  const double s = sqrt(N * (N + a + b + 1));
  for (size_t i = 0; i < nx; ++i)
    dP[i] *= s;
}

static int approx_eq(double x, double y)
{
  const double ax = fabs(x), ay = fabs(y);
  return fabs(x - y) <
         DBL_EPSILON * DBL_EPSILON + 10 * DBL_EPSILON * (ax > ay ? ax : ay);
}

/* half of the Gauss-Jacobi nodes (upper if half != 0); 0 on success */
static int gauss_half(double a, double b, int N, int half, double *x,
                      double *w)
{
  const int nk = half ? (((N + 1) % 2) ? (N + 1) / 2 + 1 : (N + 1) / 2)
                      : (N + 1) / 2;
  if (nk == 0)
    return 0;
  const double tworho = 2 * (N + 1) + a + b + 1;
  const double pi = 4 * atan(1);
  double *th0 = malloc(nk * sizeof(double)), *th1 = malloc(nk * sizeof(double));
  double *p0 = malloc(nk * sizeof(double)), *dp0 = malloc(nk * sizeof(double));
  for (int k = nk; k > 0; --k)
  {
    const int kh = half ? nk - k : k - 1;
    const double phik = (2 * k + a - 0.5) * pi / tworho;
    th1[kh] = phik + 1 / (tworho * tworho) *
                         ((0.25 - a * a) * 1 / tan(0.5 * phik) -
                          (0.25 - b * b) * tan(0.5 * phik));
  }
  int converged = 0;
  for (int it = 0; it < 200; ++it)
  {
    double *t = th0;
    th0 = th1;
    th1 = t;
    for (int k = 0; k < nk; ++k)
      x[k] = cos(th0[k]);
    jac_p(a, b, N + 1, nk, x, p0);
    jac_dp(a, b, N + 1, nk, x, dp0);
    for (int k = 0; k < nk; ++k)
      th1[k] = th0[k] - p0[k] / (-sin(th0[k]) * dp0[k]);
    int diff = 0;
    for (int k = 0; k < nk; ++k)
      diff += !approx_eq(th0[k], th1[k]);
    if (!diff)
    {
      converged = 1;
      break;
    }
  }
  if (converged)
  {
    for (int k = 0; k < nk; ++k)
      x[k] = cos(th1[k]);
    jac_dp(a, b, N + 1, nk, x, dp0);
    for (int k = 0; k < nk; ++k)
    {
      const double s = sin(th1[k]);
      w[k] = tworho / (s * s * dp0[k] * dp0[k]);
    }
  }
  free(th0);
  free(th1);
  free(p0);
  free(dp0);
  return converged ? 0 : -1;
}

static int gauss_jacobi(double a, double b, int N, double *x, double *w)
{
  const int nf = (N + 1) / 2;
  if (gauss_half(a, b, N, 1, x + nf, w + nf))
    return -1;
  if (gauss_half(b, a, N, 0, x, w))
    return -1;
  for (int k = 0; k < nf; ++k)
    x[k] *= -1;
  return 0;
}

static int gauss_lobatto(int N, double *x, double *w)
{
  const double a = 0, b = 0;
  x[0] = -1;
  x[N] = 1;
  if (N > 1 && gauss_jacobi(a + 1, b + 1, N - 2, x + 1, w + 1))
    return -1;
  jac_p(a, b, N, N + 1, x, w);
  const double fac = (2 * N + a + b + 1) / (N * (N + a + b + 1));
  for (int k = 0; k < N + 1; ++k)
    w[k] = fac / (w[k] * w[k]);
  w[0] *= (1 + b);
  w[N] *= (1 + a);
  return 0;
}

static void vandermonde(int N, size_t nx, const double *x, double *V)
{
  for (int j = 0; j <= N; ++j)
    jac_p(0, 0, j, nx, x, V + j * nx);
}

static void grad_vandermonde(int N, size_t nx, const double *x, double *V)
{
  for (int j = 0; j <= N; ++j)
    jac_dp(0, 0, j, nx, x, V + j * nx);
}

/* I (nx x (N+1)) interpolates from the order-N LGL basis to points x */
static void interp_matrix(int N, size_t nx, const double *x, const double *V,
                          double *I)
{
  double *Vx = malloc((N + 1) * nx * sizeof(double));
  vandermonde(N, nx, x, Vx);
  mat_forwardslash(nx, N + 1, Vx, V, I);
  free(Vx);
}

static void exact_mass(int N, const double *V, double *M)
{
  const int n = N + 1;
  double *I = calloc(n * n, sizeof(double));
  double *iV = malloc(n * n * sizeof(double));
  double *iVT = malloc(n * n * sizeof(double));
  for (int i = 0; i < n * n; ++i)
    M[i] = 0;
  for (int i = 0; i < n; ++i)
    I[n * i + i] = 1;
  mat_backslash(n, n, V, I, iV);
  mat_transpose(n, n, iV, n, iVT, n);
  mat_mul(n, n, n, iVT, n, iV, n, M, n);
  free(I);
  free(iV);
  free(iVT);
}

int bfam_b200_lgl_operators(int N, double *r, double *w, double *wi,
                            double *Dr)
{
  if (N < 1 || N > 15)
    return -1;
  const int n = N + 1;
  double *V = malloc(n * n * sizeof(double));
  double *Vr = malloc(n * n * sizeof(double));
  if (gauss_lobatto(N, r, w))
  {
    free(V);
    free(Vr);
    return -1;
  }
  vandermonde(N, n, r, V);
  grad_vandermonde(N, n, r, Vr);
  mat_forwardslash(n, n, Vr, V, Dr);
  for (int i = 0; i < n; ++i)
    wi[i] = (double)(1.0L / (long double)w[i]); /* as src/bfam.c:7125 */
  free(V);
  free(Vr);
  return 0;
}

/* ---------------------------------------------------- mortar operators */

/* I_a2g interpolates order-N_a values to the points lr_g; P_g2a is the L2
 * projection back, P = V_a V_a^T I^T M_g (src/bfam.c:5471-5514). */
static void interp_proj(int Na, int Ng, const double *Va, const double *Mg,
                        const double *lrg, double *I, double *P)
{
  const int na = Na + 1, ng = Ng + 1;
  double *MP = calloc((size_t)na * ng, sizeof(double));
  double *VtMP = calloc((size_t)na * ng, sizeof(double));
  interp_matrix(Na, ng, lrg, Va, I);
  for (int i = 0; i < na * ng; ++i)
    P[i] = 0;
  mat_tmul(na, ng, ng, I, ng, Mg, ng, MP, na);
  mat_tmul(na, ng, na, Va, na, MP, na, VtMP, na);
  mat_mul(na, ng, na, Va, na, VtMP, na, P, na);
  free(MP);
  free(VtMP);
}

typedef struct
{
  int N;
  double r[16], w[16], V[256], M[256];
} grid1d_t;

static int grid1d(int N, grid1d_t *g)
{
  g->N = N;
  if (gauss_lobatto(N, g->r, g->w))
    return -1;
  vandermonde(N, N + 1, g->r, g->V);
  exact_mass(N, g->V, g->M);
  return 0;
}

int bfam_b200_mortar_operators(int N_src, int N_dst, double *prj)
{
  if (N_src < 1 || N_dst < 1 || N_src > 15 || N_dst > 15)
    return -1;
  const int Ng = N_src > N_dst ? N_src : N_dst;
  const int na = N_src + 1, nb = N_dst + 1, ng = Ng + 1;
  grid1d_t ga, gb, gg;
  if (grid1d(N_src, &ga) || grid1d(N_dst, &gb) || grid1d(Ng, &gg))
    return -1;

  /* operators on the glue space: 1 P_b2f, 2 P_t2f, 3 I_f2b, 4 I_f2t
   * (src/bfam.c:5516-5541) */
  double *pg[5] = {NULL};
  for (int k = 1; k < 5; ++k)
    pg[k] = malloc((size_t)ng * ng * sizeof(double));
  {
    double lrt[16], lrb[16], Mh[256];
    for (int k = 0; k < ng; ++k)
    {
      lrt[k] = 0.5 * (gg.r[k] + 1);
      lrb[k] = 0.5 * (gg.r[k] - 1);
    }
    for (int k = 0; k < ng * ng; ++k)
      Mh[k] = 0.5 * gg.M[k];
    interp_proj(Ng, Ng, gg.V, Mh, lrt, pg[4], pg[2]);
    interp_proj(Ng, Ng, gg.V, Mh, lrb, pg[3], pg[1]);
  }

  double *I_a2g = NULL, *P_g2b = NULL;
  if (N_src < Ng && N_dst == Ng)
  {
    I_a2g = malloc((size_t)ng * na * sizeof(double));
    double *junk = malloc((size_t)ng * na * sizeof(double));
    interp_proj(N_src, Ng, ga.V, gg.M, gg.r, I_a2g, junk);
    free(junk);
  }
  if (N_src == Ng && N_dst < Ng)
  {
    double *junk = malloc((size_t)ng * nb * sizeof(double));
    P_g2b = malloc((size_t)ng * nb * sizeof(double));
    interp_proj(N_dst, Ng, gb.V, gg.M, gg.r, junk, P_g2b);
    free(junk);
  }

  /* src/bfam.c:5543-5604: prj[k] = P_g2b * pg[k] * I_a2g, missing factors
   * are identities */
  for (int k = 0; k < 5; ++k)
  {
    double *out = prj + (size_t)k * nb * na;
    double *tmp = calloc((size_t)nb * na, sizeof(double));
    const double *lP = NULL;
    if (!P_g2b && pg[k] && I_a2g)
    {
      mat_mul(nb, na, ng, pg[k], nb, I_a2g, ng, tmp, nb);
      lP = tmp;
    }
    else if (P_g2b && pg[k] && !I_a2g)
    {
      mat_mul(nb, na, ng, P_g2b, nb, pg[k], ng, tmp, nb);
      lP = tmp;
    }
    else if (!P_g2b && !pg[k] && I_a2g)
      lP = I_a2g;
    else if (!P_g2b && pg[k] && !I_a2g)
      lP = pg[k];
    else if (P_g2b && !pg[k] && !I_a2g)
      lP = P_g2b;
    if (lP)
      memcpy(out, lP, (size_t)nb * na * sizeof(double));
    else
      for (int i = 0; i < nb * na; ++i)
        out[i] = ((i % (nb + 1)) == 0) ? 1.0 : 0.0;
    free(tmp);
  }
  for (int k = 1; k < 5; ++k)
    free(pg[k]);
  free(I_a2g);
  free(P_g2b);
  return 0;
}

/* -------------------------------------------------------------- LSRK */

int bfam_b200_lsrk_coefficients(int method, double *A, double *B, double *C)
{
  switch (method)
  {
  case BFAM_B200_LSRK_KC54:
    /* Carpenter & Kennedy (1994) five-stage fourth-order 2N-storage */
    A[0] = 0.0;
    A[1] = (double)(-567301805773.0L / 1357537059087.0L);
    A[2] = (double)(-2404267990393.0L / 2016746695238.0L);
    A[3] = (double)(-3550918686646.0L / 2091501179385.0L);
    A[4] = (double)(-1275806237668.0L / 842570457699.0L);
    B[0] = (double)(1432997174477.0L / 9575080441755.0L);
    B[1] = (double)(5161836677717.0L / 13612068292357.0L);
    B[2] = (double)(1720146321549.0L / 2090206949498.0L);
    B[3] = (double)(3134564353537.0L / 4481467310338.0L);
    B[4] = (double)(2277821191437.0L / 14882151754819.0L);
    C[0] = 0.0;
    C[1] = (double)(1432997174477.0L / 9575080441755.0L);
    C[2] = (double)(2526269341429.0L / 6820363962896.0L);
    C[3] = (double)(2006345519317.0L / 3224310063776.0L);
    C[4] = (double)(2802321613138.0L / 2924317926251.0L);
    C[5] = 1.0;
    return 5;
  case BFAM_B200_LSRK_W33:
    /* Williamson (1980) three-stage third-order */
    A[0] = 0.0;
    A[1] = (double)(-5.0L / 9.0L);
    A[2] = (double)(-153.0L / 128.0L);
    B[0] = (double)(1.0L / 3.0L);
    B[1] = (double)(15.0L / 16.0L);
    B[2] = (double)(8.0L / 15.0L);
    C[0] = 0.0;
    C[1] = (double)(1.0L / 3.0L);
    C[2] = (double)(3.0L / 4.0L);
    C[3] = 1.0;
    return 3;
  case BFAM_B200_LSRK_HEUN:
    A[0] = 0.0;
    A[1] = -1.0;
    B[0] = 1.0;
    B[1] = 0.5;
    C[0] = 0.0;
    C[1] = 1.0;
    C[2] = 1.0;
    return 2;
  case BFAM_B200_LSRK_FE:
    A[0] = 0.0;
    B[0] = 1.0;
    C[0] = 0.0;
    C[1] = 1.0;
    return 1;
  default:
    return -1;
  }
}
