/*
 * ORACLE -- test infrastructure only.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library, as the checker or the
 * timed CPU baseline; the product never calls it.
 *
 * FP64 CPU restatement of the DG right-hand side and LSRK time step for the
 * isotropic velocity-stress elastic system on adapted Cartesian bricks.
 *
 * What follows the reference (bfam), with file:line:
 *  - node numbering i + Nq*(j + Nq*k), x fastest (src/bfam.c:6599-6781),
 *    faces -x,+x,-y,+y,-z,+z, face-node order of the face masks;
 *  - one-dimensional operators applied along one axis at a time, Dr
 *    column-major, as the BFAM_KRON_* loop nests (src/bfam.c:3137-3624);
 *  - hanging faces: the volume trace is interpolated to each half-size
 *    mortar piece (refine-to-bottom / refine-to-top) and the mortar flux is
 *    L2-projected back (coarsen-from-bottom / -top), piece h = 1 + a + 2b
 *    (src/bfam.c:5471-5541, 7392-7409, 4666-4800);
 *  - 2N-storage LSRK with the Carpenter-Kennedy (5,4) coefficients
 *    (src/bfam.c:9016-9039).
 * What the reference does not contain and is stated here from the
 * equations: the elastic operator and the upwind (exact Riemann) flux for
 * isotropic elasticity (Wilcox, Stadler, Burstedde, Ghattas, J. Comput.
 * Phys. 229 (2010) 9373-9396), lumped LGL mass, the discrete energy.
 *
 * Independence from the product: the LGL nodes here come from Newton's
 * method on (1-x^2) P_N'(x) with Chebyshev-Gauss-Lobatto starting points,
 * the differentiation and interpolation matrices from barycentric Lagrange
 * formulas, the L2 projection from quadrature and Gaussian elimination, and
 * neighbours from geometry (an owner map of finest-level cells), never from
 * vmapP or the glue arrays.  Physics parity against bfam itself is
 * unpinned (bfam has no elastic RHS); the operators are pinned against the
 * reference compiled from source and the physics against analytic plane
 * waves and the energy identity.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXQ 16

/* ------------------------------------------------------------ 1-D ops */

static void legendre(int N, double x, double *P, double *dP)
{
  double p0 = 1, p1 = x, d0 = 0, d1 = 1;
  if (N == 0)
  {
    *P = 1;
    *dP = 0;
    return;
  }
  for (int n = 2; n <= N; ++n)
  {
    const double p2 = ((2 * n - 1) * x * p1 - (n - 1) * p0) / n;
    const double d2 = d0 + (2 * n - 1) * p1;
    p0 = p1;
    p1 = p2;
    d0 = d1;
    d1 = d2;
  }
  *P = p1;
  *dP = d1;
}

/* LGL nodes/weights: Newton on q(x) = P_{N+1}(x) - P_{N-1}(x), whose roots
 * are +-1 and the zeros of P_N' */
void oracle_lgl_nodes(int N, double *x, double *w)
{
  const double pi = 3.14159265358979323846;
  for (int i = 0; i <= N; ++i)
  {
    double xi = -cos(pi * i / N);
    if (i > 0 && i < N)
      for (int it = 0; it < 100; ++it)
      {
        double a, da, b, db;
        legendre(N + 1, xi, &a, &da);
        legendre(N - 1, xi, &b, &db);
        const double dx = (a - b) / (da - db);
        xi -= dx;
        if (fabs(dx) < 1e-16)
          break;
      }
    x[i] = xi;
  }
  for (int i = 0; i <= N; ++i)
  {
    double P, dP;
    legendre(N, x[i], &P, &dP);
    w[i] = 2.0 / (N * (N + 1) * P * P);
  }
}

static void bary_weights(int n, const double *x, double *lam)
{
  for (int j = 0; j < n; ++j)
  {
    double p = 1;
    for (int k = 0; k < n; ++k)
      if (k != j)
        p *= (x[j] - x[k]);
    lam[j] = 1 / p;
  }
}

/* Lagrange basis of nodes x (n) evaluated at point t: L[j] */
static void lagrange_eval(int n, const double *x, const double *lam, double t,
                          double *L)
{
  for (int j = 0; j < n; ++j)
    if (t == x[j])
    {
      for (int k = 0; k < n; ++k)
        L[k] = k == j ? 1 : 0;
      return;
    }
  double s = 0;
  for (int j = 0; j < n; ++j)
    s += lam[j] / (t - x[j]);
  for (int j = 0; j < n; ++j)
    L[j] = lam[j] / (t - x[j]) / s;
}

/* D(i,j) = l_j'(x_i), stored column-major D[i + n*j] */
void oracle_diff_matrix(int N, const double *x, double *D)
{
  const int n = N + 1;
  double lam[MAXQ];
  bary_weights(n, x, lam);
  for (int i = 0; i < n; ++i)
  {
    double diag = 0;
    for (int j = 0; j < n; ++j)
      if (j != i)
      {
        const double d = lam[j] / lam[i] / (x[i] - x[j]);
        D[i + n * j] = d;
        diag -= d;
      }
    D[i + n * i] = diag;
  }
}

/* solve A X = B (n x n, m rhs), column-major, partial pivoting */
static void gauss_solve(int n, int m, double *A, double *B)
{
  for (int k = 0; k < n; ++k)
  {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i + n * k]) > fabs(A[p + n * k]))
        p = i;
    for (int j = 0; j < n; ++j)
    {
      double t = A[k + n * j];
      A[k + n * j] = A[p + n * j];
      A[p + n * j] = t;
    }
    for (int j = 0; j < m; ++j)
    {
      double t = B[k + n * j];
      B[k + n * j] = B[p + n * j];
      B[p + n * j] = t;
    }
    for (int i = k + 1; i < n; ++i)
    {
      const double l = A[i + n * k] / A[k + n * k];
      for (int j = k; j < n; ++j)
        A[i + n * j] -= l * A[k + n * j];
      for (int j = 0; j < m; ++j)
        B[i + n * j] -= l * B[k + n * j];
    }
  }
  for (int k = n - 1; k >= 0; --k)
    for (int j = 0; j < m; ++j)
    {
      double s = B[k + n * j];
      for (int i = k + 1; i < n; ++i)
        s -= A[k + n * i] * B[i + n * j];
      B[k + n * j] = s / A[k + n * k];
    }
}

/* Half-interval operators for order N.  I_b / I_t ((N+1)^2, column-major
 * I[m + n*i]): values on the bottom/top half's LGL nodes from full-interval
 * nodal values.  P_b / P_t: L2 projection of a bottom/top half-piece
 * polynomial onto the full interval, P = M^{-1} B with
 * B_im = int_{half} l_i l^{half}_m. */
void oracle_mortar_ops(int N, double *Ib, double *It, double *Pb, double *Pt)
{
  const int n = N + 1, nq = N + 2;
  double r[MAXQ], w[MAXQ], lam[MAXQ], rq[MAXQ + 1], wq[MAXQ + 1];
  oracle_lgl_nodes(N, r, w);
  bary_weights(n, r, lam);
  oracle_lgl_nodes(nq - 1, rq, wq); /* exact for degree 2N+1 */
  for (int side = 0; side < 2; ++side)
  {
    double *I = side ? It : Ib, *P = side ? Pt : Pb;
    const double sh = side ? 0.5 : -0.5;
    double L[MAXQ];
    for (int m = 0; m < n; ++m)
    {
      lagrange_eval(n, r, lam, 0.5 * r[m] + sh, L);
      for (int i = 0; i < n; ++i)
        I[m + n * i] = L[i];
    }
    double M[MAXQ * MAXQ], B[MAXQ * MAXQ];
    memset(M, 0, sizeof(M));
    memset(B, 0, sizeof(B));
    for (int q = 0; q < nq; ++q)
    {
      double Lf[MAXQ], Lh[MAXQ], Lm[MAXQ];
      lagrange_eval(n, r, lam, rq[q], Lf);
      lagrange_eval(n, r, lam, 0.5 * rq[q] + sh, Lh);
      lagrange_eval(n, r, lam, rq[q], Lm);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
          M[i + n * j] += wq[q] * Lf[i] * Lf[j];
          B[i + n * j] += 0.5 * wq[q] * Lh[i] * Lm[j];
        }
    }
    gauss_solve(n, n, M, B);
    memcpy(P, B, sizeof(double) * n * n);
  }
}

/* ------------------------------------------------------------- oracle */

typedef struct
{
  int dim, N, Nq, Np, Nfp, NF, NFLD;
  int32_t K;
  int D[3]; /* finest-level cells per axis */
  const int32_t *ec;
  double unit[3];
  double *rho, *lam, *mu;
  double r[MAXQ], w[MAXQ], Dm[MAXQ * MAXQ];
  double I[2][MAXQ * MAXQ], P[2][MAXQ * MAXQ];
  int32_t *owner; /* finest cell -> element */
  int flux;       /* 0 upwind, 1 central */
  double *work;   /* lsrk dq + rhs */
  /* Ricker point force (src_elem < 0: none): per node of the source element
   * phi_n(x_s) / (w_n J) */
  int32_t src_elem;
  double *src_W;
  double src_force[3], src_f0, src_t0;
  /* non-periodic axes: the brick's sides carry a boundary condition,
   * bc[side] (sides -x, +x, -y, +y, -z, +z): 0 free surface, 1 absorbing */
  int periodic[3];
  int bc[6];
  /* faces glued to a subdomain of another order: index per (element, face)
   * (-1: not glued) into the caller-supplied jumps gjump[n][6][Nfp] */
  int *gidx;
  int nglued;
  double *gjump;
} oracle_t;

static int32_t owner_at(const oracle_t *o, int x, int y, int z)
{
  x = ((x % o->D[0]) + o->D[0]) % o->D[0];
  y = ((y % o->D[1]) + o->D[1]) % o->D[1];
  z = o->dim == 3 ? ((z % o->D[2]) + o->D[2]) % o->D[2] : 0;
  return o->owner[x + (size_t)o->D[0] * (y + (size_t)o->D[1] * z)];
}

/* Elements are boxes of finest-level cells: ecoord[4e..4e+3] = (x, y, z,
 * size) in cells of a brick of fine[a] cells per axis and extent L[a]. */
oracle_t *oracle_new_ext(int dim, int N, int32_t K, const int32_t *ecoord,
                         const int *fine, const double *L, const double *rho,
                         const double *lam, const double *mu, int flux)
{
  if ((dim != 2 && dim != 3) || N < 1 || N >= MAXQ - 1)
    return NULL;
  oracle_t *o = calloc(1, sizeof(oracle_t));
  o->dim = dim;
  o->N = N;
  o->Nq = N + 1;
  o->Np = dim == 3 ? o->Nq * o->Nq * o->Nq : o->Nq * o->Nq;
  o->Nfp = dim == 3 ? o->Nq * o->Nq : o->Nq;
  o->NF = 2 * dim;
  o->NFLD = dim == 3 ? 9 : 5;
  o->K = K;
  o->flux = flux;
  o->src_elem = -1;
  for (int a = 0; a < 3; ++a)
    o->periodic[a] = 1;
  o->ec = ecoord;
  for (int a = 0; a < 3; ++a)
  {
    o->D[a] = a < dim ? fine[a] : 1;
    o->unit[a] = a < dim ? L[a] / fine[a] : 1.0;
  }
  o->rho = malloc(sizeof(double) * K);
  o->lam = malloc(sizeof(double) * K);
  o->mu = malloc(sizeof(double) * K);
  memcpy(o->rho, rho, sizeof(double) * K);
  memcpy(o->lam, lam, sizeof(double) * K);
  memcpy(o->mu, mu, sizeof(double) * K);
  oracle_lgl_nodes(N, o->r, o->w);
  oracle_diff_matrix(N, o->r, o->Dm);
  oracle_mortar_ops(N, o->I[0], o->I[1], o->P[0], o->P[1]);
  const size_t ncell = (size_t)o->D[0] * o->D[1] * o->D[2];
  o->owner = malloc(sizeof(int32_t) * ncell);
  for (size_t c = 0; c < ncell; ++c)
    o->owner[c] = -1;
  for (int32_t e = 0; e < K; ++e)
  {
    const int32_t *c = ecoord + 4 * e;
    const int s = c[3];
    for (int z = 0; z < (dim == 3 ? s : 1); ++z)
      for (int y = 0; y < s; ++y)
        for (int x = 0; x < s; ++x)
          o->owner[(c[0] + x) +
                   (size_t)o->D[0] * ((c[1] + y) + (size_t)o->D[1] * (c[2] + z))] = e;
  }
  for (size_t c = 0; c < ncell; ++c)
    if (o->owner[c] < 0)
    {
      free(o->owner);
      free(o->rho);
      free(o->lam);
      free(o->mu);
      free(o);
      return NULL; /* elements do not tile the brick */
    }
  return o;
}

/* bricks refined at most once: the finest cells halve the base cells */
oracle_t *oracle_new(int dim, int N, int32_t K, const int32_t *ecoord,
                     const int *nbase, const double *L, const double *rho,
                     const double *lam, const double *mu, int flux)
{
  int fine[3];
  for (int a = 0; a < 3; ++a)
    fine[a] = 2 * nbase[a];
  return oracle_new_ext(dim, N, K, ecoord, fine, L, rho, lam, mu, flux);
}

void oracle_free(oracle_t *o)
{
  if (!o)
    return;
  free(o->owner);
  free(o->rho);
  free(o->lam);
  free(o->mu);
  free(o->work);
  free(o->src_W);
  free(o->gidx);
  free(o->gjump);
  free(o);
}

/* Element holding x: the owner of the finest cell floor(x / unit) (cells
 * are half-open), and x's reference coordinates in it.  -1 if x is outside
 * the brick. */
static int32_t locate(const oracle_t *o, const double *x, double *xi)
{
  int c[3] = {0, 0, 0};
  for (int a = 0; a < o->dim; ++a)
  {
    const double f = floor(x[a] / o->unit[a]);
    if (!(f >= 0 && f < o->D[a]))
      return -1;
    c[a] = (int)f;
  }
  const int32_t e = owner_at(o, c[0], c[1], c[2]);
  const int32_t *ce = o->ec + 4 * e;
  for (int a = 0; a < 3; ++a)
    xi[a] = a < o->dim
                ? 2.0 * (x[a] - ce[a] * o->unit[a]) / (ce[3] * o->unit[a]) - 1.0
                : 0.0;
  return e;
}

/* phi_n(x) of the element's nodes (barycentric Lagrange basis) */
static void node_basis(const oracle_t *o, const double *xi, double *phi)
{
  double lam[MAXQ], L[3][MAXQ];
  bary_weights(o->Nq, o->r, lam);
  for (int a = 0; a < 3; ++a)
  {
    if (a < o->dim)
      lagrange_eval(o->Nq, o->r, lam, xi[a], L[a]);
    else
      for (int i = 0; i < o->Nq; ++i)
        L[a][i] = 1.0;
  }
  for (int n = 0; n < o->Np; ++n)
  {
    const int i = n % o->Nq, j = (n / o->Nq) % o->Nq, k = n / (o->Nq * o->Nq);
    phi[n] = L[0][i] * L[1][j] * (o->dim == 3 ? L[2][k] : 1.0);
  }
}

/* Ricker point force f(t) F at x, f(t) = (1 - 2a) exp(-a),
 * a = (pi f0 (t - t0))^2, on the velocity equation: the point force
 * projected on the Lagrange basis through the lumped LGL mass.  Returns -1
 * if x is outside the brick. */
int oracle_set_source(oracle_t *o, const double *x, const double *force,
                      double f0, double t0)
{
  double xi[3];
  const int32_t e = locate(o, x, xi);
  if (e < 0)
    return -1;
  if (!o->src_W)
    o->src_W = malloc(sizeof(double) * o->Np);
  node_basis(o, xi, o->src_W);
  const int32_t *ce = o->ec + 4 * e;
  double J = 1;
  for (int a = 0; a < o->dim; ++a)
    J *= 0.5 * ce[3] * o->unit[a];
  for (int n = 0; n < o->Np; ++n)
  {
    const int i = n % o->Nq, j = (n / o->Nq) % o->Nq, k = n / (o->Nq * o->Nq);
    const double wn = o->w[i] * o->w[j] * (o->dim == 3 ? o->w[k] : 1.0);
    o->src_W[n] /= wn * J;
  }
  o->src_elem = e;
  for (int a = 0; a < 3; ++a)
    o->src_force[a] = a < o->dim ? force[a] : 0.0;
  o->src_f0 = f0;
  o->src_t0 = t0;
  return 0;
}

/* every field interpolated at nrecv points x[3r..]: out[r * NFLD + c].
 * Returns -1 if a point is outside the brick. */
int oracle_sample(const oracle_t *o, const double *q, int nrecv,
                  const double *x, double *out)
{
  const size_t fs = (size_t)o->K * o->Np;
  double *phi = malloc(sizeof(double) * o->Np);
  for (int r = 0; r < nrecv; ++r)
  {
    double xi[3];
    const int32_t e = locate(o, x + 3 * r, xi);
    if (e < 0)
    {
      free(phi);
      return -1;
    }
    node_basis(o, xi, phi);
    for (int c = 0; c < o->NFLD; ++c)
    {
      double s = 0;
      for (int n = 0; n < o->Np; ++n)
        s += phi[n] * q[c * fs + (size_t)e * o->Np + n];
      out[r * o->NFLD + c] = s;
    }
  }
  free(phi);
  return 0;
}

/* Sides of the brick on axes with periodic[a] == 0 become boundaries with
 * condition bc[2a + side]; the ghost state is v+ = v-, S+ = -S- (free
 * surface: zero traction) or q+ = 0 (absorbing), with the element's own
 * material. */
void oracle_set_boundary(oracle_t *o, const int *periodic, const int *bc)
{
  for (int a = 0; a < 3; ++a)
    o->periodic[a] = a < o->dim ? periodic[a] : 1;
  for (int f = 0; f < 6; ++f)
    o->bc[f] = bc[f];
}

/* Faces glued to a subdomain of another order (bfam's glue between two
 * volume subdomains, src/bfam.c:7340-7414): this oracle lifts the jumps
 * (T* - T-, v* - v-) that the caller computes on the glue grid and
 * projects to this subdomain's order, J[n][6][Nfp] per glued face in list
 * order, set before each right-hand side. */
int oracle_set_glued(oracle_t *o, int n, const int32_t *elem, const int *face)
{
  free(o->gidx);
  free(o->gjump);
  o->gidx = malloc(sizeof(int) * (size_t)o->K * o->NF);
  for (size_t i = 0; i < (size_t)o->K * o->NF; ++i)
    o->gidx[i] = -1;
  for (int k = 0; k < n; ++k)
  {
    if (elem[k] < 0 || elem[k] >= o->K || face[k] < 0 || face[k] >= o->NF)
      return -1;
    o->gidx[(size_t)elem[k] * o->NF + face[k]] = k;
  }
  o->nglued = n;
  o->gjump = calloc((size_t)(n > 0 ? n : 1) * 6 * o->Nfp, sizeof(double));
  return 0;
}

void oracle_set_glued_jumps(oracle_t *o, const double *J)
{
  memcpy(o->gjump, J, sizeof(double) * (size_t)o->nglued * 6 * o->Nfp);
}

/* volume node of face node q on face f */
static int fnode(const oracle_t *o, int f, int q)
{
  const int Nq = o->Nq, N = o->N;
  const int a = q % Nq, b = q / Nq;
  if (o->dim == 2)
  {
    const int ax = f / 2, side = f % 2;
    return ax == 0 ? (side ? N : 0) + Nq * q : q + Nq * (side ? N : 0);
  }
  switch (f)
  {
  case 0: return 0 + Nq * a + Nq * Nq * b;
  case 1: return N + Nq * a + Nq * Nq * b;
  case 2: return a + 0 + Nq * Nq * b;
  case 3: return a + Nq * N + Nq * Nq * b;
  case 4: return a + Nq * b;
  default: return a + Nq * b + Nq * Nq * N;
  }
}

/* jump terms (T* - T-, v* - v-) at one face point; q holds the fields of
 * one point (vel then stress); n the outward unit normal of the minus side */
static void jumps(const oracle_t *o, const double *qm, const double *qp,
                  const double *n, double rm, double lm, double mm, double rp,
                  double lp, double mp, double *dT, double *dv)
{
  const int d = o->dim;
  double vm[3] = {0, 0, 0}, vp[3] = {0, 0, 0}, Tm[3] = {0, 0, 0},
         Tp[3] = {0, 0, 0};
  for (int a = 0; a < d; ++a)
  {
    vm[a] = qm[a];
    vp[a] = qp[a];
  }
  /* stress tensor from the field vector */
  double Sm[3][3] = {{0}}, Sp[3][3] = {{0}};
  if (d == 3)
  {
    const double *s = qm + 3, *t = qp + 3;
    Sm[0][0] = s[0]; Sm[1][1] = s[1]; Sm[2][2] = s[2];
    Sm[0][1] = Sm[1][0] = s[3]; Sm[0][2] = Sm[2][0] = s[4]; Sm[1][2] = Sm[2][1] = s[5];
    Sp[0][0] = t[0]; Sp[1][1] = t[1]; Sp[2][2] = t[2];
    Sp[0][1] = Sp[1][0] = t[3]; Sp[0][2] = Sp[2][0] = t[4]; Sp[1][2] = Sp[2][1] = t[5];
  }
  else
  {
    const double *s = qm + 2, *t = qp + 2;
    Sm[0][0] = s[0]; Sm[1][1] = s[1]; Sm[0][1] = Sm[1][0] = s[2];
    Sp[0][0] = t[0]; Sp[1][1] = t[1]; Sp[0][1] = Sp[1][0] = t[2];
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
    {
      Tm[a] += Sm[a][b] * n[b];
      Tp[a] += Sp[a][b] * n[b];
    }
  if (o->flux == 1)
  {
    for (int a = 0; a < 3; ++a)
    {
      dv[a] = 0.5 * (vp[a] - vm[a]);
      dT[a] = 0.5 * (Tp[a] - Tm[a]);
    }
    return;
  }
  const double Zpm = sqrt(rm * (lm + 2 * mm)), Zsm = sqrt(rm * mm);
  const double Zpp = sqrt(rp * (lp + 2 * mp)), Zsp = sqrt(rp * mp);
  double vnm = 0, vnp = 0, Tnm = 0, Tnp = 0;
  for (int a = 0; a < 3; ++a)
  {
    vnm += vm[a] * n[a];
    vnp += vp[a] * n[a];
    Tnm += Tm[a] * n[a];
    Tnp += Tp[a] * n[a];
  }
  /* characteristic T - Z v leaves the minus side, T + Z v the plus side */
  const double dvn = (Zpp * (vnp - vnm) + (Tnp - Tnm)) / (Zpm + Zpp);
  const double dTn = Zpm * dvn;
  for (int a = 0; a < 3; ++a)
  {
    const double vtm = vm[a] - vnm * n[a], vtp = vp[a] - vnp * n[a];
    const double Ttm = Tm[a] - Tnm * n[a], Ttp = Tp[a] - Tnp * n[a];
    const double dvt = (Zsp * (vtp - vtm) + (Ttp - Ttm)) / (Zsm + Zsp);
    dv[a] = dvn * n[a] + dvt;
    dT[a] = dTn * n[a] + Zsm * dvt;
  }
}

/* tangential axes of face f */
static void taxes(int dim, int f, int *t0, int *t1)
{
  const int a = f / 2;
  if (dim == 2)
  {
    *t0 = a == 0 ? 1 : 0;
    *t1 = -1;
    return;
  }
  *t0 = a == 0 ? 1 : 0;
  *t1 = a == 2 ? 1 : 2;
}

/* 2-D (or 1-D) tensor application out[m0 + Nq m1] = sum A0(m0,i0) A1(m1,i1)
 * in[i0 + Nq i1] for nc components stored [c][Nfp] */
static void tensor_apply(const oracle_t *o, const double *A0, const double *A1,
                         const double *in, double *out, int nc)
{
  const int Nq = o->Nq;
  if (o->dim == 2)
  {
    for (int c = 0; c < nc; ++c)
      for (int m = 0; m < Nq; ++m)
      {
        double s = 0;
        for (int i = 0; i < Nq; ++i)
          s += A0[m + Nq * i] * in[c * Nq + i];
        out[c * Nq + m] = s;
      }
    return;
  }
  const int Nfp = Nq * Nq;
  double tmp[MAXQ * MAXQ];
  for (int c = 0; c < nc; ++c)
  {
    for (int i1 = 0; i1 < Nq; ++i1)
      for (int m0 = 0; m0 < Nq; ++m0)
      {
        double s = 0;
        for (int i0 = 0; i0 < Nq; ++i0)
          s += A0[m0 + Nq * i0] * in[c * Nfp + i0 + Nq * i1];
        tmp[m0 + Nq * i1] = s;
      }
    for (int m1 = 0; m1 < Nq; ++m1)
      for (int m0 = 0; m0 < Nq; ++m0)
      {
        double s = 0;
        for (int i1 = 0; i1 < Nq; ++i1)
          s += A1[m1 + Nq * i1] * tmp[m0 + Nq * i1];
        out[c * Nfp + m0 + Nq * m1] = s;
      }
  }
}

static void face_trace(const oracle_t *o, const double *q, int32_t e, int f,
                       double *tr)
{
  const size_t fs = (size_t)o->K * o->Np;
  for (int c = 0; c < o->NFLD; ++c)
    for (int p = 0; p < o->Nfp; ++p)
      tr[c * o->Nfp + p] = q[c * fs + (size_t)e * o->Np + fnode(o, f, p)];
}

/* rhs of one element */
/* every field at the face nodes of face f of element e, [NFLD][Nfp] */
void oracle_face_trace(const oracle_t *o, const double *q, int32_t e, int f,
                       double *tr)
{
  face_trace(o, q, e, f, tr);
}

/* jump terms at n points: qm, qp [n][NFLD], minus side's outward normal nrm,
 * materials {rho, lambda, mu} of both sides -> out[n][6] (T* - T-, v* - v-) */
void oracle_point_jumps(const oracle_t *o, int n, const double *qm,
                        const double *qp, const double *nrm,
                        const double *matm, const double *matp, double *out)
{
  for (int i = 0; i < n; ++i)
    jumps(o, qm + (size_t)i * o->NFLD, qp + (size_t)i * o->NFLD, nrm, matm[0],
          matm[1], matm[2], matp[0], matp[1], matp[2], out + 6 * (size_t)i,
          out + 6 * (size_t)i + 3);
}

static void element_rhs(const oracle_t *o, const double *q, int32_t e,
                        double *rhs)
{
  const int dim = o->dim, Nq = o->Nq, Np = o->Np, Nfp = o->Nfp,
            NFLD = o->NFLD;
  const size_t fs = (size_t)o->K * Np;
  const int32_t *ce = o->ec + 4 * e;
  double rx[3];
  for (int a = 0; a < 3; ++a)
    rx[a] = 2.0 / (ce[3] * o->unit[a]);
  const double rho = o->rho[e], la = o->lam[e], mu = o->mu[e];

  /* volume: gradient of every field, one axis at a time */
  double *out = malloc(sizeof(double) * NFLD * Np);
  double *g = malloc(sizeof(double) * 3 * NFLD * Np); /* [axis][field][n] */
  for (int a = 0; a < dim; ++a)
    for (int c = 0; c < NFLD; ++c)
    {
      const double *u = q + c * fs + (size_t)e * Np;
      double *gu = g + ((size_t)a * NFLD + c) * Np;
      const int st = a == 0 ? 1 : (a == 1 ? Nq : Nq * Nq);
      for (int n = 0; n < Np; ++n)
      {
        const int idx = (n / st) % Nq, base = n - idx * st;
        double s = 0;
        for (int m = 0; m < Nq; ++m)
          s += o->Dm[idx + Nq * m] * u[base + m * st];
        gu[n] = rx[a] * s;
      }
    }
#define G(a, c, n) g[((size_t)(a)*NFLD + (c)) * Np + (n)]
  for (int n = 0; n < Np; ++n)
  {
    if (dim == 3)
    {
      const double div = G(0, 0, n) + G(1, 1, n) + G(2, 2, n);
      out[0 * Np + n] = (G(0, 3, n) + G(1, 6, n) + G(2, 7, n)) / rho;
      out[1 * Np + n] = (G(0, 6, n) + G(1, 4, n) + G(2, 8, n)) / rho;
      out[2 * Np + n] = (G(0, 7, n) + G(1, 8, n) + G(2, 5, n)) / rho;
      out[3 * Np + n] = la * div + 2 * mu * G(0, 0, n);
      out[4 * Np + n] = la * div + 2 * mu * G(1, 1, n);
      out[5 * Np + n] = la * div + 2 * mu * G(2, 2, n);
      out[6 * Np + n] = mu * (G(1, 0, n) + G(0, 1, n));
      out[7 * Np + n] = mu * (G(2, 0, n) + G(0, 2, n));
      out[8 * Np + n] = mu * (G(2, 1, n) + G(1, 2, n));
    }
    else
    {
      const double div = G(0, 0, n) + G(1, 1, n);
      out[0 * Np + n] = (G(0, 2, n) + G(1, 4, n)) / rho;
      out[1 * Np + n] = (G(0, 4, n) + G(1, 3, n)) / rho;
      out[2 * Np + n] = la * div + 2 * mu * G(0, 0, n);
      out[3 * Np + n] = la * div + 2 * mu * G(1, 1, n);
      out[4 * Np + n] = mu * (G(1, 0, n) + G(0, 1, n));
    }
  }
#undef G
  free(g);

  /* faces */
  const double wend = o->w[0];
  double trm[9 * MAXQ * MAXQ], trp[9 * MAXQ * MAXQ], tri[9 * MAXQ * MAXQ];
  double J[6 * MAXQ * MAXQ], Jp[6 * MAXQ * MAXQ], Jf[6 * MAXQ * MAXQ];
  const int NJ = 2 * 3;
  for (int f = 0; f < o->NF; ++f)
  {
    const int a = f / 2, side = f % 2;
    double nrm[3] = {0, 0, 0};
    nrm[a] = side ? 1.0 : -1.0;
    int t0, t1;
    taxes(dim, f, &t0, &t1);
    const int s = ce[3];
    /* finest cell just outside the face, at the lower tangential corner */
    int p[3] = {ce[0], ce[1], ce[2]};
    p[a] = side ? ce[a] + s : ce[a] - 1;
    if (o->gidx && o->gidx[(size_t)e * o->NF + f] >= 0)
    {
      /* glued face: the jumps come from the glue between the subdomains */
      memcpy(Jf, o->gjump + (size_t)o->gidx[(size_t)e * o->NF + f] * NJ * Nfp,
             sizeof(double) * NJ * Nfp);
      goto lift;
    }
    if (!o->periodic[a] && (p[a] < 0 || p[a] >= o->D[a]))
    {
      /* boundary face: ghost state from the element's own trace */
      face_trace(o, q, e, f, trm);
      const int free_surface = o->bc[f] == 0;
      double qm[9], qp[9], dT[3], dv[3];
      for (int pt = 0; pt < Nfp; ++pt)
      {
        for (int c = 0; c < NFLD; ++c)
        {
          qm[c] = trm[c * Nfp + pt];
          qp[c] = free_surface ? (c < dim ? qm[c] : -qm[c]) : 0.0;
        }
        jumps(o, qm, qp, nrm, rho, la, mu, rho, la, mu, dT, dv);
        for (int k = 0; k < 3; ++k)
        {
          Jf[k * Nfp + pt] = dT[k];
          Jf[(3 + k) * Nfp + pt] = dv[k];
        }
      }
      goto lift;
    }
    const int32_t nb = owner_at(o, p[0], p[1], p[2]);
    const int32_t *cn = o->ec + 4 * nb;
    const int sn = cn[3];
    face_trace(o, q, e, f, trm);
    memset(Jf, 0, sizeof(double) * NJ * Nfp);
    double qm[9], qp[9], dT[3], dv[3];
    if (sn == s)
    {
      face_trace(o, q, nb, f ^ 1, trp);
      for (int pt = 0; pt < Nfp; ++pt)
      {
        for (int c = 0; c < NFLD; ++c)
        {
          qm[c] = trm[c * Nfp + pt];
          qp[c] = trp[c * Nfp + pt];
        }
        jumps(o, qm, qp, nrm, rho, la, mu, o->rho[nb], o->lam[nb], o->mu[nb],
              dT, dv);
        for (int k = 0; k < 3; ++k)
        {
          Jf[k * Nfp + pt] = dT[k];
          Jf[(3 + k) * Nfp + pt] = dv[k];
        }
      }
    }
    else if (sn == 2 * s)
    {
      /* fine side: my piece of the neighbour's face */
      const int pa = ((ce[t0] - cn[t0]) % o->D[t0] + o->D[t0]) % o->D[t0] / s;
      const int pb = t1 >= 0
                         ? ((ce[t1] - cn[t1]) % o->D[t1] + o->D[t1]) % o->D[t1] / s
                         : 0;
      face_trace(o, q, nb, f ^ 1, trp);
      tensor_apply(o, o->I[pa], t1 >= 0 ? o->I[pb] : NULL, trp, tri, NFLD);
      for (int pt = 0; pt < Nfp; ++pt)
      {
        for (int c = 0; c < NFLD; ++c)
        {
          qm[c] = trm[c * Nfp + pt];
          qp[c] = tri[c * Nfp + pt];
        }
        jumps(o, qm, qp, nrm, rho, la, mu, o->rho[nb], o->lam[nb], o->mu[nb],
              dT, dv);
        for (int k = 0; k < 3; ++k)
        {
          Jf[k * Nfp + pt] = dT[k];
          Jf[(3 + k) * Nfp + pt] = dv[k];
        }
      }
    }
    else
    {
      /* coarse side: half-size neighbours */
      const int npc = dim == 3 ? 4 : 2;
      for (int pc = 0; pc < npc; ++pc)
      {
        const int pa = pc & 1, pb = (pc >> 1) & 1;
        int pp[3] = {p[0], p[1], p[2]};
        pp[a] = side ? ce[a] + s : ce[a] - 1;
        pp[t0] = ce[t0] + pa * (s / 2);
        if (t1 >= 0)
          pp[t1] = ce[t1] + pb * (s / 2);
        const int32_t ch = owner_at(o, pp[0], pp[1], pp[2]);
        tensor_apply(o, o->I[pa], t1 >= 0 ? o->I[pb] : NULL, trm, tri, NFLD);
        face_trace(o, q, ch, f ^ 1, trp);
        for (int pt = 0; pt < Nfp; ++pt)
        {
          for (int c = 0; c < NFLD; ++c)
          {
            qm[c] = tri[c * Nfp + pt];
            qp[c] = trp[c * Nfp + pt];
          }
          jumps(o, qm, qp, nrm, rho, la, mu, o->rho[ch], o->lam[ch],
                o->mu[ch], dT, dv);
          for (int k = 0; k < 3; ++k)
          {
            J[k * Nfp + pt] = dT[k];
            J[(3 + k) * Nfp + pt] = dv[k];
          }
        }
        tensor_apply(o, o->P[pa], t1 >= 0 ? o->P[pb] : NULL, J, Jp, NJ);
        for (int i = 0; i < NJ * Nfp; ++i)
          Jf[i] += Jp[i];
      }
    }
    /* lift with the lumped LGL mass: factor (2/h_normal) / w_end */
  lift:;
    const double Lf = rx[a] / wend;
    for (int pt = 0; pt < Nfp; ++pt)
    {
      const int vn = fnode(o, f, pt);
      const double dTx = Jf[0 * Nfp + pt], dTy = Jf[1 * Nfp + pt],
                   dTz = Jf[2 * Nfp + pt];
      const double dvx = Jf[3 * Nfp + pt], dvy = Jf[4 * Nfp + pt],
                   dvz = Jf[5 * Nfp + pt];
      const double dvn = dvx * nrm[0] + dvy * nrm[1] + dvz * nrm[2];
      if (dim == 3)
      {
        out[0 * Np + vn] += Lf * dTx / rho;
        out[1 * Np + vn] += Lf * dTy / rho;
        out[2 * Np + vn] += Lf * dTz / rho;
        out[3 * Np + vn] += Lf * (la * dvn + 2 * mu * dvx * nrm[0]);
        out[4 * Np + vn] += Lf * (la * dvn + 2 * mu * dvy * nrm[1]);
        out[5 * Np + vn] += Lf * (la * dvn + 2 * mu * dvz * nrm[2]);
        out[6 * Np + vn] += Lf * mu * (dvx * nrm[1] + dvy * nrm[0]);
        out[7 * Np + vn] += Lf * mu * (dvx * nrm[2] + dvz * nrm[0]);
        out[8 * Np + vn] += Lf * mu * (dvy * nrm[2] + dvz * nrm[1]);
      }
      else
      {
        out[0 * Np + vn] += Lf * dTx / rho;
        out[1 * Np + vn] += Lf * dTy / rho;
        out[2 * Np + vn] += Lf * (la * dvn + 2 * mu * dvx * nrm[0]);
        out[3 * Np + vn] += Lf * (la * dvn + 2 * mu * dvy * nrm[1]);
        out[4 * Np + vn] += Lf * mu * (dvx * nrm[1] + dvy * nrm[0]);
      }
    }
  }
  for (int c = 0; c < NFLD; ++c)
    memcpy(rhs + c * fs + (size_t)e * Np, out + c * Np, sizeof(double) * Np);
  free(out);
}

static void set_threads(int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* rhs (same layout as q: [field][K][Np]) */
int oracle_rhs(oracle_t *o, const double *q, double *rhs, int nthreads)
{
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t e = 0; e < o->K; ++e)
    element_rhs(o, q, e, rhs);
  return 0;
}

static int lsrk_table(int method, double *A, double *B, double *C)
{
  if (method == 0)
  {
    A[0] = 0.0;
    A[1] = -567301805773.0 / 1357537059087.0;
    A[2] = -2404267990393.0 / 2016746695238.0;
    A[3] = -3550918686646.0 / 2091501179385.0;
    A[4] = -1275806237668.0 / 842570457699.0;
    B[0] = 1432997174477.0 / 9575080441755.0;
    B[1] = 5161836677717.0 / 13612068292357.0;
    B[2] = 1720146321549.0 / 2090206949498.0;
    B[3] = 3134564353537.0 / 4481467310338.0;
    B[4] = 2277821191437.0 / 14882151754819.0;
    C[0] = 0.0;
    C[1] = 1432997174477.0 / 9575080441755.0;
    C[2] = 2526269341429.0 / 6820363962896.0;
    C[3] = 2006345519317.0 / 3224310063776.0;
    C[4] = 2802321613138.0 / 2924317926251.0;
    C[5] = 1.0;
    return 5;
  }
  return -1;
}

/* LSRK coefficient tables (method 0: KC54) for callers that drive the
 * stages themselves; returns the number of stages */
int oracle_lsrk_coeffs(int method, double *A, double *B, double *C)
{
  return lsrk_table(method, A, B, C);
}

static double ricker(double t, double f0, double t0)
{
  const double pi = 3.14159265358979323846;
  const double x = pi * f0 * (t - t0);
  return (1.0 - 2.0 * x * x) * exp(-x * x);
}

/* nsteps of 2N-storage LSRK (KC54) on q, in place, from time t; the point
 * source (if set) is evaluated at the stage times t + C_s dt */
int oracle_lsrk_from(oracle_t *o, double *q, double t, double dt, int nsteps,
                     int method, int nthreads)
{
  double A[6], B[6], C[7];
  const int ns = lsrk_table(method, A, B, C);
  if (ns < 0)
    return -1;
  const size_t n = (size_t)o->K * o->Np * o->NFLD;
  if (!o->work)
    o->work = malloc(sizeof(double) * 2 * n);
  double *dq = o->work, *rhs = o->work + n;
  memset(dq, 0, sizeof(double) * n);
  set_threads(nthreads);
  for (int st = 0; st < nsteps; ++st, t += dt)
    for (int s = 0; s < ns; ++s)
    {
      oracle_rhs(o, q, rhs, nthreads);
      if (o->src_elem >= 0)
      {
        const double f = ricker(t + C[s] * dt, o->src_f0, o->src_t0);
        const int32_t e = o->src_elem;
        for (int a = 0; a < o->dim; ++a)
          for (int n = 0; n < o->Np; ++n)
            rhs[a * (size_t)o->K * o->Np + (size_t)e * o->Np + n] +=
                f * o->src_force[a] * o->src_W[n] / o->rho[e];
      }
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i)
      {
        dq[i] = A[s] * dq[i] + dt * rhs[i];
        q[i] = q[i] + B[s] * dq[i];
      }
    }
  return 0;
}

/* discrete energy with the lumped LGL mass:
 * sum_e J_e sum_n w_n (rho |v|^2 + S : C^{-1} : S) / 2 */
double oracle_energy(const oracle_t *o, const double *q)
{
  const int dim = o->dim, Nq = o->Nq, Np = o->Np;
  const size_t fs = (size_t)o->K * Np;
  double E = 0;
  for (int32_t e = 0; e < o->K; ++e)
  {
    const int32_t *ce = o->ec + 4 * e;
    double J = 1;
    for (int a = 0; a < dim; ++a)
      J *= 0.5 * ce[3] * o->unit[a];
    const double rho = o->rho[e], la = o->lam[e], mu = o->mu[e];
    double Ee = 0;
    for (int n = 0; n < Np; ++n)
    {
      const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
      const double wn = o->w[i] * o->w[j] * (dim == 3 ? o->w[k] : 1.0);
      const size_t id = (size_t)e * Np + n;
      double kin = 0, pot = 0;
      for (int a = 0; a < dim; ++a)
        kin += q[a * fs + id] * q[a * fs + id];
      kin *= rho;
      if (dim == 3)
      {
        const double sxx = q[3 * fs + id], syy = q[4 * fs + id],
                     szz = q[5 * fs + id];
        const double tr = sxx + syy + szz;
        pot = (sxx * sxx + syy * syy + szz * szz -
               la / (3 * la + 2 * mu) * tr * tr) / (2 * mu);
        for (int c = 6; c < 9; ++c)
          pot += q[c * fs + id] * q[c * fs + id] / mu;
      }
      else
      {
        /* inverse of [[l+2m, l], [l, l+2m]] on (sxx, syy) */
        const double sxx = q[2 * fs + id], syy = q[3 * fs + id],
                     sxy = q[4 * fs + id];
        const double a = la + 2 * mu, b = la, det = a * a - b * b;
        pot = (a * sxx * sxx - 2 * b * sxx * syy + a * syy * syy) / det +
              sxy * sxy / mu;
      }
      Ee += wn * (kin + pot);
    }
    E += 0.5 * J * Ee;
  }
  return E;
}

int oracle_lsrk(oracle_t *o, double *q, double dt, int nsteps, int method,
                int nthreads)
{
  return oracle_lsrk_from(o, q, 0.0, dt, nsteps, method, nthreads);
}
