/*
 * Material and initial data for the elastic benchmark problems.  The
 * reference provides field arrays and an init callback type
 * (bfam_subdomain_init_field_t, src/bfam.h:781-784) but no elastic data, so
 * these are stated from the equations:
 *   rho dv/dt = div S,   dS/dt = lambda (div v) I + mu (grad v + grad v^T).
 */
#include "bfam_b200_host.h"

#include <math.h>

void bfam_b200_material_random(int32_t K, uint64_t seed, double rho_lo,
                               double rho_hi, double cp_lo, double cp_hi,
                               double r_lo, double r_hi, double *rho,
                               double *lambda, double *mu)
{
  bfam_b200_pcg32_t rng;
  bfam_b200_pcg32_seed(&rng, seed, 2);
  for (int32_t e = 0; e < K; ++e)
  {
    const double u1 = bfam_b200_pcg32_uniform(&rng);
    const double u2 = bfam_b200_pcg32_uniform(&rng);
    const double u3 = bfam_b200_pcg32_uniform(&rng);
    const double r = rho_lo + (rho_hi - rho_lo) * u1;
    const double cp = cp_lo + (cp_hi - cp_lo) * u2;
    const double cs = cp / (r_lo + (r_hi - r_lo) * u3);
    rho[e] = r;
    mu[e] = r * cs * cs;
    lambda[e] = r * (cp * cp - 2 * cs * cs);
  }
}

void bfam_b200_node_coordinates(const bfam_b200_mesh_t *m, const double *r,
                                double *x, double *y, double *z)
{
  const int Nq = m->Nq, Np = m->Np;
  for (int32_t e = 0; e < m->K; ++e)
    for (int n = 0; n < Np; ++n)
    {
      const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
      const double *x0 = m->x0 + 3 * e, *h = m->h + 3 * e;
      const size_t id = (size_t)e * Np + n;
      x[id] = x0[0] + 0.5 * h[0] * (r[i] + 1);
      y[id] = x0[1] + 0.5 * h[1] * (r[j] + 1);
      if (z)
        z[id] = m->dim == 3 ? x0[2] + 0.5 * h[2] * (r[k] + 1) : 0.0;
    }
}

void bfam_b200_init_plane_wave(const bfam_b200_mesh_t *m, const double *r,
                               const double *kv, double A, double rho,
                               double lambda, double mu, double time,
                               double *const *fields)
{
  const int dim = m->dim, Nq = m->Nq, Np = m->Np;
  const double cp = sqrt((lambda + 2 * mu) / rho);
  double kk = 0;
  for (int a = 0; a < dim; ++a)
    kk += kv[a] * kv[a];
  kk = sqrt(kk);
  double nh[3] = {0, 0, 0};
  for (int a = 0; a < dim; ++a)
    nh[a] = kv[a] / kk;
  const double om = cp * kk;
  for (int32_t e = 0; e < m->K; ++e)
    for (int n = 0; n < Np; ++n)
    {
      const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
      const double *x0 = m->x0 + 3 * e, *h = m->h + 3 * e;
      double X[3];
      X[0] = x0[0] + 0.5 * h[0] * (r[i] + 1);
      X[1] = x0[1] + 0.5 * h[1] * (r[j] + 1);
      X[2] = dim == 3 ? x0[2] + 0.5 * h[2] * (r[k] + 1) : 0.0;
      double ph = -om * time;
      for (int a = 0; a < dim; ++a)
        ph += kv[a] * X[a];
      const double s = sin(ph);
      const double sv = A * s, ss = -(A / cp) * s;
      const size_t id = (size_t)e * Np + n;
      if (dim == 3)
      {
        fields[0][id] = sv * nh[0];
        fields[1][id] = sv * nh[1];
        fields[2][id] = sv * nh[2];
        fields[3][id] = ss * (lambda + 2 * mu * nh[0] * nh[0]);
        fields[4][id] = ss * (lambda + 2 * mu * nh[1] * nh[1]);
        fields[5][id] = ss * (lambda + 2 * mu * nh[2] * nh[2]);
        fields[6][id] = ss * (2 * mu * nh[0] * nh[1]);
        fields[7][id] = ss * (2 * mu * nh[0] * nh[2]);
        fields[8][id] = ss * (2 * mu * nh[1] * nh[2]);
      }
      else
      {
        fields[0][id] = sv * nh[0];
        fields[1][id] = sv * nh[1];
        fields[2][id] = ss * (lambda + 2 * mu * nh[0] * nh[0]);
        fields[3][id] = ss * (lambda + 2 * mu * nh[1] * nh[1]);
        fields[4][id] = ss * (2 * mu * nh[0] * nh[1]);
      }
    }
}

void bfam_b200_init_gaussian_pulse(const bfam_b200_mesh_t *m, const double *r,
                                   const double *c, double width,
                                   double *const *fields)
{
  const int dim = m->dim, Nq = m->Nq, Np = m->Np;
  const int nf = dim == 3 ? 9 : 5;
  for (int32_t e = 0; e < m->K; ++e)
    for (int n = 0; n < Np; ++n)
    {
      const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
      const double *x0 = m->x0 + 3 * e, *h = m->h + 3 * e;
      double d2 = 0;
      const double X0 = x0[0] + 0.5 * h[0] * (r[i] + 1) - c[0];
      const double X1 = x0[1] + 0.5 * h[1] * (r[j] + 1) - c[1];
      d2 = X0 * X0 + X1 * X1;
      if (dim == 3)
      {
        const double X2 = x0[2] + 0.5 * h[2] * (r[k] + 1) - c[2];
        d2 += X2 * X2;
      }
      const double p = exp(-d2 / (width * width));
      const size_t id = (size_t)e * Np + n;
      for (int f = 0; f < nf; ++f)
        fields[f][id] = 0.0;
      for (int a = 0; a < dim; ++a)
        fields[dim + a][id] = -p;
    }
}
