/*
 * Test infrastructure only (part of the oracle's checker, never the product).
 *
 * Exported entry points around the reference's own setup numerics, compiled
 * from the reference's source by oracle/build_ref.sh (this file is appended
 * to the extracted line ranges, so the reference's static functions are
 * visible here).  Used by tests/ to pin the oracle's and the product's LGL,
 * interpolation/projection operators and PCG32 stream bit-for-bit.
 */

/* r, w, wi, Dr (column-major) and V for order N, the same call sequence as
 * bfam_subdomain_dgx_generic_init (src/bfam.c:7106-7120). */
void bfam_ref_lgl(int N, double *r, double *w, double *wi, double *Dr,
                  double *V)
{
  const int Nrp = N + 1;
  bfam_long_real_t *lr = bfam_malloc_aligned(Nrp * sizeof(bfam_long_real_t));
  bfam_long_real_t *lw = bfam_malloc_aligned(Nrp * sizeof(bfam_long_real_t));
  bfam_long_real_t *lV =
      bfam_malloc_aligned(Nrp * Nrp * sizeof(bfam_long_real_t));
  bfam_long_real_t *lDr =
      bfam_malloc_aligned(Nrp * Nrp * sizeof(bfam_long_real_t));
  bfam_jacobi_gauss_lobatto_quadrature(0, 0, N, lr, lw);
  bfam_jacobi_p_vandermonde(0, 0, N, Nrp, lr, lV);
  bfam_jacobi_p_differentiation(0, 0, N, Nrp, lr, lV, lDr);
  for (int n = 0; n < Nrp; ++n)
  {
    r[n] = (double)lr[n];
    w[n] = (double)lw[n];
    wi[n] = (double)(1.0l / lw[n]);
  }
  for (int n = 0; n < Nrp * Nrp; ++n)
  {
    Dr[n] = (double)lDr[n];
    V[n] = (double)lV[n];
  }
  bfam_free_aligned(lr);
  bfam_free_aligned(lw);
  bfam_free_aligned(lV);
  bfam_free_aligned(lDr);
}

/* Exact (modal) mass matrix for order N (src/bfam.c:3110-3133). */
void bfam_ref_mass(int N, double *M)
{
  const int Nrp = N + 1;
  bfam_long_real_t lr[Nrp], lw[Nrp], lV[Nrp * Nrp], lM[Nrp * Nrp];
  bfam_jacobi_gauss_lobatto_quadrature(0, 0, N, lr, lw);
  bfam_jacobi_p_vandermonde(0, 0, N, Nrp, lr, lV);
  bfam_jacobi_p_mass(0, 0, N, lV, lM);
  for (int n = 0; n < Nrp * Nrp; ++n)
    M[n] = (double)lM[n];
}

/* The five operators of create_interpolators (src/bfam.c:5606-5691) from
 * order N_src to N_dst: [same, coarsen-from-bottom, coarsen-from-top,
 * refine-to-bottom, refine-to-top], each (N_dst+1) x (N_src+1) column-major.
 * prj[0] is the identity (written out) when N_src == N_dst. */
void bfam_ref_interpolator(int N_src, int N_dst, double *prj, double *mass_prj,
                           double *wi_mass_prj)
{
  bfam_subdomain_dgx_interpolator_t a2b, b2a;
  create_interpolators(&a2b, N_src != N_dst ? &b2a : NULL, N_src, N_dst);
  const int n = (N_src + 1) * (N_dst + 1);
  for (int k = 0; k < 5; ++k)
  {
    for (int i = 0; i < n; ++i)
    {
      if (a2b.prj[k])
        prj[k * n + i] = a2b.prj[k][i];
      else
        prj[k * n + i] = ((i % (N_dst + 2)) == 0) ? 1.0 : 0.0;
      mass_prj[k * n + i] = a2b.mass_prj[k][i];
      wi_mass_prj[k * n + i] = a2b.wi_mass_prj[k][i];
    }
  }
}

/* n raw 32-bit outputs of the reference PCG32 after srandom(seed, seq). */
void bfam_ref_pcg32(uint64_t seed, uint64_t seq, int n, uint32_t *out)
{
  bfam_pcg32_random_t rng;
  bfam_pcg32_srandom_r(&rng, seed, seq);
  for (int i = 0; i < n; ++i)
    out[i] = bfam_pcg32_random_r(&rng);
}

/* n bounded outputs of the reference PCG32 after srandom(seed, seq). */
void bfam_ref_pcg32_bounded(uint64_t seed, uint64_t seq, uint32_t bound, int n,
                            uint32_t *out)
{
  bfam_pcg32_random_t rng;
  bfam_pcg32_srandom_r(&rng, seed, seq);
  for (int i = 0; i < n; ++i)
    out[i] = bfam_pcg32_boundedrand_r(&rng, bound);
}
