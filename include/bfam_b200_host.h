/*
 * bfam_b200 host front end: what an application gets from bfam's mesh and
 * setup layer, for adapted Cartesian bricks, without p4est.
 *
 * Everything here is host C.  It produces exactly the arrays that bfam's
 * bfam_subdomain_dgx_t and bfam_subdomain_dgx_glue_data_t hold
 * (src/bfam.h:1319-1420 of the reference), in bfam's numbering, so they can
 * be handed to the device layer declared in bfam_gpu.h the same way an
 * application would hand over arrays taken from a real bfam domain.
 */
#ifndef BFAM_B200_HOST_H
#define BFAM_B200_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- PCG32 */
/* Same generator and seeding as bfam_pcg32_srandom_r /
 * bfam_pcg32_boundedrand_r (src/bfam.c:8334-8386). */
typedef struct
{
  uint64_t state;
  uint64_t inc;
} bfam_b200_pcg32_t;

void bfam_b200_pcg32_seed(bfam_b200_pcg32_t *rng, uint64_t initstate,
                          uint64_t initseq);
uint32_t bfam_b200_pcg32_next(bfam_b200_pcg32_t *rng);
uint32_t bfam_b200_pcg32_bounded(bfam_b200_pcg32_t *rng, uint32_t bound);
/* uniform double in [0,1): next() * 2^-32 */
double bfam_b200_pcg32_uniform(bfam_b200_pcg32_t *rng);

/* ------------------------------------------------------ LGL operators */
/* r, w, wi = 1/w (N+1 each) and the differentiation matrix Dr
 * ((N+1)^2, column-major: D(i,j) = Dr[i + j*(N+1)]), computed the way
 * bfam_subdomain_dgx_generic_init does (src/bfam.c:7106-7120). */
int bfam_b200_lgl_operators(int N, double *r, double *w, double *wi,
                            double *Dr);

/* The five 1-D mortar operators of create_interpolators
 * (src/bfam.c:5606-5691) from order N_src to N_dst, each
 * (N_dst+1) x (N_src+1) column-major, stored back to back in `prj`:
 *   0 same (identity written out when N_src == N_dst),
 *   1 coarsen from bottom, 2 coarsen from top   (L2 projections),
 *   3 refine to bottom,    4 refine to top      (interpolations).
 * A glue grid's interpolation[0..2] are operators {0,3,4} of
 * (N_m -> N_g) and its projection[0..2] are operators {0,1,2} of
 * (N_g -> N_m) (src/bfam.c:7392-7409). */
int bfam_b200_mortar_operators(int N_src, int N_dst, double *prj);

/* ------------------------------------------------------------- LSRK */
/* Method numbering follows bfamo_lsrk_method_t (src/bfam.h:1848-1854). */
enum
{
  BFAM_B200_LSRK_KC54 = 0,
  BFAM_B200_LSRK_FE = 1,
  BFAM_B200_LSRK_HEUN = 2,
  BFAM_B200_LSRK_W33 = 3
};
/* Fills A, B (n_stages each) and C (n_stages + 1); returns n_stages, or -1
 * for an unknown method.  Coefficients are those of bfamo_lsrk_init
 * (src/bfam.c:9012-9089). Arrays must hold at least 6 entries. */
int bfam_b200_lsrk_coefficients(int method, double *A, double *B, double *C);

/* ------------------------------------------------------ brick meshes */
/* A brick of nx x ny (x nz) base cells on [0,Lx] x [0,Ly] (x [0,Lz]), each
 * base cell optionally refined once (one level, so 2:1 balance holds by
 * construction).  Elements are ordered along the Morton (z-order) curve of
 * the base cells, children of a refined cell in child z-order, as p4est
 * orders the leaves of a forest. */
typedef struct
{
  int dim;           /* 2 or 3 */
  int N;             /* polynomial order */
  int n[3];          /* base cells per axis (n[2] ignored in 2D) */
  double L[3];       /* domain extent per axis */
  int periodic[3];   /* 0: the two sides of the axis are domain boundaries */
  double refine_prob; /* probability that a base cell is refined */
  uint64_t seed;     /* PCG32 seed; the refinement draw uses stream 1 */
  const uint8_t *refine_flags; /* optional explicit flags per base cell in
                                  (x fastest) lexicographic order; overrides
                                  refine_prob when not NULL */
} bfam_b200_brick_spec_t;

typedef struct
{
  int dim, N, Nq, Np, Nfp, Nfaces;
  int32_t K; /* volume elements */
  /* element boxes in integer units of the finest level (half a base cell):
   * ecoord[4k+0..2] = lower corner, ecoord[4k+3] = edge length (2 or 1) */
  int32_t *ecoord;
  double *x0; /* K*3 lower corner */
  double *h;  /* K*3 edge lengths */
  /* bfam volume connectivity (src/bfam.c:7702-7732): EToE/EToF with the
   * element itself for faces that go through glue */
  int32_t *EToE;
  int8_t *EToF;
  int32_t *vmapM; /* K*Nfaces*Nfp, src/bfam.c:6783-6877 */
  int32_t *vmapP;
  /* one local glue grid (src/bfam.c:7328-7520), in receive order
   * (sorted by minus element, face, hanging number) */
  int32_t Kg;
  int32_t *EToEm;
  int8_t *EToFm;
  int8_t *EToHm;
  int32_t *EToEp;
  int8_t *EToHp;
  int8_t *EToOp;
  int32_t num_refined; /* refined base cells */
  /* boundary faces of non-periodic axes (the minus side of bfam's boundary
   * glue, src/bfam.c:7851-7899), in (element, face) order; their vmapP
   * points to the element itself */
  int32_t Kb;
  int32_t *EToEb;
  int8_t *EToFb;
} bfam_b200_mesh_t;

/* Returns 0 on success, nonzero (and *out = NULL) on bad input. */
int bfam_b200_brick_mesh_new(const bfam_b200_brick_spec_t *spec,
                             bfam_b200_mesh_t **out);
void bfam_b200_brick_mesh_free(bfam_b200_mesh_t *mesh);

/* -------------------------------------------- material, initial data */
/* Per-element isotropic material drawn with PCG32 stream 2:
 * rho ~ U[rho_lo,rho_hi], cp ~ U[cp_lo,cp_hi], cs = cp / U[r_lo,r_hi];
 * written as rho, lambda = rho (cp^2 - 2 cs^2), mu = rho cs^2. */
void bfam_b200_material_random(int32_t K, uint64_t seed, double rho_lo,
                               double rho_hi, double cp_lo, double cp_hi,
                               double r_lo, double r_hi, double *rho,
                               double *lambda, double *mu);

/* Node coordinates (K*Np per axis) of the LGL nodes r (N+1). */
void bfam_b200_node_coordinates(const bfam_b200_mesh_t *mesh, const double *r,
                                double *x, double *y, double *z);

/* Field order: 3D vx vy vz sxx syy szz sxy sxz syz; 2D vx vy sxx syy sxy.
 * fields[f] points at K*Np values of field f (bfam's per-field arrays). */

/* Plane P wave v = A n sin(k.x - w t), S = -(A/cp)(lambda I + 2 mu n n^T)
 * sin(k.x - w t), n = k/|k|, w = cp |k|, in homogeneous material. */
void bfam_b200_init_plane_wave(const bfam_b200_mesh_t *mesh, const double *r,
                               const double *k, double amplitude, double rho,
                               double lambda, double mu, double time,
                               double *const *fields);

/* Gaussian pressure pulse: v = 0, S = -exp(-|x-c|^2 / width^2) I. */
void bfam_b200_init_gaussian_pulse(const bfam_b200_mesh_t *mesh,
                                   const double *r, const double *center,
                                   double width, double *const *fields);

#ifdef __cplusplus
}
#endif
#endif
