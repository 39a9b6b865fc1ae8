/*
 * Test infrastructure only: the interface of oracle/bfam_split_driver.c
 * (compiled with the reference's src/bfam.c into oracle/_ref/).  Include
 * after <bfam.h>.
 */
#ifndef BFAM_SPLIT_DRIVER_H
#define BFAM_SPLIT_DRIVER_H

#include <stdint.h>

typedef struct
{
  int n[3];        /* base trees per axis */
  int periodic[3]; /* periodic axes */
  double L[3];     /* brick extent */
  int N;           /* order */
  uint64_t seed;
  int levels;  /* refinement passes */
  double prob; /* refinement probability per pass */
} bfref_spec_t;

typedef struct
{
  int dim, N, Nq, Np, Nfp, NF;
  int32_t K;
  double *r, *w, *Dr; /* the subdomain's LGL operators (Nq, Nq, Nq*Nq) */
  int32_t *vmapM, *vmapP;
  int32_t *quads; /* [K][5]: tree, level, x, y, z (p4est integer coords) */
  double *x0, *h; /* [K][3] */
  int max_level;
  int32_t root_len;
  int32_t num_trees;
  double *tree_x0, *tree_h; /* [num_trees][3] */
  /* local glue grid (hanging faces) */
  int32_t Kg;
  int32_t *EToEm, *EToEp;
  int8_t *EToFm, *EToHm, *EToHp, *EToOp;
  double *interp[3], *proj[3]; /* NULL: identity */
  /* boundary glue grids (minus side), concatenated in domain order */
  int32_t Kb;
  int32_t *EToEb;
  int8_t *EToFb;
  int num_local_glue, num_boundary_glue;
} bfref_mesh_t;

typedef struct bfref_domain bfref_domain_t;

int bfref_dim(void);
/* the reference's front end on a brick; NULL on bad input */
bfref_domain_t *bfref_domain_new(const bfref_spec_t *spec);
/* the bfam domain it built (valid until bfref_domain_free) */
bfam_domain_pxest_t *bfref_domain_pxest(bfref_domain_t *d);
void bfref_domain_free(bfref_domain_t *d);
/* copies of the arrays bfam holds after the split */
int bfref_mesh_new(bfref_domain_t *d, bfref_mesh_t **out);
void bfref_mesh_free(bfref_mesh_t *m);

#endif
