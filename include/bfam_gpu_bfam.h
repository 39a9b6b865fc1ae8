/*
 * bfam_gpu_bfam.h -- bfam's objects in, the bfam_gpu device layer out.
 *
 * Header-only adapter for applications built on bfam: include it after the
 * application's own <bfam.h> (compiled with its BFAM_DGX_DIMENSION) and link
 * libbfam_b200.so.  It reads the subdomains bfam_domain_pxest_split_dgx_
 * subdomains produced (src/bfam.c:7565-8054) and hands their arrays to the
 * plain C-ABI of bfam_gpu.h:
 *
 *   reference (bfam)                                  here
 *   -----------------------------------------------------------------------
 *   bfam_domain_get_subdomains(dom, match, tags)      bfam_gpu_domain_upload
 *     (src/bfam.c:2255-2308) selecting the volume     (domain, match, volume
 *     subdomain (bfam_subdomain_dgx_t,                 tags, glue tags, field
 *     src/bfam.h:1364-1420), its local glue grid       names, options)
 *     (bfam_subdomain_dgx_glue_data_t,
 *     src/bfam.h:1319-1362) and boundary glue grids
 *   the same on a bfam_domain_pxest_t, element        bfam_gpu_domain_upload_pxest
 *     geometry from the forest's quadrants (EToQ,
 *     ID_QUAD_* layout, src/bfam.h:1600-1606)
 *   bfamo_lsrk_init(ts, dom, prefix, method, match,   bfam_gpu_lsrk_init
 *     tags, aux_rates, user_data)
 *     (src/bfam.h:1859-1863, src/bfam.c:8996-9090)
 *   the field arrays of bfam_subdomain_dgx_field_add  bfam_gpu_domain_download /
 *     (src/bfam.c:6574-6597)                           bfam_gpu_domain_push
 *
 * Element geometry: bfam stores none of its own; its VTK writer reads node
 * coordinates from the fields "_grid_x0", "_grid_x1", "_grid_x2"
 * (src/bfam.c:6113-6118), which the application fills.  The upload reads
 * each element's affine box from its first and last node there (names
 * configurable), or, in the _pxest form, from the p4est quadrant of each
 * element (tree, level, corner) and the brick connectivity's tree boxes.
 * Material: per-node fields (default "rho", "lam", "mu"), constant per
 * element; node 0 is read.
 *
 * Every function returns 0 or a negative BFAM_GPU_E* code with the message in
 * bfam_gpu_last_error().
 */
#ifndef BFAM_GPU_BFAM_H
#define BFAM_GPU_BFAM_H

#include "bfam_gpu.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef BFAM_H
#error "include the application's <bfam.h> before bfam_gpu_bfam.h"
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* condition of the faces of one boundary glue subdomain (BFAM_GPU_BC_*) */
typedef int (*bfam_gpu_bc_fn_t)(bfam_subdomain_t *glue, void *arg);

typedef struct
{
  bfam_gpu_options_t gpu; /* flux, precision, memory budget, device */
  /* per-node material fields, constant per element; NULL: "rho", "lam",
   * "mu" */
  const char *material[3];
  /* node coordinate fields; NULL: "_grid_x0", "_grid_x1", "_grid_x2" (not
   * read by the _pxest form) */
  const char *grid[3];
  /* boundary glue subdomains of the volume (NULL-terminated tags, matched
   * with BFAM_DOMAIN_OR, e.g. {"_glue_boundary", NULL}); NULL: none */
  const char **boundary_tags;
  /* condition per boundary glue subdomain; NULL: free surface */
  bfam_gpu_bc_fn_t boundary_condition;
  void *boundary_arg;
  /* _pxest form: the application's coordinates of a connectivity vertex v
   * are vertex_scale[a] * conn->vertices[3 v + a] (0: 1) */
  double vertex_scale[3];
} bfam_gpu_bfam_options_t;

/* ---------------------------------------------------------------- helpers */

static inline int bfam_gpu_bfam_fail_(int code, const char *what)
{
  return bfam_gpu_record_error(code, what);
}

/* The one dgx volume subdomain matching the tags. */
static inline int bfam_gpu_bfam_volume_(bfam_domain_t *domain,
                                        bfam_domain_match_t match,
                                        const char **volume_tags,
                                        bfam_subdomain_dgx_t **out)
{
  bfam_subdomain_t **subs = (bfam_subdomain_t **)malloc(
      sizeof(bfam_subdomain_t *) * (size_t)(domain->num_subdomains + 1));
  bfam_locidx_t n = 0;
  bfam_domain_get_subdomains(domain, match, volume_tags,
                             domain->num_subdomains, subs, &n);
  *out = n == 1 ? (bfam_subdomain_dgx_t *)subs[0] : NULL;
  free(subs);
  if (n != 1)
    return bfam_gpu_bfam_fail_(
        BFAM_GPU_EUNSUPPORTED,
        "bfam_gpu_bfam: the volume tags must match exactly one subdomain "
        "(one device domain per volume subdomain)");
  if (!bfam_subdomain_has_tag(&(*out)->base, "_subdomain_dgx") ||
      (*out)->dim != BFAM_DGX_DIMENSION)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: the volume subdomain is not a "
                               "dgx subdomain of the application's dimension");
  return 0;
}

static inline double *bfam_gpu_bfam_field_(bfam_subdomain_dgx_t *s,
                                           const char *name)
{
  return (double *)bfam_dictionary_get_value_ptr(&s->base.fields, name);
}

static inline int bfam_gpu_bfam_nfields_(const char **fields)
{
  int n = 0;
  while (fields && fields[n])
    ++n;
  return n;
}

/* Shared by both upload forms; pxest != NULL takes geometry from its
 * quadrants. */
static inline int bfam_gpu_bfam_upload_(bfam_domain_t *domain,
                                        bfam_domain_pxest_t *pxest,
                                        bfam_domain_match_t match,
                                        const char **volume_tags,
                                        const char **glue_tags,
                                        const char **fields,
                                        const bfam_gpu_bfam_options_t *opts,
                                        bfam_gpu_domain_t **out)
{
  if (!out)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL, "bfam_gpu_bfam: out is NULL");
  *out = NULL;
  if (!domain || !volume_tags || !fields || !opts)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: domain, volume tags, fields or "
                               "options is NULL");
  bfam_subdomain_dgx_t *v = NULL;
  int rc = bfam_gpu_bfam_volume_(domain, match, volume_tags, &v);
  if (rc)
    return rc;
  const int dim = BFAM_DGX_DIMENSION;
  const int nfld = dim == 3 ? 9 : 5;
  if (bfam_gpu_bfam_nfields_(fields) != nfld)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: fields must name the 5 (2D) or "
                               "9 (3D) state fields, NULL-terminated");
  const int Np = v->Np;
  const bfam_locidx_t K = v->K;
  double *q[9];
  for (int f = 0; f < nfld; ++f)
    if (!(q[f] = bfam_gpu_bfam_field_(v, fields[f])))
      return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                                 "bfam_gpu_bfam: a state field is not in the "
                                 "volume subdomain's field dictionary");

  /* material, node 0 of every element */
  static const char *const mat_default[3] = {"rho", "lam", "mu"};
  double *mat[3] = {NULL, NULL, NULL};
  for (int i = 0; i < 3 && !rc; ++i)
  {
    const char *nm = opts->material[i] ? opts->material[i] : mat_default[i];
    const double *src = bfam_gpu_bfam_field_(v, nm);
    mat[i] = (double *)malloc(sizeof(double) * (size_t)K);
    if (!src)
      rc = bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: a material field is missing");
    for (bfam_locidx_t e = 0; src && e < K; ++e)
      mat[i][e] = src[(size_t)e * Np];
  }

  bfam_gpu_volume_t vol;
  memset(&vol, 0, sizeof(vol));
  vol.dim = dim;
  vol.N = v->N;
  vol.K = K;
  vol.r = v->r;
  vol.w = v->w;
  vol.Dr = v->Dr;
  vol.vmapM = v->vmapM;
  vol.vmapP = v->vmapP;
  vol.rho = mat[0];
  vol.lambda = mat[1];
  vol.mu = mat[2];

  /* geometry */
  double *x0 = NULL, *h = NULL;
  int32_t *quads = NULL;
  double *tree_x0 = NULL, *tree_h = NULL;
  bfam_gpu_quadrants_t qd;
  memset(&qd, 0, sizeof(qd));
  if (rc)
    ;
  else if (!pxest)
  {
    static const char *const grid_default[3] = {"_grid_x0", "_grid_x1",
                                                "_grid_x2"};
    x0 = (double *)calloc(3 * (size_t)K, sizeof(double));
    h = (double *)calloc(3 * (size_t)K, sizeof(double));
    for (int a = 0; a < dim && !rc; ++a)
    {
      const double *g =
          bfam_gpu_bfam_field_(v, opts->grid[a] ? opts->grid[a] : grid_default[a]);
      if (!g)
        rc = bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                                 "bfam_gpu_bfam: a node coordinate field is "
                                 "missing");
      for (bfam_locidx_t e = 0; g && e < K; ++e)
      {
        x0[3 * e + a] = g[(size_t)e * Np];
        h[3 * e + a] = g[(size_t)e * Np + Np - 1] - g[(size_t)e * Np];
      }
    }
    vol.x0 = x0;
    vol.h = h;
  }
  else
  {
    /* quadrant of each element through EToQ; trees are the brick
     * connectivity's boxes (lower corner: vertex 0, edges: to the last
     * vertex) */
    p4est_t *px = pxest->pxest;
    p4est_connectivity_t *conn = pxest->conn;
    const p4est_locidx_t nq = px->local_num_quadrants;
    int32_t *qt = (int32_t *)malloc(sizeof(int32_t) * 5 * (size_t)nq);
    for (p4est_topidx_t t = px->first_local_tree; t <= px->last_local_tree;
         ++t)
    {
      p4est_tree_t *tree = p4est_tree_array_index(px->trees, t);
      for (size_t i = 0; i < tree->quadrants.elem_count; ++i)
      {
        const p4est_quadrant_t *qq =
            p4est_quadrant_array_index(&tree->quadrants, i);
        const size_t k = tree->quadrants_offset + i;
        qt[5 * k + 0] = (int32_t)t;
        qt[5 * k + 1] = qq->level;
        qt[5 * k + 2] = qq->x;
        qt[5 * k + 3] = qq->y;
#if BFAM_DGX_DIMENSION == 3
        qt[5 * k + 4] = qq->z;
#else
        qt[5 * k + 4] = 0;
#endif
      }
    }
    quads = (int32_t *)malloc(sizeof(int32_t) * 5 * (size_t)K);
    for (bfam_locidx_t e = 0; e < K; ++e)
      memcpy(quads + 5 * (size_t)e, qt + 5 * (size_t)v->EToQ[e],
             sizeof(int32_t) * 5);
    free(qt);
    tree_x0 = (double *)calloc(3 * (size_t)conn->num_trees, sizeof(double));
    tree_h = (double *)calloc(3 * (size_t)conn->num_trees, sizeof(double));
    for (p4est_topidx_t t = 0; t < conn->num_trees; ++t)
    {
      const p4est_topidx_t *tv = conn->tree_to_vertex + P4EST_CHILDREN * t;
      for (int a = 0; a < dim; ++a)
      {
        const double sc = opts->vertex_scale[a] != 0 ? opts->vertex_scale[a] : 1;
        tree_x0[3 * t + a] = sc * conn->vertices[3 * tv[0] + a];
        tree_h[3 * t + a] =
            sc * conn->vertices[3 * tv[P4EST_CHILDREN - 1] + a] -
            tree_x0[3 * t + a];
      }
    }
    qd.num_trees = (int32_t)conn->num_trees;
    qd.tree_x0 = tree_x0;
    qd.tree_h = tree_h;
    qd.quads = quads;
    qd.root_len = P4EST_ROOT_LEN;
  }

  /* the volume's local glue grid (hanging faces) and boundary glue grids */
  bfam_gpu_glue_t glue;
  memset(&glue, 0, sizeof(glue));
  bfam_gpu_boundary_t bnd;
  memset(&bnd, 0, sizeof(bnd));
  int32_t *bE = NULL;
  int8_t *bF = NULL, *bT = NULL;
  bfam_subdomain_t **subs = (bfam_subdomain_t **)malloc(
      sizeof(bfam_subdomain_t *) * (size_t)(domain->num_subdomains + 1));
  bfam_locidx_t ns = 0;
  if (!rc && glue_tags)
  {
    bfam_domain_get_subdomains(domain, BFAM_DOMAIN_OR, glue_tags,
                               domain->num_subdomains, subs, &ns);
    int found = 0;
    for (bfam_locidx_t s = 0; s < ns && !rc; ++s)
    {
      bfam_subdomain_dgx_t *g = (bfam_subdomain_dgx_t *)subs[s];
      bfam_subdomain_dgx_glue_data_t *gm =
          (bfam_subdomain_dgx_glue_data_t *)g->base.glue_m;
      bfam_subdomain_dgx_glue_data_t *gp =
          (bfam_subdomain_dgx_glue_data_t *)g->base.glue_p;
      if (!gm || !gp || gm->base.sub_m != &v->base)
        continue;
      if (gp->base.id_s != gm->base.id_s || gp->base.rank != gm->base.rank)
      {
        rc = bfam_gpu_bfam_fail_(BFAM_GPU_EUNSUPPORTED,
                                 "bfam_gpu_bfam: a glue grid joins the volume "
                                 "to another subdomain or rank (declare it "
                                 "with bfam_gpu_pglue_create)");
        break;
      }
      if (found++)
      {
        rc = bfam_gpu_bfam_fail_(BFAM_GPU_EUNSUPPORTED,
                                 "bfam_gpu_bfam: more than one local glue grid "
                                 "on the volume subdomain");
        break;
      }
      glue.K = g->K;
      glue.EToEp = gp->EToEp;
      glue.EToHp = gp->EToHp;
      glue.EToOp = gp->EToOp;
      glue.EToEm = gm->EToEm;
      glue.EToFm = gm->EToFm;
      glue.EToHm = gm->EToHm;
      for (int i = 0; i < 3; ++i)
      {
        glue.interpolation[i] = gm->interpolation[i];
        glue.projection[i] = gm->projection[i];
      }
      if (g->N != v->N)
        rc = bfam_gpu_bfam_fail_(BFAM_GPU_EUNSUPPORTED,
                                 "bfam_gpu_bfam: the local glue grid's order "
                                 "differs from the volume's");
    }
  }
  if (!rc && opts->boundary_tags)
  {
    bfam_domain_get_subdomains(domain, BFAM_DOMAIN_OR, opts->boundary_tags,
                               domain->num_subdomains, subs, &ns);
    int32_t Kb = 0;
    for (bfam_locidx_t s = 0; s < ns; ++s)
    {
      bfam_subdomain_dgx_glue_data_t *gm =
          (bfam_subdomain_dgx_glue_data_t *)subs[s]->glue_m;
      if (gm && gm->base.sub_m == &v->base)
        Kb += ((bfam_subdomain_dgx_t *)subs[s])->K;
    }
    bE = (int32_t *)malloc(sizeof(int32_t) * (size_t)(Kb ? Kb : 1));
    bF = (int8_t *)malloc((size_t)(Kb ? Kb : 1));
    bT = (int8_t *)malloc((size_t)(Kb ? Kb : 1));
    int32_t o = 0;
    for (bfam_locidx_t s = 0; s < ns; ++s)
    {
      bfam_subdomain_dgx_t *g = (bfam_subdomain_dgx_t *)subs[s];
      bfam_subdomain_dgx_glue_data_t *gm =
          (bfam_subdomain_dgx_glue_data_t *)g->base.glue_m;
      if (!gm || gm->base.sub_m != &v->base)
        continue;
      const int ty = opts->boundary_condition
                         ? opts->boundary_condition(&g->base, opts->boundary_arg)
                         : BFAM_GPU_BC_FREE_SURFACE;
      for (bfam_locidx_t k = 0; k < g->K; ++k, ++o)
      {
        bE[o] = gm->EToEm[k];
        bF[o] = gm->EToFm[k];
        bT[o] = (int8_t)ty;
      }
    }
    bnd.K = Kb;
    bnd.EToE = bE;
    bnd.EToF = bF;
    bnd.type = bT;
  }
  free(subs);

  if (!rc)
    rc = pxest ? bfam_gpu_domain_create_from_quadrants(&vol, &glue, &bnd, &qd,
                                                       &opts->gpu, out)
               : bfam_gpu_domain_create_with_boundary(&vol, &glue, &bnd,
                                                      &opts->gpu, out);
  if (!rc)
  {
    rc = bfam_gpu_domain_set_fields(*out, (const double *const *)q);
    if (rc)
    {
      bfam_gpu_domain_free(*out);
      *out = NULL;
    }
  }
  for (int i = 0; i < 3; ++i)
    free(mat[i]);
  free(x0);
  free(h);
  free(quads);
  free(tree_x0);
  free(tree_h);
  free(bE);
  free(bF);
  free(bT);
  return rc;
}

/* ------------------------------------------------------------ entry points */

/* Upload the one volume subdomain matching volume_tags (with `match`), the
 * local glue grid among the glue_tags subdomains that joins it to itself
 * (its 2:1 hanging faces; NULL tags: a conforming mesh), its boundary glue
 * grids (opts->boundary_tags) and its state fields[0..nf) (bfam field names
 * in the device order vx vy [vz] sxx syy [szz] sxy [sxz syz], NULL-terminated)
 * into a new device domain.  Geometry from the node coordinate fields. */
static inline int bfam_gpu_domain_upload(bfam_domain_t *domain,
                                         bfam_domain_match_t match,
                                         const char **volume_tags,
                                         const char **glue_tags,
                                         const char **fields,
                                         const bfam_gpu_bfam_options_t *opts,
                                         bfam_gpu_domain_t **out)
{
  return bfam_gpu_bfam_upload_(domain, NULL, match, volume_tags, glue_tags,
                               fields, opts, out);
}

/* The same for a p4est-managed domain, with every element's box computed on
 * the device from its quadrant (bfam_gpu_domain_create_from_quadrants); the
 * node coordinate fields are not read.  The connectivity's trees must be
 * axis-aligned boxes in the application's coordinates (a brick). */
static inline int bfam_gpu_domain_upload_pxest(
    bfam_domain_pxest_t *domain, bfam_domain_match_t match,
    const char **volume_tags, const char **glue_tags, const char **fields,
    const bfam_gpu_bfam_options_t *opts, bfam_gpu_domain_t **out)
{
  if (!domain)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL, "bfam_gpu_bfam: domain is NULL");
  return bfam_gpu_bfam_upload_(&domain->base, domain, match, volume_tags,
                               glue_tags, fields, opts, out);
}

/* Copy the device state back into the volume subdomain's state fields
 * (synchronous). */
static inline int bfam_gpu_domain_download(bfam_gpu_domain_t *gdom,
                                           bfam_domain_t *domain,
                                           bfam_domain_match_t match,
                                           const char **volume_tags,
                                           const char **fields)
{
  bfam_subdomain_dgx_t *v = NULL;
  int rc = bfam_gpu_bfam_volume_(domain, match, volume_tags, &v);
  if (rc)
    return rc;
  const int nfld = bfam_gpu_domain_num_fields(gdom);
  if (bfam_gpu_bfam_nfields_(fields) != nfld ||
      bfam_gpu_domain_field_length(gdom) != (size_t)v->K * v->Np)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: fields or sizes do not match "
                               "the device domain");
  double *q[9];
  for (int f = 0; f < nfld; ++f)
    if (!(q[f] = bfam_gpu_bfam_field_(v, fields[f])))
      return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                                 "bfam_gpu_bfam: a state field is missing");
  return bfam_gpu_domain_get_fields(gdom, q);
}

/* Copy the volume subdomain's state fields to the device again (after the
 * application changed them on the host). */
static inline int bfam_gpu_domain_push(bfam_gpu_domain_t *gdom,
                                       bfam_domain_t *domain,
                                       bfam_domain_match_t match,
                                       const char **volume_tags,
                                       const char **fields)
{
  bfam_subdomain_dgx_t *v = NULL;
  int rc = bfam_gpu_bfam_volume_(domain, match, volume_tags, &v);
  if (rc)
    return rc;
  const int nfld = bfam_gpu_domain_num_fields(gdom);
  if (bfam_gpu_bfam_nfields_(fields) != nfld ||
      bfam_gpu_domain_field_length(gdom) != (size_t)v->K * v->Np)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: fields or sizes do not match "
                               "the device domain");
  const double *q[9];
  for (int f = 0; f < nfld; ++f)
    if (!(q[f] = bfam_gpu_bfam_field_(v, fields[f])))
      return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                                 "bfam_gpu_bfam: a state field is missing");
  return bfam_gpu_domain_set_fields(gdom, q);
}

/* LSRK stepper in the shape of bfamo_lsrk_init: aux_rates(sub, lsrk_prefix,
 * user_data) is called for every subdomain matching subdom_tags, as bfam
 * does to let the application create its rate fields (the stage rates
 * themselves live on the device), then the stepper is set up on the device
 * domain with bfamo_lsrk_method_t numbering (0 KC54, 1 FE, 2 HEUN, 3 W33),
 * starting at time 0. */
typedef void (*bfam_gpu_aux_rates_t)(bfam_subdomain_t *thisSubdomain,
                                     const char *prefix, void *user_data);

static inline int bfam_gpu_lsrk_init(bfam_ts_lsrk_t **ts,
                                     bfam_gpu_domain_t *gdom,
                                     bfam_domain_t *dom,
                                     const char *lsrk_prefix, int method,
                                     bfam_domain_match_t subdom_match,
                                     const char **subdom_tags,
                                     bfam_gpu_aux_rates_t aux_rates,
                                     void *user_data)
{
  if (!ts || !gdom || !dom)
    return bfam_gpu_bfam_fail_(BFAM_GPU_EINVAL,
                               "bfam_gpu_bfam: ts, device domain or domain is "
                               "NULL");
  if (aux_rates && subdom_tags)
  {
    bfam_subdomain_t **subs = (bfam_subdomain_t **)malloc(
        sizeof(bfam_subdomain_t *) * (size_t)(dom->num_subdomains + 1));
    bfam_locidx_t n = 0;
    bfam_domain_get_subdomains(dom, subdom_match, subdom_tags,
                               dom->num_subdomains, subs, &n);
    for (bfam_locidx_t s = 0; s < n; ++s)
      aux_rates(subs[s], lsrk_prefix, user_data);
    free(subs);
  }
  return bfam_ts_lsrk_init(ts, gdom, method, 0.0);
}

#ifdef __cplusplus
}
#endif
#endif
