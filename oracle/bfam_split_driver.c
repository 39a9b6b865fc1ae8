/*
 * Test infrastructure only.  Compiled by oracle/build_ref.sh together with
 * the reference's own src/bfam.c and its vendored p4est-1.1 (serial) into
 * oracle/_ref/libbfam_ref{2,3}d.so, once per dimension
 * (-DBFAM_DGX_DIMENSION=2 or 3).  Only tests/ load it, as the source of
 * bfam's own split of an adapted brick; the product never does.
 *
 * bfref_domain_new() runs the reference's mesh front end on a brick:
 *   p4est_connectivity_new_brick / p8est_connectivity_new_brick,
 *   bfam_domain_pxest_new_ext (src/bfam.c:3805),
 *   `levels` passes of seeded random refinement (pass l refines each
 *   quadrant of level l with probability prob, PCG32 stream 1 + l, in forest
 *   order), p4est_balance (full connectivity: faces, edges, corners),
 *   bfam_domain_pxest_split_dgx_subdomains (src/bfam.c:7565-8054) into one
 *   volume subdomain of order N with its local (hanging-face) and boundary
 *   glue subdomains.
 * bfref_mesh_new() returns the arrays bfam holds after the split -- the
 * volume subdomain's vmapM/vmapP and LGL operators (src/bfam.h:1364-1420),
 * the local glue grid's EToEm/EToFm/EToHm (minus side) and EToEp/EToHp/EToOp
 * (plus side) with interpolation[3]/projection[3] (src/bfam.h:1319-1362),
 * the boundary glue grids' minus-side faces -- plus each element's p4est
 * quadrant (tree, level, integer corner) and affine box, read from the forest
 * through the subdomain's EToQ.
 */
#include <bfam.h>

#include "bfam_split_driver.h"

#include <stdlib.h>
#include <string.h>

#define NFACE P4EST_FACES

/* PCG32 (M. E. O'Neill, pcg-random.org), the generator every seeded draw of
 * the test problems uses; uniform numbers are next() * 2^-32 */
typedef struct
{
  uint64_t state, inc;
} drv_rng_t;

static uint32_t drv_next(drv_rng_t *g)
{
  const uint64_t old = g->state;
  g->state = old * 6364136223846793005ULL + (g->inc | 1u);
  const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = (uint32_t)(old >> 59u);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

static void drv_seed(drv_rng_t *g, uint64_t s, uint64_t seq)
{
  g->state = 0u;
  g->inc = (seq << 1u) | 1u;
  (void)drv_next(g);
  g->state += s;
  (void)drv_next(g);
}


typedef struct
{
  drv_rng_t rng;
  int level;
  double prob;
} drv_refine_t;

static int drv_refine_cb(p4est_t *p, p4est_topidx_t t, p4est_quadrant_t *q)
{
  (void)t;
  drv_refine_t *r = p->user_pointer;
  if (q->level != r->level)
    return 0;
  return drv_next(&r->rng) * (1.0 / 4294967296.0) < r->prob;
}

static int drv_inited = 0;

static void drv_init(void)
{
  if (drv_inited)
    return;
  sc_init(sc_MPI_COMM_WORLD, 0, 0, NULL, SC_LP_SILENT);
  p4est_init(NULL, SC_LP_SILENT);
  bfam_log_init(0, stderr, BFAM_LL_SILENT);
  drv_inited = 1;
}

struct bfref_domain
{
  bfam_domain_pxest_t *domain;
  p4est_connectivity_t *conn;
  double L[3];
  int n[3];
};

int bfref_dim(void) { return BFAM_DGX_DIMENSION; }

/* Build the forest and split it with the reference's own code. */
bfref_domain_t *bfref_domain_new(const bfref_spec_t *spec)
{
  drv_init();
  if (spec->N < 1 || spec->levels < 0 || spec->levels > 8)
    return NULL;
  for (int a = 0; a < BFAM_DGX_DIMENSION; ++a)
    if (spec->n[a] < 1)
      return NULL;
  bfref_domain_t *d = calloc(1, sizeof(*d));
  for (int a = 0; a < 3; ++a)
  {
    d->L[a] = spec->L[a];
    d->n[a] = spec->n[a];
  }
#if BFAM_DGX_DIMENSION == 2
  d->conn = p4est_connectivity_new_brick(spec->n[0], spec->n[1],
                                         spec->periodic[0], spec->periodic[1]);
#else
  d->conn = p8est_connectivity_new_brick(spec->n[0], spec->n[1], spec->n[2],
                                         spec->periodic[0], spec->periodic[1],
                                         spec->periodic[2]);
#endif
  d->domain = bfam_domain_pxest_new_ext(sc_MPI_COMM_WORLD, d->conn, 0, 0, 1);
  p4est_t *px = d->domain->pxest;
  drv_refine_t rf;
  void *saved = px->user_pointer;
  for (int l = 0; l < spec->levels; ++l)
  {
    drv_seed(&rf.rng, spec->seed, 1 + (uint64_t)l);
    rf.level = l;
    rf.prob = spec->prob;
    px->user_pointer = &rf;
    p4est_refine(px, 0, drv_refine_cb, bfam_domain_pxest_quadrant_init);
  }
  px->user_pointer = saved;
  p4est_balance(px, P4EST_CONNECT_FULL, bfam_domain_pxest_quadrant_init);

  const p4est_locidx_t K = px->local_num_quadrants;
  bfam_locidx_t *sub = calloc((size_t)K, sizeof(bfam_locidx_t));
  int Ns[1] = {spec->N};
  bfam_domain_pxest_split_dgx_subdomains(d->domain, 1, sub, NULL, Ns, NULL,
                                         NULL, NULL);
  free(sub);
  return d;
}

bfam_domain_pxest_t *bfref_domain_pxest(bfref_domain_t *d)
{
  return d->domain;
}

void bfref_domain_free(bfref_domain_t *d)
{
  if (!d)
    return;
  bfam_domain_pxest_free(d->domain);
  bfam_free(d->domain);
  p4est_connectivity_destroy(d->conn);
  free(d);
}

static double *dup_d(const double *s, size_t n)
{
  if (!s)
    return NULL;
  double *p = malloc(sizeof(double) * n);
  memcpy(p, s, sizeof(double) * n);
  return p;
}

/* subdomains of the domain carrying `tag` */
static bfam_locidx_t drv_subs(bfam_domain_t *dom, const char *tag,
                              bfam_subdomain_t **out, bfam_locidx_t cap)
{
  const char *tags[] = {tag, NULL};
  bfam_locidx_t n = 0;
  bfam_domain_get_subdomains(dom, BFAM_DOMAIN_OR, tags, cap, out, &n);
  return n;
}

/* Tree boxes of the brick: tree t's lower corner is its first vertex times
 * the base cell size (a brick's vertices are integer lattice points). */
static void drv_tree_boxes(const bfref_domain_t *d, double *x0, double *h)
{
  const p4est_connectivity_t *c = d->conn;
  for (p4est_topidx_t t = 0; t < c->num_trees; ++t)
  {
    const p4est_topidx_t v = c->tree_to_vertex[P4EST_CHILDREN * t];
    for (int a = 0; a < 3; ++a)
    {
      const double cell = a < BFAM_DGX_DIMENSION ? d->L[a] / d->n[a] : 0.0;
      x0[3 * t + a] = c->vertices[3 * v + a] * cell;
      h[3 * t + a] = cell;
    }
  }
}

int bfref_mesh_new(bfref_domain_t *d, bfref_mesh_t **out)
{
  *out = NULL;
  bfam_domain_t *dom = (bfam_domain_t *)d->domain;
  bfam_subdomain_t *subs[4096];
  const bfam_locidx_t nv = drv_subs(dom, "_volume", subs, 4096);
  if (nv != 1)
    return 1;
  bfam_subdomain_dgx_t *v = (bfam_subdomain_dgx_t *)subs[0];
  bfref_mesh_t *m = calloc(1, sizeof(*m));
  const int dim = BFAM_DGX_DIMENSION;
  m->dim = dim;
  m->N = v->N;
  m->Nq = v->N + 1;
  m->Np = v->Np;
  m->Nfp = dim == 3 ? m->Nq * m->Nq : m->Nq;
  m->NF = NFACE;
  m->K = v->K;
  m->r = dup_d(v->r, m->Nq);
  m->w = dup_d(v->w, m->Nq);
  m->Dr = dup_d(v->Dr, (size_t)m->Nq * m->Nq);
  const size_t nmap = (size_t)v->K * NFACE * m->Nfp;
  m->vmapM = malloc(sizeof(int32_t) * nmap);
  m->vmapP = malloc(sizeof(int32_t) * nmap);
  memcpy(m->vmapM, v->vmapM, sizeof(int32_t) * nmap);
  memcpy(m->vmapP, v->vmapP, sizeof(int32_t) * nmap);

  /* quadrants through EToQ (element -> local quadrant of the forest) */
  p4est_t *px = d->domain->pxest;
  const p4est_locidx_t nq = px->local_num_quadrants;
  int32_t *qt = malloc(sizeof(int32_t) * (size_t)nq * 5);
  for (p4est_topidx_t t = px->first_local_tree; t <= px->last_local_tree; ++t)
  {
    p4est_tree_t *tree = p4est_tree_array_index(px->trees, t);
    for (size_t i = 0; i < tree->quadrants.elem_count; ++i)
    {
      const p4est_quadrant_t *q = p4est_quadrant_array_index(&tree->quadrants, i);
      const size_t k = tree->quadrants_offset + i;
      qt[5 * k + 0] = (int32_t)t;
      qt[5 * k + 1] = q->level;
      qt[5 * k + 2] = q->x;
      qt[5 * k + 3] = q->y;
#if BFAM_DGX_DIMENSION == 3
      qt[5 * k + 4] = q->z;
#else
      qt[5 * k + 4] = 0;
#endif
    }
  }
  m->num_trees = (int32_t)d->conn->num_trees;
  m->tree_x0 = malloc(sizeof(double) * 3 * m->num_trees);
  m->tree_h = malloc(sizeof(double) * 3 * m->num_trees);
  drv_tree_boxes(d, m->tree_x0, m->tree_h);
  m->root_len = P4EST_ROOT_LEN;
  m->quads = malloc(sizeof(int32_t) * 5 * (size_t)m->K);
  m->x0 = malloc(sizeof(double) * 3 * (size_t)m->K);
  m->h = malloc(sizeof(double) * 3 * (size_t)m->K);
  m->max_level = 0;
  for (int32_t e = 0; e < m->K; ++e)
  {
    const int32_t k = v->EToQ[e];
    memcpy(m->quads + 5 * (size_t)e, qt + 5 * (size_t)k, sizeof(int32_t) * 5);
    const int32_t t = qt[5 * k], lvl = qt[5 * k + 1];
    if (lvl > m->max_level)
      m->max_level = lvl;
    for (int a = 0; a < 3; ++a)
    {
      const double th = m->tree_h[3 * t + a];
      m->x0[3 * e + a] =
          a < dim ? m->tree_x0[3 * t + a] +
                        th * ((double)qt[5 * k + 2 + a] / P4EST_ROOT_LEN)
                  : 0.0;
      m->h[3 * e + a] = a < dim ? th / (double)(1 << lvl) : 0.0;
    }
  }
  free(qt);

  /* local glue grid(s) of this volume subdomain */
  const bfam_locidx_t ng = drv_subs(dom, "_glue_local", subs, 4096);
  m->num_local_glue = ng;
  if (ng > 1)
  {
    free(m);
    return 2;
  }
  if (ng == 1)
  {
    bfam_subdomain_dgx_t *g = (bfam_subdomain_dgx_t *)subs[0];
    bfam_subdomain_dgx_glue_data_t *gm =
        (bfam_subdomain_dgx_glue_data_t *)g->base.glue_m;
    bfam_subdomain_dgx_glue_data_t *gp =
        (bfam_subdomain_dgx_glue_data_t *)g->base.glue_p;
    const int32_t Kg = g->K;
    m->Kg = Kg;
    m->EToEm = malloc(sizeof(int32_t) * Kg);
    m->EToEp = malloc(sizeof(int32_t) * Kg);
    m->EToFm = malloc(Kg);
    m->EToHm = malloc(Kg);
    m->EToHp = malloc(Kg);
    m->EToOp = malloc(Kg);
    memcpy(m->EToEm, gm->EToEm, sizeof(int32_t) * Kg);
    memcpy(m->EToFm, gm->EToFm, Kg);
    memcpy(m->EToHm, gm->EToHm, Kg);
    memcpy(m->EToEp, gp->EToEp, sizeof(int32_t) * Kg);
    memcpy(m->EToHp, gp->EToHp, Kg);
    memcpy(m->EToOp, gp->EToOp, Kg);
    const size_t nn = (size_t)m->Nq * m->Nq;
    for (int i = 0; i < 3; ++i)
    {
      m->interp[i] = dup_d(gm->interpolation[i], nn);
      m->proj[i] = dup_d(gm->projection[i], nn);
    }
  }

  /* boundary glue grids, concatenated */
  const bfam_locidx_t nb = drv_subs(dom, "_glue_boundary", subs, 4096);
  m->num_boundary_glue = nb;
  int32_t Kb = 0;
  for (bfam_locidx_t s = 0; s < nb; ++s)
    Kb += ((bfam_subdomain_dgx_t *)subs[s])->K;
  m->Kb = Kb;
  m->EToEb = malloc(sizeof(int32_t) * (Kb ? Kb : 1));
  m->EToFb = malloc(Kb ? Kb : 1);
  for (bfam_locidx_t s = 0, o = 0; s < nb; ++s)
  {
    bfam_subdomain_dgx_t *g = (bfam_subdomain_dgx_t *)subs[s];
    bfam_subdomain_dgx_glue_data_t *gm =
        (bfam_subdomain_dgx_glue_data_t *)g->base.glue_m;
    memcpy(m->EToEb + o, gm->EToEm, sizeof(int32_t) * g->K);
    memcpy(m->EToFb + o, gm->EToFm, g->K);
    o += g->K;
  }
  *out = m;
  return 0;
}

void bfref_mesh_free(bfref_mesh_t *m)
{
  if (!m)
    return;
  free(m->r);
  free(m->w);
  free(m->Dr);
  free(m->vmapM);
  free(m->vmapP);
  free(m->quads);
  free(m->x0);
  free(m->h);
  free(m->tree_x0);
  free(m->tree_h);
  free(m->EToEm);
  free(m->EToEp);
  free(m->EToFm);
  free(m->EToHm);
  free(m->EToHp);
  free(m->EToOp);
  for (int i = 0; i < 3; ++i)
  {
    free(m->interp[i]);
    free(m->proj[i]);
  }
  free(m->EToEb);
  free(m->EToFb);
  free(m);
}
