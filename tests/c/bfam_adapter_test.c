/*
 * C test of the adapter from bfam's objects to the bfam_gpu C-ABI
 * (include/bfam_gpu_bfam.h), compiled against the reference's own
 * src/bfam.h and linked with the reference's src/bfam.c (built from source
 * into oracle/_ref/ by oracle/build_ref.sh) and bfam_b200/libbfam_b200.so.
 * tests/test_bfam_adapter.py runs it on a GPU and checks its output against
 * the oracle.
 *
 *   bfam_adapter_test{2,3}d IN OUT
 *
 * It builds the adapted brick with bfam's own front end (p4est brick,
 * seeded refinement passes, 2:1 balance, bfam_domain_pxest_split_dgx_
 * subdomains), adds the state, material and node coordinate fields to the
 * volume subdomain with bfam_domain_add_fields and fills them from IN, uploads
 * the domain through bfam_gpu_domain_upload (node coordinate fields) or
 * bfam_gpu_domain_upload_pxest (quadrants), evaluates the right-hand side,
 * sets up the stepper with bfam_gpu_lsrk_init (bfamo_lsrk_init's shape,
 * aux_rates adding "lsrk_" rate fields as a bfam application does), steps,
 * and downloads the state into bfam's field arrays, which it writes to OUT.
 *
 * IN  (native endianness): int32 hdr[16] = {magic 0x62666164, dim, N, n0, n1,
 *     n2, periodic0, periodic1, periodic2, levels, seed, nsteps, flux,
 *     precision, geometry (0 node coordinate fields, 1 quadrants), bc};
 *     double prob, L0, L1, L2, dt; int32 K; double rho[K], lam[K], mu[K];
 *     double q0[nfields][K Np].
 * OUT: int32 {status, K, aux_rates calls, checks passed}; double
 *     rhs[nfields][K Np]; double q[nfields][K Np].
 */
#include <bfam.h>

#include "bfam_gpu_bfam.h"
#include "bfam_split_driver.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define DIM BFAM_DGX_DIMENSION
#define NFLD (DIM == 3 ? 9 : 5)

#if DIM == 3
static const char *field_names[] = {"vx",  "vy",  "vz",  "sxx", "syy",
                                    "szz", "sxy", "sxz", "syz", NULL};
#else
static const char *field_names[] = {"vx", "vy", "sxx", "syy", "sxy", NULL};
#endif
static const char *aux_names[] = {"rho", "lam", "mu", "_grid_x0", "_grid_x1",
                                  "_grid_x2", NULL};

static int read_all(FILE *f, void *p, size_t n)
{
  return fread(p, 1, n, f) == n ? 0 : 1;
}

typedef struct
{
  int calls;
} aux_state_t;

/* what a bfam application's aux_rates does: add the rate fields */
static void aux_rates(bfam_subdomain_t *sub, const char *prefix, void *user)
{
  aux_state_t *st = (aux_state_t *)user;
  char name[64];
  for (int f = 0; field_names[f]; ++f)
  {
    snprintf(name, sizeof(name), "%s%s", prefix, field_names[f]);
    sub->field_add(sub, name);
  }
  ++st->calls;
}

static int bc_value;
static int bc_fn(bfam_subdomain_t *glue, void *arg)
{
  (void)glue;
  return *(int *)arg;
}

static int report(const char *what, int rc)
{
  char msg[512];
  bfam_gpu_last_error(msg, sizeof(msg));
  fprintf(stderr, "bfam_adapter_test: %s failed (%d): %s\n", what, rc, msg);
  return rc;
}

int main(int argc, char **argv)
{
  if (argc != 3)
  {
    fprintf(stderr, "usage: %s IN OUT\n", argv[0]);
    return 2;
  }
  FILE *in = fopen(argv[1], "rb");
  if (!in)
    return 2;
  int32_t hdr[16];
  double dv[5];
  int32_t Kin;
  if (read_all(in, hdr, sizeof(hdr)) || read_all(in, dv, sizeof(dv)) ||
      read_all(in, &Kin, sizeof(Kin)) || hdr[0] != 0x62666164 || hdr[1] != DIM)
  {
    fprintf(stderr, "bfam_adapter_test: bad input header\n");
    return 2;
  }
  bfref_spec_t spec;
  memset(&spec, 0, sizeof(spec));
  for (int a = 0; a < 3; ++a)
  {
    spec.n[a] = hdr[3 + a];
    spec.periodic[a] = hdr[6 + a];
    spec.L[a] = dv[1 + a];
  }
  spec.N = hdr[2];
  spec.levels = hdr[9];
  spec.seed = (uint64_t)hdr[10];
  spec.prob = dv[0];
  const int nsteps = hdr[11], geometry = hdr[14];
  bc_value = hdr[15];
  const double dt = dv[4];

  bfref_domain_t *ref = bfref_domain_new(&spec);
  if (!ref)
    return 3;
  bfam_domain_pxest_t *pdom = bfref_domain_pxest(ref);
  bfam_domain_t *dom = &pdom->base;
  const char *volume[] = {"_volume", NULL};
  const char *glue[] = {"_glue_local", NULL};
  const char *boundary[] = {"_glue_boundary", NULL};
  bfam_domain_add_fields(dom, BFAM_DOMAIN_OR, volume, field_names);
  bfam_domain_add_fields(dom, BFAM_DOMAIN_OR, volume, aux_names);

  bfam_subdomain_t *subs[2];
  bfam_locidx_t ns = 0;
  bfam_domain_get_subdomains(dom, BFAM_DOMAIN_OR, volume, 2, subs, &ns);
  if (ns != 1)
    return 3;
  bfam_subdomain_dgx_t *v = (bfam_subdomain_dgx_t *)subs[0];
  const int Np = v->Np, Nq = v->N + 1;
  const bfam_locidx_t K = v->K;
  if (K != Kin)
  {
    fprintf(stderr, "bfam_adapter_test: K = %d, input has %d\n", K, Kin);
    return 3;
  }
  const size_t n = (size_t)K * Np;

  /* material broadcast to the nodes, state */
  double *mat = malloc(sizeof(double) * 3 * (size_t)K);
  if (read_all(in, mat, sizeof(double) * 3 * (size_t)K))
    return 2;
  for (int i = 0; i < 3; ++i)
  {
    double *fld = bfam_dictionary_get_value_ptr(&v->base.fields, aux_names[i]);
    for (bfam_locidx_t e = 0; e < K; ++e)
      for (int j = 0; j < Np; ++j)
        fld[(size_t)e * Np + j] = mat[(size_t)i * K + e];
  }
  for (int f = 0; f < NFLD; ++f)
  {
    double *fld = bfam_dictionary_get_value_ptr(&v->base.fields, field_names[f]);
    if (read_all(in, fld, sizeof(double) * n))
      return 2;
  }
  fclose(in);

  /* node coordinates (what a bfam application fills for its VTK output):
   * the quadrant of each element in its brick tree */
  {
    p4est_t *px = pdom->pxest;
    p4est_connectivity_t *conn = pdom->conn;
    double *g[3];
    for (int a = 0; a < 3; ++a)
      g[a] = bfam_dictionary_get_value_ptr(&v->base.fields, aux_names[3 + a]);
    for (bfam_locidx_t e = 0; e < K; ++e)
    {
      const p4est_locidx_t k = v->EToQ[e];
      p4est_topidx_t t = px->first_local_tree;
      p4est_tree_t *tree = p4est_tree_array_index(px->trees, t);
      while ((size_t)k >= tree->quadrants_offset + tree->quadrants.elem_count)
        tree = p4est_tree_array_index(px->trees, ++t);
      const p4est_quadrant_t *q = p4est_quadrant_array_index(
          &tree->quadrants, (size_t)k - tree->quadrants_offset);
      const p4est_topidx_t v0 = conn->tree_to_vertex[P4EST_CHILDREN * t];
      p4est_qcoord_t qc[3] = {q->x, q->y, 0};
#if DIM == 3
      qc[2] = q->z;
#endif
      double x0[3] = {0, 0, 0}, h[3] = {0, 0, 0};
      for (int a = 0; a < DIM; ++a)
      {
        const double cell = spec.L[a] / spec.n[a];
        x0[a] = cell * conn->vertices[3 * v0 + a] +
                cell * ((double)qc[a] / P4EST_ROOT_LEN);
        h[a] = cell / (double)(1 << q->level);
      }
      for (int j = 0; j < Np; ++j)
      {
        const int ix[3] = {j % Nq, (j / Nq) % Nq, j / (Nq * Nq)};
        for (int a = 0; a < 3; ++a)
          g[a][(size_t)e * Np + j] =
              a < DIM ? x0[a] + 0.5 * h[a] * (v->r[ix[a]] + 1.0) : 0.0;
      }
    }
  }

  bfam_gpu_bfam_options_t opts;
  memset(&opts, 0, sizeof(opts));
  opts.gpu.flux = hdr[12];
  opts.gpu.precision = hdr[13];
  opts.boundary_tags = boundary;
  opts.boundary_condition = bc_fn;
  opts.boundary_arg = &bc_value;
  for (int a = 0; a < DIM; ++a)
    opts.vertex_scale[a] = spec.L[a] / spec.n[a];

  int checks = 0;
  bfam_gpu_domain_t *gdom = NULL;
  int rc;

  /* a field list of the wrong length is refused with a message */
  {
    const char *short_list[] = {"vx", NULL};
    rc = bfam_gpu_domain_upload(dom, BFAM_DOMAIN_OR, volume, glue, short_list,
                                &opts, &gdom);
    char msg[256];
    bfam_gpu_last_error(msg, sizeof(msg));
    if (rc != BFAM_GPU_EINVAL || gdom || !strstr(msg, "bfam_gpu_bfam"))
      return report("rejecting a short field list", rc ? rc : -99);
    ++checks;
  }

  rc = geometry ? bfam_gpu_domain_upload_pxest(pdom, BFAM_DOMAIN_OR, volume,
                                               glue, field_names, &opts, &gdom)
                : bfam_gpu_domain_upload(dom, BFAM_DOMAIN_OR, volume, glue,
                                         field_names, &opts, &gdom);
  if (rc)
    return report("upload", rc);
  ++checks;

  double *rhs = malloc(sizeof(double) * NFLD * n);
  double *rp[9];
  for (int f = 0; f < NFLD; ++f)
    rp[f] = rhs + (size_t)f * n;
  if ((rc = bfam_gpu_domain_rhs(gdom, rp)))
    return report("rhs", rc);

  aux_state_t aux = {0};
  bfam_ts_lsrk_t *ts = NULL;
  if ((rc = bfam_gpu_lsrk_init(&ts, gdom, dom, "lsrk_", 0, BFAM_DOMAIN_OR,
                               volume, aux_rates, &aux)))
    return report("lsrk init", rc);
  if (!bfam_dictionary_get_value_ptr(&v->base.fields, "lsrk_vx"))
    return report("aux_rates fields", -98);
  ++checks;
  if (nsteps > 0 && (rc = bfam_ts_lsrk_step(ts, dt, nsteps, 1)))
    return report("step", rc);
  if ((rc = bfam_gpu_domain_sync(gdom)))
    return report("sync", rc);
  if ((rc = bfam_gpu_domain_download(gdom, dom, BFAM_DOMAIN_OR, volume,
                                     field_names)))
    return report("download", rc);
  ++checks;

  /* push the downloaded state back and download again: unchanged */
  {
    double *first = malloc(sizeof(double) * n);
    double *vx = bfam_dictionary_get_value_ptr(&v->base.fields, "vx");
    memcpy(first, vx, sizeof(double) * n);
    if ((rc = bfam_gpu_domain_push(gdom, dom, BFAM_DOMAIN_OR, volume,
                                   field_names)))
      return report("push", rc);
    memset(vx, 0, sizeof(double) * n);
    if ((rc = bfam_gpu_domain_download(gdom, dom, BFAM_DOMAIN_OR, volume,
                                       field_names)))
      return report("download after push", rc);
    if (memcmp(first, vx, sizeof(double) * n))
      return report("push/download round trip", -97);
    free(first);
    ++checks;
  }

  FILE *out = fopen(argv[2], "wb");
  if (!out)
    return 2;
  const int32_t head[4] = {0, K, aux.calls, checks};
  fwrite(head, sizeof(head), 1, out);
  fwrite(rhs, sizeof(double), NFLD * n, out);
  for (int f = 0; f < NFLD; ++f)
    fwrite(bfam_dictionary_get_value_ptr(&v->base.fields, field_names[f]),
           sizeof(double), n, out);
  fclose(out);

  bfam_ts_lsrk_free(ts);
  bfam_gpu_domain_free(gdom);
  free(rhs);
  free(mat);
  bfref_domain_free(ref);
  return 0;
}
