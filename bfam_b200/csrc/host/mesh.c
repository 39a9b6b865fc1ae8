/*
 * Brick mesher that emits bfam's volume and glue data model.
 *
 * For the adapted Cartesian bricks used here (one refinement level on top of
 * a periodic brick of base cells) this produces what
 * bfam_domain_pxest_split_dgx_subdomains (src/bfam.c:7565-7840) produces
 * from a p4est forest for a single volume subdomain:
 *  - EToE/EToF: same-size neighbours, the element itself for faces that
 *    are hanging (src/bfam.c:7702-7732);
 *  - vmapM/vmapP from the face masks (src/bfam.c:6599-6877);
 *  - one local glue grid holding every hanging face, one glue element per
 *    (element, face, hanging piece), sorted in receive order (element, face,
 *    hanging number) with EToEp giving the partner's receive position
 *    (src/bfam.c:4587-4800, 7328-7520, 1942-2042).
 * Hanging pieces are numbered 1 + a + 2b where a (b) is the half along the
 * face's first (second) tangential axis, the p4est face-child order under
 * orientation 0; every face of an aligned brick has orientation 0.
 */
#include "bfam_b200_host.h"

#include <stdlib.h>
#include <string.h>

static uint64_t morton_key(int dim, int x, int y, int z)
{
  uint64_t key = 0;
  for (int b = 0; b < 21; ++b)
  {
    key |= (uint64_t)((x >> b) & 1) << (dim * b);
    key |= (uint64_t)((y >> b) & 1) << (dim * b + 1);
    if (dim == 3)
      key |= (uint64_t)((z >> b) & 1) << (dim * b + 2);
  }
  return key;
}

typedef struct
{
  uint64_t key;
  int32_t cell;
} keyed_t;

static int keyed_cmp(const void *a, const void *b)
{
  const keyed_t *x = a, *y = b;
  return (x->key > y->key) - (x->key < y->key);
}

/* face-node n of face f -> volume node (src/bfam.c:6641-6700 ordering) */
static int gmask(int dim, int Nq, int f, int n)
{
  const int N = Nq - 1;
  if (dim == 2)
  {
    switch (f)
    {
    case 0: return n * Nq;
    case 1: return n * Nq + N;
    case 2: return n;
    default: return N * Nq + n;
    }
  }
  const int a = n % Nq, b = n / Nq;
  switch (f)
  {
  case 0: return Nq * a + Nq * Nq * b;
  case 1: return N + Nq * a + Nq * Nq * b;
  case 2: return a + Nq * Nq * b;
  case 3: return a + Nq * N + Nq * Nq * b;
  case 4: return a + Nq * b;
  default: return a + Nq * b + Nq * Nq * N;
  }
}

/* tangential axes of a face normal to `axis` (first = faster face index) */
static void face_axes(int dim, int axis, int *t0, int *t1)
{
  if (dim == 2)
  {
    *t0 = axis == 0 ? 1 : 0;
    *t1 = -1;
    return;
  }
  *t0 = axis == 0 ? 1 : 0;
  *t1 = axis == 2 ? 1 : 2;
}

void bfam_b200_brick_mesh_free(bfam_b200_mesh_t *m)
{
  if (!m)
    return;
  free(m->ecoord);
  free(m->x0);
  free(m->h);
  free(m->EToE);
  free(m->EToF);
  free(m->vmapM);
  free(m->vmapP);
  free(m->EToEm);
  free(m->EToFm);
  free(m->EToEb);
  free(m->EToFb);
  free(m->EToHm);
  free(m->EToEp);
  free(m->EToHp);
  free(m->EToOp);
  free(m);
}

int bfam_b200_brick_mesh_new(const bfam_b200_brick_spec_t *spec,
                             bfam_b200_mesh_t **out)
{
  *out = NULL;
  const int dim = spec->dim;
  if (dim != 2 && dim != 3)
    return 1;
  if (spec->N < 1 || spec->N > 15)
    return 2;
  int n[3] = {spec->n[0], spec->n[1], dim == 3 ? spec->n[2] : 1};
  for (int a = 0; a < dim; ++a)
  {
    if (n[a] < 1 || n[a] > (1 << 20))
      return 3;
  }
  const int64_t ncell64 = (int64_t)n[0] * n[1] * n[2];
  if (ncell64 * (dim == 3 ? 8 : 4) > INT32_MAX / 2)
    return 5;
  const int32_t ncell = (int32_t)ncell64;

  /* base cells in Morton order */
  keyed_t *order = malloc(sizeof(keyed_t) * ncell);
  for (int z = 0, c = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x, ++c)
      {
        order[c].key = morton_key(dim, x, y, z);
        order[c].cell = c;
      }
  qsort(order, ncell, sizeof(keyed_t), keyed_cmp);

  uint8_t *refined = calloc(ncell, 1);
  int32_t num_refined = 0;
  if (spec->refine_flags)
  {
    for (int32_t c = 0; c < ncell; ++c)
      refined[c] = spec->refine_flags[c] ? 1 : 0;
  }
  else
  {
    bfam_b200_pcg32_t rng;
    bfam_b200_pcg32_seed(&rng, spec->seed, 1);
    for (int32_t i = 0; i < ncell; ++i)
      refined[order[i].cell] =
          bfam_b200_pcg32_uniform(&rng) < spec->refine_prob ? 1 : 0;
  }
  const int nchild = dim == 3 ? 8 : 4;
  int32_t *first = malloc(sizeof(int32_t) * ncell);
  int32_t K = 0;
  for (int32_t i = 0; i < ncell; ++i)
  {
    const int32_t c = order[i].cell;
    first[c] = K;
    K += refined[c] ? nchild : 1;
    num_refined += refined[c];
  }

  bfam_b200_mesh_t *m = calloc(1, sizeof(bfam_b200_mesh_t));
  const int Nq = spec->N + 1;
  const int NF = 2 * dim;
  m->dim = dim;
  m->N = spec->N;
  m->Nq = Nq;
  m->Np = dim == 3 ? Nq * Nq * Nq : Nq * Nq;
  m->Nfp = dim == 3 ? Nq * Nq : Nq;
  m->Nfaces = NF;
  m->K = K;
  m->num_refined = num_refined;
  m->ecoord = malloc(sizeof(int32_t) * 4 * K);
  m->x0 = malloc(sizeof(double) * 3 * K);
  m->h = malloc(sizeof(double) * 3 * K);
  m->EToE = malloc(sizeof(int32_t) * NF * K);
  m->EToF = malloc(sizeof(int8_t) * NF * K);
  int32_t *ecell = malloc(sizeof(int32_t) * K); /* base cell of element */
  int8_t *echild = malloc(sizeof(int8_t) * K);  /* child id or -1 */

  double unit[3];
  for (int a = 0; a < 3; ++a)
    unit[a] = (a < dim ? spec->L[a] : 1.0) / (2.0 * n[a]);

  for (int32_t i = 0; i < ncell; ++i)
  {
    const int32_t c = order[i].cell;
    const int bx = c % n[0], by = (c / n[0]) % n[1], bz = c / (n[0] * n[1]);
    const int nch = refined[c] ? nchild : 1;
    for (int ch = 0; ch < nch; ++ch)
    {
      const int32_t e = first[c] + ch;
      const int cx = refined[c] ? (ch & 1) : 0;
      const int cy = refined[c] ? ((ch >> 1) & 1) : 0;
      const int cz = refined[c] ? ((ch >> 2) & 1) : 0;
      const int size = refined[c] ? 1 : 2;
      m->ecoord[4 * e + 0] = 2 * bx + cx;
      m->ecoord[4 * e + 1] = 2 * by + cy;
      m->ecoord[4 * e + 2] = dim == 3 ? 2 * bz + cz : 0;
      m->ecoord[4 * e + 3] = size;
      for (int a = 0; a < 3; ++a)
      {
        m->x0[3 * e + a] = a < dim ? m->ecoord[4 * e + a] * unit[a] : 0.0;
        m->h[3 * e + a] = a < dim ? size * unit[a] : 0.0;
      }
      ecell[e] = c;
      echild[e] = refined[c] ? (int8_t)ch : (int8_t)-1;
    }
  }

  /* neighbour search; pass 0 counts glue, pass 1 fills */
  int32_t *glue_first = malloc(sizeof(int32_t) * NF * K);
  int32_t Kg = 0;
  m->EToEb = malloc(sizeof(int32_t) * NF * (size_t)K);
  m->EToFb = malloc(sizeof(int8_t) * NF * (size_t)K);
  m->Kb = 0;
  for (int pass = 0; pass < 2; ++pass)
  {
    int32_t g = 0;
    for (int32_t e = 0; e < K; ++e)
    {
      const int32_t c = ecell[e];
      int bc[3] = {c % n[0], (c / n[0]) % n[1], c / (n[0] * n[1])};
      int cc[3] = {0, 0, 0};
      if (echild[e] >= 0)
      {
        cc[0] = echild[e] & 1;
        cc[1] = (echild[e] >> 1) & 1;
        cc[2] = (echild[e] >> 2) & 1;
      }
      for (int f = 0; f < NF; ++f)
      {
        const int a = f / 2, s = f % 2;
        int t0, t1;
        face_axes(dim, a, &t0, &t1);
        int nb[3] = {bc[0], bc[1], bc[2]};
        nb[a] = (bc[a] + (s ? 1 : -1) + n[a]) % n[a];
        const int32_t cn = nb[0] + n[0] * (nb[1] + n[1] * nb[2]);
        if (pass == 0)
          glue_first[NF * e + f] = -1;
        /* a face on a non-periodic side of the brick: the element's base
         * cell touches that side and the face is not toward a sibling */
        const int outer = echild[e] < 0 || (s ? cc[a] == 1 : cc[a] == 0);
        if (!spec->periodic[a] && outer &&
            (s ? bc[a] == n[a] - 1 : bc[a] == 0))
        {
          m->EToE[NF * e + f] = e;
          m->EToF[NF * e + f] = (int8_t)f;
          if (pass == 1)
          {
            m->EToEb[m->Kb] = e;
            m->EToFb[m->Kb] = (int8_t)f;
            ++m->Kb;
          }
          continue;
        }
        if (echild[e] < 0)
        {
          if (!refined[cn])
          {
            m->EToE[NF * e + f] = first[cn];
            m->EToF[NF * e + f] = (int8_t)(f ^ 1);
          }
          else
          {
            m->EToE[NF * e + f] = e;
            m->EToF[NF * e + f] = (int8_t)f;
            const int P = nchild / 2;
            if (pass == 0)
            {
              glue_first[NF * e + f] = g;
              g += P;
            }
            else
            {
              for (int hh = 0; hh < P; ++hh, ++g)
              {
                int k3[3] = {0, 0, 0};
                k3[a] = s ? 0 : 1;
                k3[t0] = hh & 1;
                if (t1 >= 0)
                  k3[t1] = (hh >> 1) & 1;
                const int32_t nk = first[cn] + k3[0] + 2 * k3[1] + 4 * k3[2];
                const int nf = f ^ 1;
                m->EToEm[g] = e;
                m->EToFm[g] = (int8_t)f;
                m->EToHm[g] = (int8_t)(hh + 1);
                m->EToEp[g] = glue_first[NF * nk + nf];
                m->EToHp[g] = 0;
                m->EToOp[g] = 0;
              }
            }
          }
        }
        else
        {
          const int inside = s ? (cc[a] == 0) : (cc[a] == 1);
          if (inside || refined[cn])
          {
            int k3[3] = {cc[0], cc[1], cc[2]};
            k3[a] = 1 - cc[a];
            const int32_t base = inside ? first[c] : first[cn];
            m->EToE[NF * e + f] = base + k3[0] + 2 * k3[1] + 4 * k3[2];
            m->EToF[NF * e + f] = (int8_t)(f ^ 1);
          }
          else
          {
            m->EToE[NF * e + f] = e;
            m->EToF[NF * e + f] = (int8_t)f;
            if (pass == 0)
            {
              glue_first[NF * e + f] = g;
              g += 1;
            }
            else
            {
              const int hp = 1 + cc[t0] + (t1 >= 0 ? 2 * cc[t1] : 0);
              const int32_t nk = first[cn];
              const int nf = f ^ 1;
              m->EToEm[g] = e;
              m->EToFm[g] = (int8_t)f;
              m->EToHm[g] = 0;
              m->EToEp[g] = glue_first[NF * nk + nf] + (hp - 1);
              m->EToHp[g] = (int8_t)hp;
              m->EToOp[g] = 0;
              ++g;
            }
          }
        }
      }
    }
    if (pass == 0)
    {
      Kg = g;
      m->Kg = Kg;
      m->EToEm = malloc(sizeof(int32_t) * (Kg ? Kg : 1));
      m->EToFm = malloc(sizeof(int8_t) * (Kg ? Kg : 1));
      m->EToHm = malloc(sizeof(int8_t) * (Kg ? Kg : 1));
      m->EToEp = malloc(sizeof(int32_t) * (Kg ? Kg : 1));
      m->EToHp = malloc(sizeof(int8_t) * (Kg ? Kg : 1));
      m->EToOp = malloc(sizeof(int8_t) * (Kg ? Kg : 1));
    }
  }

  /* vmapM / vmapP (orientation 0 everywhere on an aligned brick) */
  const int Nfp = m->Nfp, Np = m->Np;
  const size_t nmap = (size_t)K * NF * Nfp;
  m->vmapM = malloc(sizeof(int32_t) * nmap);
  m->vmapP = malloc(sizeof(int32_t) * nmap);
  for (int32_t e = 0; e < K; ++e)
    for (int f = 0; f < NF; ++f)
    {
      const int32_t nk = m->EToE[NF * e + f];
      const int nf = m->EToF[NF * e + f];
      const size_t sk = ((size_t)e * NF + f) * Nfp;
      for (int q = 0; q < Nfp; ++q)
      {
        m->vmapM[sk + q] = (int32_t)(e * Np + gmask(dim, Nq, f, q));
        m->vmapP[sk + q] = (int32_t)(nk * Np + gmask(dim, Nq, nf, q));
      }
    }

  free(glue_first);
  free(ecell);
  free(echild);
  free(first);
  free(refined);
  free(order);
  *out = m;
  return 0;
}
