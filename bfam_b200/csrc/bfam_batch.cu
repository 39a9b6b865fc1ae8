// C-ABI of the time-dependent extras (point source, receivers) and of
// batches of domains (declared in include/bfam_gpu.h).
//
// A batch groups its domains by (dim, order, precision, flux, operators).
// Each group owns a flat work list of (domain, element) pairs, domain-major,
// and per state parity an array of the stage kernel's domain views (state
// buffers, time step, source, clock of each domain).  One LSRK stage is one
// persistent launch per group; groups run on streams forked from the
// batch's stream, and the step ends with one post-step launch over all
// domains (receivers, clocks).  A step is captured once per parity into a
// CUDA graph and replayed.
#include "bfam_gpu.h"
#include "dg_extras.cuh"
#include "dg_pglue.cuh"
#include "dg_stage.cuh"
#include "gpu_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

using namespace bfam_b200;
using namespace bfam_b200::host;

namespace
{

// ------------------------------------------------------------ batch tiles

typedef void (*batch_launch_fn)(const DomainView *, const int2 *, int,
                                const StageParams &, const double *hops,
                                int grid, cudaStream_t);
typedef cudaError_t (*batch_prepare_fn)();
typedef int (*batch_occupancy_fn)();

struct BatchTile
{
  int NT = 0, MINB = 0, NBUF = 1;
  int EPC = 1; // elements per CTA (NT threads each)
  batch_launch_fn launch = nullptr;
  // the same tile compiled without the coarse-face pass, for launches
  // whose elements have no coarse-side hanging face (level 0 of domains
  // without faces glued to another order)
  batch_launch_fn launch_nc = nullptr;
  batch_prepare_fn prepare = nullptr;
  batch_occupancy_fn occupancy = nullptr;
};

template <int DIM, int N, int NT, int MINB, typename CT, int EPC = 1>
struct TileImpl
{
  static constexpr int NB = EPC == 1 ? nbuf<DIM, N, CT>() : 1;
  static constexpr auto kernel =
      dg_stage_batch_kernel<DIM, N, NT, MINB, MODE_STAGE, CT, NB, EPC>;
  static constexpr auto kernel_nc =
      dg_stage_batch_kernel<DIM, N, NT, MINB, MODE_STAGE_NC, CT, NB, EPC>;
  static constexpr size_t SMEM = stage_smem_bytes<DIM, N, CT, EPC>();
  static void launch(const DomainView *v, const int2 *w, int nwork,
                     const StageParams &sp, const double *hops, int grid,
                     cudaStream_t st)
  {
    const DiffOp<N, CT> dop = make_diffop<N, CT>(hops);
    kernel<<<grid, NT * EPC, SMEM, st>>>(v, w, nwork, sp, dop);
  }
  static void launch_nc(const DomainView *v, const int2 *w, int nwork,
                        const StageParams &sp, const double *hops, int grid,
                        cudaStream_t st)
  {
    const DiffOp<N, CT> dop = make_diffop<N, CT>(hops);
    kernel_nc<<<grid, NT * EPC, SMEM, st>>>(v, w, nwork, sp, dop);
  }
  static cudaError_t prepare()
  {
    cudaError_t e = cudaFuncSetAttribute(
        (const void *)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)SMEM);
    if (e != cudaSuccess)
      return e;
    return cudaFuncSetAttribute((const void *)kernel_nc,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)SMEM);
  }
  static int occupancy()
  {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, NT * EPC,
                                                      SMEM) != cudaSuccess)
    {
      cudaGetLastError();
      return 0;
    }
    return n;
  }
  static BatchTile make()
  {
    BatchTile t;
    t.NT = NT;
    t.MINB = MINB;
    t.EPC = EPC;
    t.NBUF = NB;
    t.launch = launch;
    t.launch_nc = launch_nc;
    t.prepare = prepare;
    t.occupancy = occupancy;
    return t;
  }
};

// Tile shapes per order.  Tile 0 is the single-domain kernel's shape (its
// register budget sized for the CTAs the shared memory admits); the others
// trade registers for resident CTAs or threads for nodes per thread (N = 7:
// 384 threads, one per face node, over 512 nodes).  At N = 5 the batch
// kernel, which reads its domain views and work items from memory, spills
// at tile 0's five CTAs in FP64; the four-CTA tile beside it does not.
template <typename CT> std::vector<BatchTile> tiles_for(int dim, int N)
{
  std::vector<BatchTile> v;
#define T(D, NN, NT, MB) v.push_back(TileImpl<D, NN, NT, MB, CT>::make())
#define TE(D, NN, NT, MB, E) v.push_back(TileImpl<D, NN, NT, MB, CT, E>::make())
#define T0(D, NN) T(D, NN, (Shape<D, NN>::NT), (stage_min_ctas<D, NN, CT>()))
  if (dim == 3)
  {
    // beside one element per CTA: E elements per CTA of E x threads (each
    // element its own tile and barrier), down to one warp per element at
    // the low orders (register budget for the CTAs the shared memory admits)
    switch (N)
    {
    case 1: T0(3, 1); TE(3, 1, 32, 8, 4); TE(3, 1, 32, 4, 8); break;
    case 2: T0(3, 2); TE(3, 2, 32, 8, 4); TE(3, 2, 64, 4, 2); break;
    case 3:
      T0(3, 3); T(3, 3, 96, 4); T(3, 3, 128, 4);
      TE(3, 3, 96, 3, 2); TE(3, 3, 96, 2, 4); TE(3, 3, 32, 6, 4);
      TE(3, 3, 64, 4, 4);
      break;
    case 4: T0(3, 4); TE(3, 4, 160, 2, 2); break;
    case 5: T0(3, 5); T(3, 5, 224, 4); T(3, 5, 224, 3); T(3, 5, 224, 1);
      T(3, 5, 256, 2); TE(3, 5, 224, 2, 2);
      break;
    case 6: T0(3, 6); break;
    case 7: T0(3, 7); T(3, 7, 384, 1); break;
    default: break;
    }
  }
  else if (dim == 2)
  {
    switch (N)
    {
    case 1: T0(2, 1); break;
    case 2: T0(2, 2); break;
    case 3: T0(2, 3); break;
    case 4: T0(2, 4); break;
    case 5: T0(2, 5); break;
    case 6: T0(2, 6); break;
    case 7: T0(2, 7); break;
    case 8: T0(2, 8); break;
    default: break;
    }
  }
#undef T0
#undef TE
#undef T
  return v;
}

std::vector<BatchTile> tiles(int dim, int N, int precision)
{
  return precision == BFAM_GPU_PRECISION_FP32 ? tiles_for<float>(dim, N)
                                              : tiles_for<double>(dim, N);
}

// ----------------------------------------------------- point location

// Lagrange basis of the nodes r (n of them) at t
void lagrange(const double *r, int n, double t, double *phi)
{
  for (int i = 0; i < n; ++i)
  {
    double p = 1.0;
    for (int m = 0; m < n; ++m)
      if (m != i)
        p *= (t - r[m]) / (r[i] - r[m]);
    phi[i] = p;
  }
}

// element whose half-open box [x0, x0 + h) holds x, and x's reference
// coordinates there; -1 if none
int locate(const bfam_gpu_domain_t *d, const double *x, double *xi)
{
  for (int32_t e = 0; e < d->K; ++e)
  {
    bool in = true;
    for (int a = 0; a < d->dim && in; ++a)
    {
      const double lo = d->hx0[3 * (size_t)e + a], h = d->hh[3 * (size_t)e + a];
      in = x[a] >= lo && x[a] < lo + h;
    }
    if (in)
    {
      for (int a = 0; a < 3; ++a)
        xi[a] = a < d->dim ? 2.0 * (x[a] - d->hx0[3 * (size_t)e + a]) /
                                     d->hh[3 * (size_t)e + a] -
                                 1.0
                           : 0.0;
      return e;
    }
  }
  return -1;
}

// phi_n(x) over the element's nodes n = i + Nq (j + Nq k)
void node_weights(const bfam_gpu_domain_t *d, const double *xi, double *wn)
{
  const int Nq = d->Nq;
  std::vector<double> p[3];
  for (int a = 0; a < 3; ++a)
  {
    p[a].assign(Nq, 1.0);
    if (a < d->dim)
      lagrange(d->hr.data(), Nq, xi[a], p[a].data());
  }
  for (int n = 0; n < d->Np; ++n)
  {
    const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
    wn[n] = p[0][i] * p[1][j] * (d->dim == 3 ? p[2][k] : 1.0);
  }
}

PostView post_view(bfam_gpu_domain_t *d, int cur, double dt)
{
  PostView p;
  p.q = d->q[cur];
  p.fs = d->fs;
  p.Np = d->Np;
  p.nfld = d->NFLD;
  p.nrecv = d->nrecv;
  p.max_samples = d->max_samples;
  p.relem = d->recv_elem;
  p.rw = d->recv_w;
  p.seis = d->seis;
  p.clock = d->clock;
  p.dt = dt;
  return p;
}

} // namespace

namespace bfam_b200
{
namespace host
{

int set_clock(bfam_gpu_domain_t *d, double t, int reset)
{
  dg_set_clock_kernel<<<1, 1, 0, d->stream>>>(d->clock, t, reset ? 3 : 1);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  CUDA_TRY(cudaGetLastError());
  d->clock_valid = true;
  return 0;
}

int launch_post(bfam_gpu_domain_t *d, int cur, double dt)
{
  dg_post_step_one<<<1, POST_THREADS, 0, d->stream>>>(post_view(d, cur, dt));
  g_launches.fetch_add(1, std::memory_order_relaxed);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

} // namespace host
} // namespace bfam_b200

// ------------------------------------------------------------------ batch

struct bfam_gpu_batch
{
  struct Group
  {
    int dim = 0, N = 0, precision = 0, flux = 0;
    std::vector<int> doms; // indices into the batch's domain list
    std::vector<double> hops;
    std::vector<BatchTile> tiles;
    int tile = 0, ctas_per_sm = 0;
    int64_t nwork = 0; // elements of all levels
    DomainView *views[2] = {nullptr, nullptr}; // per batch parity
    // per launch level: (domain, element) work list, its length and grid
    std::vector<int2 *> work;
    std::vector<int64_t> nwork_l;
    std::vector<int> grid;
    int ahead = 0; // L2 prefetch distance of one-buffer tiles (work items)
    // no domain of the group has faces glued to another order, so level 0
    // holds no element with a coarse-side face (launched without that pass)
    bool level0_nc = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
  };
  int device = 0, sms = 0;
  int ns = 0;
  double A[6] = {0}, B[6] = {0}, C[7] = {0};
  std::vector<bfam_gpu_domain_t *> doms;
  std::vector<int> cur0;     // each domain's state buffer at batch parity 0
  std::vector<unsigned> gen; // each domain's extras generation in the views
  std::vector<double> t, dt; // per domain: time, step of the current views
  std::vector<Group> groups;
  PostView *post[2] = {nullptr, nullptr};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t fork = nullptr;
  cudaEvent_t order = nullptr; // orders the batch against the domains' streams
  int parity = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool views_ok = false;
  std::vector<void *> allocs;
  // glue between domains: its two domains' indices in the batch
  std::vector<bfam_gpu_pglue_t *> pglues;
  std::vector<int> pglue_dom[2];
};

// Glue between two domains: per pair the glued face, its mortar slot and the
// side's operators, on the device.
struct bfam_gpu_pglue
{
  bfam_gpu_domain_t *d[2] = {nullptr, nullptr};
  int32_t K = 0;
  int Ng = 0, flux = 0, device = 0;
  std::vector<int32_t> entries[2]; // boundary-list entries (host)
  int32_t *elem[2] = {nullptr, nullptr}, *slot[2] = {nullptr, nullptr};
  int8_t *face[2] = {nullptr, nullptr};
  double *I[2] = {nullptr, nullptr}, *P[2] = {nullptr, nullptr};
  std::vector<void *> allocs;
};

namespace
{

// allocation ordered on the batch's stream, complete on return
int batch_alloc(bfam_gpu_batch_t *b, void **p, size_t bytes)
{
  cudaError_t e = pool_alloc(p, bytes ? bytes : 16, b->device, b->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return fail(BFAM_GPU_ENOMEM, "batch cudaMalloc(%zu): %s", bytes,
                cudaGetErrorString(e));
  }
  b->allocs.push_back(*p);
  return 0;
}

void batch_release(bfam_gpu_batch_t *b)
{
  if (!b)
    return;
  cudaSetDevice(b->device);
  for (int i = 0; i < 2; ++i)
    if (b->graph[i])
      cudaGraphExecDestroy(b->graph[i]);
  for (auto &g : b->groups)
  {
    if (g.stream)
      cudaStreamDestroy(g.stream);
    if (g.done)
      cudaEventDestroy(g.done);
  }
  if (b->fork)
    cudaEventDestroy(b->fork);
  if (b->order)
    cudaEventDestroy(b->order);
  // after the last step on the batch's stream (the groups' streams join it)
  for (void *p : b->allocs)
    cudaFreeAsync(p, b->stream);
  if (b->own_stream && b->stream)
    cudaStreamDestroy(b->stream);
  delete b;
}

void drop_graphs(bfam_gpu_batch_t *b)
{
  for (int i = 0; i < 2; ++i)
    if (b->graph[i])
    {
      cudaGraphExecDestroy(b->graph[i]);
      b->graph[i] = nullptr;
    }
}

int choose_grid(bfam_gpu_batch_t *b, bfam_gpu_batch_t::Group &g)
{
  const BatchTile &t = g.tiles[g.tile];
  CUDA_TRY(t.prepare());
  int occ = t.occupancy();
  if (occ <= 0)
    return fail(BFAM_GPU_EUNSUPPORTED,
                "tile %d (%d threads) of order %d does not fit on an SM",
                g.tile, t.NT, g.N);
  const int per_sm = g.ctas_per_sm > 0 && g.ctas_per_sm < occ ? g.ctas_per_sm
                                                               : occ;
  const int64_t full = (int64_t)per_sm * b->sms;
  // a persistent grid for two-buffer tiles; one CTA per work item for
  // one-buffer tiles
  const bool persistent = t.NBUF == 2;
  // L2 lookahead in work items: half a wave of resident elements
  g.ahead = persistent ? 0
                       : (int)std::min<int64_t>(full * t.EPC / 2, INT32_MAX);
  g.grid.resize(g.nwork_l.size());
  for (size_t l = 0; l < g.nwork_l.size(); ++l)
    g.grid[l] = (int)(persistent ? (g.nwork_l[l] > full ? full : g.nwork_l[l])
                                 : (g.nwork_l[l] + t.EPC - 1) / t.EPC);
  return 0;
}

// views (both parities) and post views from the domains' current buffers
// and time steps
int upload_views(bfam_gpu_batch_t *b)
{
  const int nd = (int)b->doms.size();
  // earlier steps may still read the view arrays
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < nd; ++i)
  {
    b->cur0[i] = b->doms[i]->cur;
    b->gen[i] = b->doms[i]->extras_gen;
  }
  for (auto &g : b->groups)
    for (int p = 0; p < 2; ++p)
    {
      std::vector<DomainView> v(g.doms.size());
      for (size_t k = 0; k < g.doms.size(); ++k)
      {
        const int i = g.doms[k];
        v[k] = view(b->doms[i], (b->cur0[i] + p) & 1);
        v[k].dt = b->dt[i];
      }
      CUDA_TRY(cudaMemcpy(g.views[p], v.data(), v.size() * sizeof(DomainView),
                          cudaMemcpyHostToDevice));
    }
  // post views: the state after a step from parity p is at parity p + ns
  for (int p = 0; p < 2; ++p)
  {
    std::vector<PostView> pv(nd);
    for (int i = 0; i < nd; ++i)
      pv[i] = post_view(b->doms[i], (b->cur0[i] + p + b->ns) & 1, b->dt[i]);
    CUDA_TRY(cudaMemcpy(b->post[p], pv.data(), nd * sizeof(PostView),
                        cudaMemcpyHostToDevice));
  }
  b->parity = 0;
  b->views_ok = true;
  drop_graphs(b);
  return 0;
}

// one step from batch parity p: every stage of every group, then the
// post-step kernel over all domains
int issue_step_glued(bfam_gpu_batch_t *b, int p);
int issue_step(bfam_gpu_batch_t *b, int p)
{
  if (!b->pglues.empty())
    return issue_step_glued(b, p);
  CUDA_TRY(cudaEventRecord(b->fork, b->stream));
  int launches = 0;
  for (auto &g : b->groups)
  {
    CUDA_TRY(cudaStreamWaitEvent(g.stream, b->fork, 0));
    const BatchTile &t = g.tiles[g.tile];
    for (int s = 0; s < b->ns; ++s)
    {
      StageParams sp;
      sp.A = b->A[s];
      sp.B = b->B[s];
      sp.dt = 0;
      sp.C = b->C[s];
      sp.first_stage = s == 0;
      sp.flux = g.flux;
      sp.ahead = g.ahead;
      // levels in order: coarse elements after the fine ones across their
      // hanging faces
      for (size_t l = 0; l < g.work.size(); ++l)
      {
        (l == 0 && g.level0_nc ? t.launch_nc : t.launch)(
            g.views[(p + s) & 1], g.work[l], (int)g.nwork_l[l], sp,
            g.hops.data(), g.grid[l], g.stream);
        CUDA_TRY(cudaGetLastError());
        ++launches;
      }
    }
    CUDA_TRY(cudaEventRecord(g.done, g.stream));
    CUDA_TRY(cudaStreamWaitEvent(b->stream, g.done, 0));
  }
  dg_post_step_kernel<<<(int)b->doms.size(), POST_THREADS, 0, b->stream>>>(
      b->post[p]);
  CUDA_TRY(cudaGetLastError());
  ++launches;
  g_launches.fetch_add(launches, std::memory_order_relaxed);
  return 0;
}

int launches_per_step(const bfam_gpu_batch_t *b)
{
  int n = 1 + b->ns * (int)b->pglues.size();
  for (const auto &g : b->groups)
    n += b->ns * (int)g.work.size();
  return n;
}

// the coupling kernel's view of glue k at state parity par
PGlueView pglue_view(const bfam_gpu_batch_t *b, size_t k, int par)
{
  const bfam_gpu_pglue_t *g = b->pglues[k];
  PGlueView v;
  for (int sd = 0; sd < 2; ++sd)
  {
    const int i = b->pglue_dom[sd][k];
    const bfam_gpu_domain_t *d = b->doms[i];
    PGlueSide &S = v.s[sd];
    S.q = d->q[(b->cur0[i] + par) & 1];
    S.fs = d->fs;
    S.N = d->N;
    S.ed = d->ed;
    S.mbuf = d->mbuf;
    S.elem = g->elem[sd];
    S.face = g->face[sd];
    S.slot = g->slot[sd];
    S.I = g->I[sd];
    S.P = g->P[sd];
  }
  v.K = g->K;
  v.Ng = g->Ng;
  v.flux = g->flux;
  return v;
}

// With glue between domains the groups meet at every stage: the coupling
// launches read every glued domain's stage input and fill the glued faces'
// slots before any element launch of the stage.
int issue_step_glued(bfam_gpu_batch_t *b, int p)
{
  int launches = 0;
  for (int s = 0; s < b->ns; ++s)
  {
    const int par = (p + s) & 1;
    for (size_t k = 0; k < b->pglues.size(); ++k)
    {
      const PGlueView v = pglue_view(b, k, par);
      if (b->doms[0]->dim == 3)
        dg_pglue_kernel<3><<<v.K, PGLUE_THREADS, 0, b->stream>>>(v);
      else
        dg_pglue_kernel<2><<<v.K, PGLUE_THREADS, 0, b->stream>>>(v);
      CUDA_TRY(cudaGetLastError());
      ++launches;
    }
    CUDA_TRY(cudaEventRecord(b->fork, b->stream));
    for (auto &g : b->groups)
    {
      CUDA_TRY(cudaStreamWaitEvent(g.stream, b->fork, 0));
      const BatchTile &t = g.tiles[g.tile];
      StageParams sp;
      sp.A = b->A[s];
      sp.B = b->B[s];
      sp.dt = 0;
      sp.C = b->C[s];
      sp.first_stage = s == 0;
      sp.flux = g.flux;
      sp.ahead = g.ahead;
      for (size_t l = 0; l < g.work.size(); ++l)
      {
        (l == 0 && g.level0_nc ? t.launch_nc : t.launch)(
            g.views[par], g.work[l], (int)g.nwork_l[l], sp, g.hops.data(),
            g.grid[l], g.stream);
        CUDA_TRY(cudaGetLastError());
        ++launches;
      }
      CUDA_TRY(cudaEventRecord(g.done, g.stream));
      CUDA_TRY(cudaStreamWaitEvent(b->stream, g.done, 0));
    }
  }
  dg_post_step_kernel<<<(int)b->doms.size(), POST_THREADS, 0, b->stream>>>(
      b->post[p]);
  CUDA_TRY(cudaGetLastError());
  ++launches;
  g_launches.fetch_add(launches, std::memory_order_relaxed);
  return 0;
}

// every glued face of the batch's domains joined by exactly one of its glues,
// and glued domains stepping with one time step
int check_glue(const bfam_gpu_batch_t *b, const double *dt)
{
  const int nd = (int)b->doms.size();
  std::vector<std::vector<int>> used(nd);
  for (int i = 0; i < nd; ++i)
    used[i].assign(b->doms[i]->bslot.size(), 0);
  for (size_t k = 0; k < b->pglues.size(); ++k)
  {
    const int i0 = b->pglue_dom[0][k], i1 = b->pglue_dom[1][k];
    if (dt[i0] != dt[i1] || b->t[i0] != b->t[i1])
      return fail(BFAM_GPU_EINVAL,
                  "glued domains %d and %d step with different times or time "
                  "steps",
                  i0, i1);
    for (int sd = 0; sd < 2; ++sd)
      for (int32_t e : b->pglues[k]->entries[sd])
        ++used[b->pglue_dom[sd][k]][e];
  }
  for (int i = 0; i < nd; ++i)
    for (size_t e = 0; e < used[i].size(); ++e)
      if ((b->doms[i]->bslot[e] >= 0) != (used[i][e] == 1))
        return fail(BFAM_GPU_EINVAL,
                    "domain %d: glued face (boundary entry %zu) is joined by "
                    "%d glues of the batch",
                    i, e, used[i][e]);
  return 0;
}

} // namespace

extern "C" {

// ---------------------------------------------------- source, receivers

int bfam_gpu_domain_set_source(bfam_gpu_domain_t *d,
                               const bfam_gpu_source_t *src)
{
  if (!d)
    return fail(BFAM_GPU_EINVAL, "NULL domain");
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (!src)
  {
    dev_free(d, d->src_w_alloc);
    d->src_w_alloc = nullptr;
    d->src = PointSource{-1, nullptr, {0, 0, 0}, 0, 0};
    ++d->extras_gen;
    return 0;
  }
  if (int rc = host_geometry(d))
    return rc;
  double xi[3];
  const int e = locate(d, src->x, xi);
  if (e < 0)
    return fail(BFAM_GPU_EINVAL, "source point (%g, %g, %g) lies in no element",
                src->x[0], src->x[1], src->x[2]);
  // phi_n(x_s) / (w_n J), J = prod_a h_a / 2
  std::vector<double> wn(d->Np);
  node_weights(d, xi, wn.data());
  double J = 1.0;
  for (int a = 0; a < d->dim; ++a)
    J *= 0.5 * d->hh[3 * (size_t)e + a];
  const int Nq = d->Nq;
  for (int n = 0; n < d->Np; ++n)
  {
    const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
    const double w = d->hw[i] * d->hw[j] * (d->dim == 3 ? d->hw[k] : 1.0);
    wn[n] /= w * J;
  }
  if (!d->src_w_alloc)
  {
    int rc = dev_alloc(d, &d->src_w_alloc, sizeof(double) * d->Np);
    if (rc)
      return rc;
  }
  CUDA_TRY(cudaMemcpy(d->src_w_alloc, wn.data(), sizeof(double) * d->Np,
                      cudaMemcpyHostToDevice));
  d->src.elem = e;
  d->src.w = static_cast<const double *>(d->src_w_alloc);
  for (int a = 0; a < 3; ++a)
    d->src.force[a] = a < d->dim ? src->force[a] : 0.0;
  d->src.f0 = src->f0;
  d->src.t0 = src->t0;
  ++d->extras_gen;
  return 0;
}

int bfam_gpu_domain_set_receivers(bfam_gpu_domain_t *d, int nrecv,
                                  const double *x, int max_samples)
{
  if (!d || nrecv < 0 || (nrecv > 0 && (!x || max_samples <= 0)))
    return fail(BFAM_GPU_EINVAL, "bad receiver arguments");
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (int rc = host_geometry(d))
    return rc;
  std::vector<int> elem(nrecv);
  std::vector<double> w((size_t)nrecv * d->Np);
  for (int r = 0; r < nrecv; ++r)
  {
    double xi[3];
    elem[r] = locate(d, x + 3 * r, xi);
    if (elem[r] < 0)
      return fail(BFAM_GPU_EINVAL, "receiver %d (%g, %g, %g) lies in no element",
                  r, x[3 * r], x[3 * r + 1], x[3 * r + 2]);
    node_weights(d, xi, w.data() + (size_t)r * d->Np);
  }
  dev_free(d, d->recv_elem);
  dev_free(d, d->recv_w);
  dev_free(d, d->seis);
  d->recv_elem = nullptr;
  d->recv_w = nullptr;
  d->seis = nullptr;
  d->nrecv = 0;
  d->max_samples = 0;
  ++d->extras_gen;
  if (nrecv == 0)
    return 0;
  int rc = upload(d, &d->recv_elem, elem.data(), elem.size());
  if (!rc)
    rc = upload(d, &d->recv_w, w.data(), w.size());
  if (!rc)
    rc = dev_alloc(d, (void **)&d->seis,
                   sizeof(double) * (size_t)max_samples * nrecv * d->NFLD);
  if (rc)
    return rc;
  d->nrecv = nrecv;
  d->max_samples = max_samples;
  // samples restart at zero; the clock keeps its time
  dg_set_clock_kernel<<<1, 1, 0, d->stream>>>(d->clock, 0.0, 2);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int bfam_gpu_domain_get_seismograms(bfam_gpu_domain_t *d, double *out,
                                    int *nsamples)
{
  if (!d || !nsamples)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(d->device));
  DomainClock c;
  CUDA_TRY(cudaMemcpyAsync(&c, d->clock, sizeof(c), cudaMemcpyDeviceToHost,
                           d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  const int n = c.nsamp < d->max_samples ? c.nsamp : d->max_samples;
  *nsamples = n;
  if (n > 0 && out)
    CUDA_TRY(cudaMemcpy(out, d->seis,
                        sizeof(double) * (size_t)n * d->nrecv * d->NFLD,
                        cudaMemcpyDeviceToHost));
  return 0;
}

// ---------------------------------------------------------------- tiles

int bfam_gpu_tile_count(int dim, int N)
{
  return (int)tiles(dim, N, BFAM_GPU_PRECISION_FP64).size();
}

int bfam_gpu_tile_shape(int dim, int N, int tile, int *threads, int *min_ctas)
{
  const auto t = tiles(dim, N, BFAM_GPU_PRECISION_FP64);
  if (tile < 0 || tile >= (int)t.size() || !threads || !min_ctas)
    return fail(BFAM_GPU_EINVAL, "no tile %d for dim %d order %d", tile, dim,
                N);
  *threads = t[tile].NT;
  *min_ctas = t[tile].MINB;
  return 0;
}

int bfam_gpu_tile_elements(int dim, int N, int tile)
{
  const auto t = tiles(dim, N, BFAM_GPU_PRECISION_FP64);
  if (tile < 0 || tile >= (int)t.size())
    return fail(BFAM_GPU_EINVAL, "no tile %d for dim %d order %d", tile, dim,
                N);
  return t[tile].EPC;
}

// ---------------------------------------------------------------- batch

int bfam_gpu_batch_create(bfam_gpu_domain_t *const *doms, int ndom,
                          int method, const double *t0,
                          bfam_gpu_batch_t **out)
{
  if (!out)
    return fail(BFAM_GPU_EINVAL, "out is NULL");
  *out = nullptr;
  if (!doms || ndom <= 0)
    return fail(BFAM_GPU_EINVAL, "need at least one domain");
  for (int i = 0; i < ndom; ++i)
  {
    if (!doms[i])
      return fail(BFAM_GPU_EINVAL, "domain %d is NULL", i);
    if (doms[i]->device != doms[0]->device)
      return fail(BFAM_GPU_EINVAL, "domains on different devices");
    for (int j = 0; j < i; ++j)
      if (doms[j] == doms[i])
        return fail(BFAM_GPU_EINVAL, "domain %d appears twice", i);
  }
  // LSRK coefficients from a stepper object (same tables)
  bfam_ts_lsrk_t *ts = nullptr;
  int rc = bfam_ts_lsrk_init(&ts, doms[0], method, 0.0);
  if (rc)
    return rc;
  bfam_gpu_batch_t *b = new bfam_gpu_batch_t();
  b->ns = ts->ns;
  std::memcpy(b->A, ts->A, sizeof(b->A));
  std::memcpy(b->B, ts->B, sizeof(b->B));
  std::memcpy(b->C, ts->C, sizeof(b->C));
  bfam_ts_lsrk_free(ts);
  b->device = doms[0]->device;
  b->doms.assign(doms, doms + ndom);
  b->cur0.assign(ndom, 0);
  b->gen.assign(ndom, 0);
  b->dt.assign(ndom, 0.0);
  b->t.assign(ndom, 0.0);
#define TRY(x)                                                                 \
  do                                                                           \
  {                                                                            \
    int rc_ = (x);                                                             \
    if (rc_)                                                                   \
    {                                                                          \
      batch_release(b);                                                        \
      return rc_;                                                              \
    }                                                                          \
  } while (0)
#define CTRY(x)                                                                \
  do                                                                           \
  {                                                                            \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess)                                                     \
    {                                                                          \
      batch_release(b);                                                        \
      return fail(BFAM_GPU_ECUDA, "%s: %s", #x, cudaGetErrorString(e_));       \
    }                                                                          \
  } while (0)
  CTRY(cudaSetDevice(b->device));
  CTRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount,
                              b->device));
  CTRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  b->own_stream = true;
  CTRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  CTRY(cudaEventCreateWithFlags(&b->order, cudaEventDisableTiming));
  // groups
  std::map<std::tuple<int, int, int, int, std::vector<double>>, int> key;
  for (int i = 0; i < ndom; ++i)
  {
    bfam_gpu_domain_t *d = doms[i];
    auto k = std::make_tuple(d->dim, d->N, d->precision, d->flux, d->hops);
    auto it = key.find(k);
    int g;
    if (it == key.end())
    {
      g = (int)b->groups.size();
      key.emplace(k, g);
      b->groups.emplace_back();
      auto &G = b->groups.back();
      G.dim = d->dim;
      G.N = d->N;
      G.precision = d->precision;
      G.flux = d->flux;
      G.hops = d->hops;
      G.tiles = tiles(d->dim, d->N, d->precision);
      if (G.tiles.empty())
      {
        batch_release(b);
        return fail(BFAM_GPU_EUNSUPPORTED, "no batch kernel for dim %d order %d",
                    d->dim, d->N);
      }
    }
    else
      g = it->second;
    b->groups[g].doms.push_back(i);
    b->groups[g].nwork += d->K;
  }
  for (auto &G : b->groups)
  {
    if (G.nwork > INT32_MAX)
    {
      batch_release(b);
      return fail(BFAM_GPU_EINVAL, "group of order %d has %lld elements",
                  G.N, (long long)G.nwork);
    }
    int nl = 1;
    G.level0_nc = true;
    for (int i : G.doms)
    {
      nl = std::max(nl, doms[i]->nlevels);
      if (doms[i]->nglued)
        G.level0_nc = false;
    }
    for (int l = 0; l < nl; ++l)
    {
      // level l of every domain, domain-major
      std::vector<int2> work;
      for (size_t k = 0; k < G.doms.size(); ++k)
      {
        const bfam_gpu_domain_t *d = doms[G.doms[k]];
        if (d->nlevels == 1)
        {
          if (l == 0)
            for (int32_t e = 0; e < d->K; ++e)
              work.push_back(make_int2((int)k, e));
        }
        else if (l < d->nlevels)
          for (int32_t j = d->level_off[l]; j < d->level_off[l + 1]; ++j)
            work.push_back(make_int2((int)k, d->helist[j]));
      }
      if (work.empty())
        continue;
      int2 *dw = nullptr;
      TRY(batch_alloc(b, (void **)&dw, work.size() * sizeof(int2)));
      CTRY(cudaMemcpy(dw, work.data(), work.size() * sizeof(int2),
                      cudaMemcpyHostToDevice));
      G.work.push_back(dw);
      G.nwork_l.push_back((int64_t)work.size());
    }
    for (int p = 0; p < 2; ++p)
      TRY(batch_alloc(b, (void **)&G.views[p],
                      G.doms.size() * sizeof(DomainView)));
    CTRY(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
    CTRY(cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming));
    TRY(choose_grid(b, G));
  }
  for (int p = 0; p < 2; ++p)
    TRY(batch_alloc(b, (void **)&b->post[p], ndom * sizeof(PostView)));
  // device clocks: set from t0, or kept (read back) without it
  for (int i = 0; i < ndom; ++i)
  {
    if (t0)
    {
      b->t[i] = t0[i];
      dg_set_clock_kernel<<<1, 1, 0, doms[i]->stream>>>(doms[i]->clock, t0[i],
                                                         1);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      CTRY(cudaGetLastError());
    }
    else
    {
      DomainClock c;
      CTRY(cudaMemcpyAsync(&c, doms[i]->clock, sizeof(c),
                           cudaMemcpyDeviceToHost, doms[i]->stream));
      CTRY(cudaStreamSynchronize(doms[i]->stream));
      b->t[i] = c.time;
    }
    doms[i]->clock_valid = true;
  }
  for (int i = 0; i < ndom; ++i)
    CTRY(cudaStreamSynchronize(doms[i]->stream));
#undef CTRY
#undef TRY
  *out = b;
  return 0;
}

int bfam_gpu_batch_set_stream(bfam_gpu_batch_t *b, void *stream)
{
  if (!b)
    return fail(BFAM_GPU_EINVAL, "NULL batch");
  CUDA_TRY(cudaSetDevice(b->device));
  if (b->own_stream && b->stream)
  {
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    cudaStreamDestroy(b->stream);
    b->own_stream = false;
    b->stream = nullptr;
  }
  if (stream)
    b->stream = static_cast<cudaStream_t>(stream);
  else
  {
    CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  drop_graphs(b);
  return 0;
}

int bfam_gpu_batch_step(bfam_gpu_batch_t *b, const double *dt, int nsteps,
                        int use_graph)
{
  if (!b || !dt || nsteps < 0)
    return fail(BFAM_GPU_EINVAL, "bad arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  const int nd = (int)b->doms.size();
  if (int rc = check_glue(b, dt))
    return rc;
  // the domains' buffers at the current parity, and the time steps, must be
  // those the views were built with
  bool stale = !b->views_ok;
  for (int i = 0; i < nd && !stale; ++i)
    stale = dt[i] != b->dt[i] ||
            b->doms[i]->cur != ((b->cur0[i] + b->parity) & 1) ||
            b->doms[i]->extras_gen != b->gen[i];
  // work queued on the domains' own streams (uploads) comes first
  for (int i = 0; i < nd; ++i)
  {
    CUDA_TRY(cudaEventRecord(b->order, b->doms[i]->stream));
    CUDA_TRY(cudaStreamWaitEvent(b->stream, b->order, 0));
  }
  if (stale)
  {
    for (int i = 0; i < nd; ++i)
      b->dt[i] = dt[i];
    int rc = upload_views(b);
    if (rc)
      return rc;
  }
  const int per_step = launches_per_step(b);
  for (int st = 0; st < nsteps; ++st)
  {
    const int p = b->parity;
    if (use_graph)
    {
      if (!b->graph[p])
      {
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(b->stream,
                                        cudaStreamCaptureModeThreadLocal));
        const int rc = issue_step(b, p);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc)
          return rc;
        if (ce != cudaSuccess)
          return fail(BFAM_GPU_ECUDA, "graph capture: %s",
                      cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&b->graph[p], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess)
          return fail(BFAM_GPU_ECUDA, "graph instantiate: %s",
                      cudaGetErrorString(ce));
        g_launches.fetch_sub(per_step, std::memory_order_relaxed);
      }
      CUDA_TRY(cudaGraphLaunch(b->graph[p], b->stream));
      g_launches.fetch_add(per_step, std::memory_order_relaxed);
    }
    else
    {
      const int rc = issue_step(b, p);
      if (rc)
        return rc;
    }
    b->parity = (p + b->ns) & 1;
    for (int i = 0; i < nd; ++i)
    {
      b->doms[i]->cur = (b->cur0[i] + b->parity) & 1;
      b->t[i] += dt[i];
    }
  }
  // and later work on the domains' streams (downloads) after the batch
  CUDA_TRY(cudaEventRecord(b->order, b->stream));
  for (int i = 0; i < nd; ++i)
    CUDA_TRY(cudaStreamWaitEvent(b->doms[i]->stream, b->order, 0));
  return 0;
}

int bfam_gpu_batch_time(const bfam_gpu_batch_t *b, int i, double *t)
{
  if (!b || !t || i < 0 || i >= (int)b->doms.size())
    return fail(BFAM_GPU_EINVAL, "bad arguments");
  *t = b->t[i];
  return 0;
}

int bfam_gpu_batch_sync(bfam_gpu_batch_t *b)
{
  if (!b)
    return fail(BFAM_GPU_EINVAL, "NULL batch");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (auto *d : b->doms)
  {
    int rc = bfam_gpu_domain_sync(d);
    if (rc)
      return rc;
  }
  return 0;
}

int bfam_gpu_batch_launches_per_step(const bfam_gpu_batch_t *b)
{
  return b ? launches_per_step(b) : 0;
}

int bfam_gpu_batch_free(bfam_gpu_batch_t *b)
{
  batch_release(b);
  return 0;
}

int bfam_gpu_batch_num_groups(const bfam_gpu_batch_t *b)
{
  return b ? (int)b->groups.size() : 0;
}

int bfam_gpu_batch_group_info(const bfam_gpu_batch_t *b, int g, int *dim,
                              int *N, int *precision, int64_t *elements)
{
  if (!b || g < 0 || g >= (int)b->groups.size())
    return fail(BFAM_GPU_EINVAL, "no group %d", g);
  const auto &G = b->groups[g];
  if (dim)
    *dim = G.dim;
  if (N)
    *N = G.N;
  if (precision)
    *precision = G.precision;
  if (elements)
    *elements = G.nwork;
  return 0;
}

int bfam_gpu_batch_set_tile(bfam_gpu_batch_t *b, int g, int tile,
                            int ctas_per_sm)
{
  if (!b || g < 0 || g >= (int)b->groups.size())
    return fail(BFAM_GPU_EINVAL, "no group %d", g);
  auto &G = b->groups[g];
  if (tile < 0 || tile >= (int)G.tiles.size() || ctas_per_sm < 0)
    return fail(BFAM_GPU_EINVAL, "no tile %d for order %d", tile, G.N);
  CUDA_TRY(cudaSetDevice(b->device));
  const int old_tile = G.tile, old_cps = G.ctas_per_sm;
  G.tile = tile;
  G.ctas_per_sm = ctas_per_sm;
  int rc = choose_grid(b, G);
  if (rc)
  {
    G.tile = old_tile;
    G.ctas_per_sm = old_cps;
    choose_grid(b, G);
    return rc;
  }
  drop_graphs(b);
  return 0;
}

} // extern "C"

// ------------------------------------------------------- glue between domains

namespace
{

void pglue_release(bfam_gpu_pglue_t *g)
{
  if (!g)
    return;
  cudaSetDevice(g->device);
  for (void *p : g->allocs)
    cudaFree(p);
  delete g;
}

template <typename T>
int pglue_upload(bfam_gpu_pglue_t *g, T **dst, const T *src, size_t n)
{
  cudaError_t e = cudaMalloc((void **)dst, n * sizeof(T));
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return fail(BFAM_GPU_ENOMEM, "glue cudaMalloc: %s", cudaGetErrorString(e));
  }
  g->allocs.push_back(*dst);
  CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// a side's operators: identity (NULL, or given) when N == Ng, otherwise an
// interpolation I and projection P with P I = identity (true of every
// interpolation to a finer LGL grid and the L2 projection back)
int check_glue_ops(int N, int Ng, const double *I, const double *P,
                   const char *side)
{
  const int n = N + 1, m = Ng + 1;
  if (N == Ng)
  {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
      {
        const double id = i == j ? 1.0 : 0.0;
        if ((I && std::fabs(I[i + n * j] - id) > 1e-13) ||
            (P && std::fabs(P[i + n * j] - id) > 1e-13))
          return fail(BFAM_GPU_EINVAL,
                      "glue side %s has the glue order but its operators are "
                      "not identities",
                      side);
      }
    return 0;
  }
  if (!I || !P)
    return fail(BFAM_GPU_EINVAL,
                "glue side %s (order %d < glue order %d) needs both operators",
                side, N, Ng);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
    {
      double s = 0; // (P I)(i, j): P is n x m, I is m x n
      for (int k = 0; k < m; ++k)
        s += P[i + n * k] * I[k + m * j];
      if (std::fabs(s - (i == j ? 1.0 : 0.0)) > 1e-11)
        return fail(BFAM_GPU_EINVAL,
                    "glue side %s: projection after interpolation is not the "
                    "identity (operators do not match orders %d and %d)",
                    side, N, Ng);
    }
  return 0;
}

} // namespace

extern "C" {

int bfam_gpu_pglue_create(bfam_gpu_domain_t *dm, bfam_gpu_domain_t *dp,
                          const bfam_gpu_pglue_desc_t *desc,
                          bfam_gpu_pglue_t **out)
{
  if (!out)
    return fail(BFAM_GPU_EINVAL, "out is NULL");
  *out = nullptr;
  if (!dm || !dp || !desc || desc->K <= 0 || !desc->bm || !desc->bp)
    return fail(BFAM_GPU_EINVAL, "bad glue arguments");
  if (dm == dp)
    return fail(BFAM_GPU_EINVAL, "a glue joins two different domains");
  if (dm->device != dp->device || dm->dim != dp->dim || dm->flux != dp->flux)
    return fail(BFAM_GPU_EINVAL,
                "glued domains differ in device, dimension or flux");
  const int Ng = desc->N_g;
  if (Ng < std::max(dm->N, dp->N) || Ng + 1 > PGLUE_MAXQ)
    return fail(BFAM_GPU_EINVAL,
                "glue order %d must be >= both orders (%d, %d) and <= %d", Ng,
                dm->N, dp->N, PGLUE_MAXQ - 1);
  if (int rc = check_glue_ops(dm->N, Ng, desc->I_m2g, desc->P_g2m, "m"))
    return rc;
  if (int rc = check_glue_ops(dp->N, Ng, desc->I_p2g, desc->P_g2p, "p"))
    return rc;
  bfam_gpu_domain_t *d[2] = {dm, dp};
  for (int sd = 0; sd < 2; ++sd)
    if (int rc = host_geometry(d[sd]))
      return rc;
  const int32_t K = desc->K;
  std::vector<int32_t> elem[2], slot[2];
  std::vector<int8_t> face[2];
  std::vector<char> seen[2];
  for (int sd = 0; sd < 2; ++sd)
  {
    elem[sd].resize(K);
    slot[sd].resize(K);
    face[sd].resize(K);
    seen[sd].assign(d[sd]->bslot.size(), 0);
  }
  for (int32_t k = 0; k < K; ++k)
  {
    const int32_t b[2] = {desc->bm[k], desc->bp[k]};
    for (int sd = 0; sd < 2; ++sd)
    {
      const bfam_gpu_domain_t *x = d[sd];
      if (b[sd] < 0 || b[sd] >= (int32_t)x->bslot.size() ||
          x->bslot[b[sd]] < 0)
        return fail(BFAM_GPU_EINVAL,
                    "glue pair %d: entry %d of side %c is not a glued face", k,
                    b[sd], sd ? 'p' : 'm');
      if (seen[sd][b[sd]]++)
        return fail(BFAM_GPU_EINVAL,
                    "glue pair %d: entry %d of side %c is glued twice", k,
                    b[sd], sd ? 'p' : 'm');
      elem[sd][k] = x->bE[b[sd]];
      face[sd][k] = x->bF[b[sd]];
      slot[sd][k] = x->bslot[b[sd]];
    }
    const int f = face[0][k], ax = f >> 1;
    if (face[1][k] != (f ^ 1))
      return fail(BFAM_GPU_EINVAL,
                  "glue pair %d joins faces %d and %d (need opposite faces "
                  "of one axis)",
                  k, f, face[1][k]);
    // the two faces cover the same extent along the face (glue orientation
    // 0, same size)
    for (int a = 0; a < dm->dim; ++a)
    {
      if (a == ax)
        continue;
      const size_t i0 = 3 * (size_t)elem[0][k] + a,
                   i1 = 3 * (size_t)elem[1][k] + a;
      const double scale = std::max(dm->hh[i0], dp->hh[i1]);
      if (std::fabs(dm->hx0[i0] - dp->hx0[i1]) > 1e-12 * scale ||
          std::fabs(dm->hh[i0] - dp->hh[i1]) > 1e-12 * scale)
        return fail(BFAM_GPU_EINVAL,
                    "glue pair %d: the faces do not coincide along axis %d "
                    "(hanging or shifted faces are not supported)",
                    k, a);
    }
  }
  CUDA_TRY(cudaSetDevice(dm->device));
  bfam_gpu_pglue_t *g = new bfam_gpu_pglue_t();
  g->d[0] = dm;
  g->d[1] = dp;
  g->K = K;
  g->Ng = Ng;
  g->flux = dm->flux;
  g->device = dm->device;
  g->entries[0].assign(desc->bm, desc->bm + K);
  g->entries[1].assign(desc->bp, desc->bp + K);
  const double *ops[2][2] = {{desc->I_m2g, desc->P_g2m},
                             {desc->I_p2g, desc->P_g2p}};
  int rc = 0;
  for (int sd = 0; sd < 2 && !rc; ++sd)
  {
    const size_t n = (size_t)(d[sd]->N + 1) * (Ng + 1);
    rc = pglue_upload(g, &g->elem[sd], elem[sd].data(), K);
    if (!rc)
      rc = pglue_upload(g, &g->face[sd], face[sd].data(), K);
    if (!rc)
      rc = pglue_upload(g, &g->slot[sd], slot[sd].data(), K);
    // same order: identity, applied as a copy
    if (!rc && d[sd]->N != Ng)
      rc = pglue_upload(g, &g->I[sd], ops[sd][0], n);
    if (!rc && d[sd]->N != Ng)
      rc = pglue_upload(g, &g->P[sd], ops[sd][1], n);
  }
  if (rc)
  {
    pglue_release(g);
    return rc;
  }
  *out = g;
  return 0;
}

int bfam_gpu_pglue_free(bfam_gpu_pglue_t *g)
{
  pglue_release(g);
  return 0;
}

int bfam_gpu_batch_add_pglue(bfam_gpu_batch_t *b, bfam_gpu_pglue_t *g)
{
  if (!b || !g)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  int idx[2] = {-1, -1};
  for (int sd = 0; sd < 2; ++sd)
    for (size_t i = 0; i < b->doms.size(); ++i)
      if (b->doms[i] == g->d[sd])
        idx[sd] = (int)i;
  if (idx[0] < 0 || idx[1] < 0)
    return fail(BFAM_GPU_EINVAL, "a glued domain is not in the batch");
  for (auto *x : b->pglues)
    if (x == g)
      return fail(BFAM_GPU_EINVAL, "glue added twice");
  b->pglues.push_back(g);
  b->pglue_dom[0].push_back(idx[0]);
  b->pglue_dom[1].push_back(idx[1]);
  drop_graphs(b);
  return 0;
}

} // extern "C"
