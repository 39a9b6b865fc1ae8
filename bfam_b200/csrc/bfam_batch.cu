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
  batch_launch_fn launch = nullptr;
  batch_prepare_fn prepare = nullptr;
  batch_occupancy_fn occupancy = nullptr;
};

template <int DIM, int N, int NT, int MINB, typename CT> struct TileImpl
{
  static constexpr auto kernel =
      dg_stage_batch_kernel<DIM, N, NT, MINB, MODE_STAGE, CT,
                            nbuf<DIM, N, CT>()>;
  static void launch(const DomainView *v, const int2 *w, int nwork,
                     const StageParams &sp, const double *hops, int grid,
                     cudaStream_t st)
  {
    const DiffOp<N, CT> dop = make_diffop<N, CT>(hops);
    kernel<<<grid, NT, stage_smem_bytes<DIM, N, CT>(), st>>>(v, w, nwork, sp,
                                                             dop);
  }
  static cudaError_t prepare()
  {
    return cudaFuncSetAttribute((const void *)kernel,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)stage_smem_bytes<DIM, N, CT>());
  }
  static int occupancy()
  {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, kernel, NT, stage_smem_bytes<DIM, N, CT>()) != cudaSuccess)
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
    t.NBUF = nbuf<DIM, N, CT>();
    t.launch = launch;
    t.prepare = prepare;
    t.occupancy = occupancy;
    return t;
  }
};

// Tile shapes per order.  Tile 0 is the single-domain kernel's shape (its
// register budget sized for the CTAs the shared memory admits); the others
// trade registers for resident CTAs or threads for nodes per thread (N = 7:
// 384 threads, one per face node, over 512 nodes).
template <typename CT> std::vector<BatchTile> tiles_for(int dim, int N)
{
  std::vector<BatchTile> v;
#define T(D, NN, NT, MB) v.push_back(TileImpl<D, NN, NT, MB, CT>::make())
#define T0(D, NN) T(D, NN, (Shape<D, NN>::NT), (stage_min_ctas<D, NN, CT>()))
  if (dim == 3)
  {
    switch (N)
    {
    case 1: T0(3, 1); break;
    case 2: T0(3, 2); break;
    case 3: T0(3, 3); T(3, 3, 96, 4); T(3, 3, 128, 4); break;
    case 4: T0(3, 4); break;
    case 5: T0(3, 5); T(3, 5, 224, 1); T(3, 5, 256, 2); break;
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
};

namespace
{

int batch_alloc(bfam_gpu_batch_t *b, void **p, size_t bytes)
{
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
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
  if (b->own_stream && b->stream)
    cudaStreamDestroy(b->stream);
  for (void *p : b->allocs)
    cudaFree(p);
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
  g.grid.resize(g.nwork_l.size());
  for (size_t l = 0; l < g.nwork_l.size(); ++l)
    g.grid[l] = (int)(persistent && g.nwork_l[l] > full ? full : g.nwork_l[l]);
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
int issue_step(bfam_gpu_batch_t *b, int p)
{
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
      // levels in order: coarse elements after the fine ones across their
      // hanging faces
      for (size_t l = 0; l < g.work.size(); ++l)
      {
        t.launch(g.views[(p + s) & 1], g.work[l], (int)g.nwork_l[l], sp,
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
  int n = 1;
  for (const auto &g : b->groups)
    n += b->ns * (int)g.work.size();
  return n;
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
    for (int i : G.doms)
      nl = std::max(nl, doms[i]->nlevels);
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
