// C-ABI of the B200 device layer (declared in include/bfam_gpu.h).
//
// Host side: validates the bfam arrays handed over, turns vmapP and the
// glue grid into compact per-element neighbour tables, uploads geometry,
// material and operators, owns the device state and launches the fused
// stage kernel once per LSRK stage (optionally replayed from a CUDA graph).
#include "bfam_gpu.h"
#include "dg_energy.cuh"
#include "dg_geometry.cuh"
#include "dg_stage.cuh"
#include "gpu_internal.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

using namespace bfam_b200;
using namespace bfam_b200::host;

namespace bfam_b200
{
namespace host
{

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

} // namespace host
} // namespace bfam_b200

namespace
{

template <int DIM, int N, typename CT, int MODE>
constexpr auto single_kernel =
    dg_stage_kernel<DIM, N, Shape<DIM, N>::NT, stage_min_ctas<DIM, N, CT>(),
                    MODE, CT, nbuf<DIM, N, CT>()>;

// n work items on a persistent grid of `grid` CTAs
template <int DIM, int N, typename CT>
void stage_launch(const DomainView &v, int n, const StageParams &sp,
                  const double *hops, int mode, int grid, cudaStream_t stream)
{
  using S = Shape<DIM, N>;
  const DiffOp<N, CT> dop = make_diffop<N, CT>(hops);
  const size_t smem = stage_smem_bytes<DIM, N, CT>();
  if (mode == MODE_STAGE)
    single_kernel<DIM, N, CT, MODE_STAGE><<<grid, S::NT, smem, stream>>>(
        v, n, sp, dop);
  else if (mode == MODE_STAGE_NC)
    single_kernel<DIM, N, CT, MODE_STAGE_NC><<<grid, S::NT, smem, stream>>>(
        v, n, sp, dop);
  else
    single_kernel<DIM, N, CT, MODE_RHS><<<grid, S::NT, smem, stream>>>(
        v, n, sp, dop);
}

template <typename K> cudaError_t allow_smem(K kernel, int bytes)
{
  return cudaFuncSetAttribute((const void *)kernel,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              bytes);
}

// shared-memory opt-in, and the resident CTAs per SM of both modes
template <int DIM, int N, typename CT> cudaError_t stage_prepare(int *occ)
{
  using S = Shape<DIM, N>;
  const int smem = (int)stage_smem_bytes<DIM, N, CT>();
  cudaError_t e = allow_smem(single_kernel<DIM, N, CT, MODE_STAGE>, smem);
  if (e == cudaSuccess)
    e = allow_smem(single_kernel<DIM, N, CT, MODE_RHS>, smem);
  if (e == cudaSuccess)
    e = allow_smem(single_kernel<DIM, N, CT, MODE_STAGE_NC>, smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ[MODE_STAGE], single_kernel<DIM, N, CT, MODE_STAGE>, S::NT, smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ[MODE_RHS], single_kernel<DIM, N, CT, MODE_RHS>, S::NT, smem);
  return e;
}

template <int DIM, int N, typename CT> KernelSet make_set()
{
  using S = Shape<DIM, N>;
  KernelSet k;
  k.launch = stage_launch<DIM, N, CT>;
  k.prepare = stage_prepare<DIM, N, CT>;
  k.energy = dg_energy_kernel<DIM, N>;
  k.NT = S::NT;
  k.smem = stage_smem_bytes<DIM, N, CT>();
  k.nbuf = nbuf<DIM, N, CT>();
  return k;
}

} // namespace

namespace bfam_b200
{
namespace host
{

// precision: BFAM_GPU_PRECISION_FP64 (double) or _FP32 (float right-hand side)
bool kernel_set(int dim, int N, int precision, KernelSet *out)
{
#define BFAM_CASE(D, NN)                                                       \
  if (dim == D && N == NN)                                                     \
  {                                                                            \
    *out = precision == BFAM_GPU_PRECISION_FP32 ? make_set<D, NN, float>()     \
                                                : make_set<D, NN, double>();   \
    return true;                                                               \
  }
  BFAM_CASE(2, 1) BFAM_CASE(2, 2) BFAM_CASE(2, 3) BFAM_CASE(2, 4)
  BFAM_CASE(2, 5) BFAM_CASE(2, 6) BFAM_CASE(2, 7) BFAM_CASE(2, 8)
  BFAM_CASE(3, 1) BFAM_CASE(3, 2) BFAM_CASE(3, 3) BFAM_CASE(3, 4)
  BFAM_CASE(3, 5) BFAM_CASE(3, 6) BFAM_CASE(3, 7)
#undef BFAM_CASE
  return false;
}

} // namespace host
} // namespace bfam_b200

namespace
{

int gmask_host(int dim, int Nq, int f, int pn)
{
  const int N = Nq - 1;
  if (dim == 2)
  {
    switch (f)
    {
    case 0: return pn * Nq;
    case 1: return pn * Nq + N;
    case 2: return pn;
    default: return N * Nq + pn;
    }
  }
  const int a = pn % Nq, b = pn / Nq;
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

} // namespace

namespace bfam_b200
{
namespace host
{

// Domain and batch memory comes from a stream-ordered pool that this
// library creates per device and owns (not the device's default pool, whose
// settings other code in the process shares).  Freed blocks stay in the pool
// for reuse (release threshold: never): a server that creates and frees a
// domain per request then neither maps nor unmaps device memory, and a free
// does not wait for the device.  What the pool holds is returned to the
// device only when the process exits.
cudaMemPool_t library_pool(int device)
{
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  if (device < 0 || device >= 64)
    return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[device])
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess)
    {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      pools[device] = pool;
    }
    cudaGetLastError();
  }
  return pools[device];
}

// stream-ordered allocation from the library's pool (the device's default
// pool if the library's could not be created)
cudaError_t pool_alloc(void **p, size_t bytes, int device, cudaStream_t stream)
{
  cudaMemPool_t pool = library_pool(device);
  return pool ? cudaMallocFromPoolAsync(p, bytes, pool, stream)
              : cudaMallocAsync(p, bytes, stream);
}

// free device memory plus what the library's pool holds unused
size_t free_device_bytes(int device)
{
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
    return 0;
  cudaMemPool_t pool = library_pool(device);
  uint64_t reserved = 0, used = 0;
  if (pool &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent,
                              &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) ==
          cudaSuccess &&
      reserved > used)
    free_b += reserved - used;
  cudaGetLastError();
  return free_b;
}

// allocation ordered on the domain's stream, complete on return (usable
// from any stream)
int dev_alloc(bfam_gpu_domain_t *d, void **p, size_t bytes)
{
  bytes = bytes ? bytes : 16;
  if (d->budget && d->bytes + bytes > d->budget)
    return fail(BFAM_GPU_ENOMEM,
                "device budget exceeded: %zu + %zu bytes > budget %zu",
                d->bytes, bytes, d->budget);
  cudaError_t e = pool_alloc(p, bytes, d->device, d->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return fail(BFAM_GPU_ENOMEM, "device allocation of %zu bytes: %s", bytes,
                cudaGetErrorString(e));
  }
  d->allocs.push_back(*p);
  d->alloc_bytes.push_back(bytes);
  d->bytes += bytes;
  return 0;
}

void dev_free(bfam_gpu_domain_t *d, void *p)
{
  if (!p)
    return;
  for (size_t i = 0; i < d->allocs.size(); ++i)
    if (d->allocs[i] == p)
    {
      // ordered after the domain's work; batches make the domain's stream
      // wait for their steps, so it is also after every batch use
      cudaFreeAsync(p, d->stream);
      d->bytes -= d->alloc_bytes[i];
      d->allocs.erase(d->allocs.begin() + i);
      d->alloc_bytes.erase(d->alloc_bytes.begin() + i);
      return;
    }
}

int host_geometry(bfam_gpu_domain_t *d)
{
  if (!d->hx0.empty() || !d->gx0)
    return 0;
  std::vector<double> x0(3 * (size_t)d->K), h(3 * (size_t)d->K);
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  CUDA_TRY(cudaMemcpy(x0.data(), d->gx0, sizeof(double) * x0.size(),
                      cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(h.data(), d->gh, sizeof(double) * h.size(),
                      cudaMemcpyDeviceToHost));
  d->hx0.swap(x0);
  d->hh.swap(h);
  return 0;
}

void release(bfam_gpu_domain_t *d)
{
  if (!d)
    return;
  cudaSetDevice(d->device);
  for (auto &pl : d->prof_pending)
  {
    cudaEventDestroy(pl.t0);
    cudaEventDestroy(pl.t1);
  }
  for (cudaEvent_t ev : d->prof_free)
    cudaEventDestroy(ev);
  for (void *p : d->allocs)
    cudaFreeAsync(p, d->stream);
  d->allocs.clear();
  if (d->own_stream && d->stream)
    cudaStreamDestroy(d->stream);
  delete d;
}

DomainView view(bfam_gpu_domain_t *d, int in)
{
  DomainView v;
  v.K = d->K;
  v.fs = d->fs;
  v.qin = d->q[in];
  v.qout = d->q[in ^ 1];
  v.dq = d->dq;
  v.rhs = d->rhs;
  v.ed = d->ed;
  v.fdesc = d->fdesc;
  v.fcE = d->fcE;
  v.fslot = d->fslot;
  v.mbuf = d->mbuf;
  v.elist = nullptr;
  v.ops = d->ops;
  v.err = d->err;
  v.dt = 0;
  v.src = d->src;
  v.clock = d->clock;
  return v;
}

int launch_stage(bfam_gpu_domain_t *d, int in, double A, double B, double C,
                 double dt, int first, int mode)
{
  StageParams sp;
  sp.A = A;
  sp.B = B;
  sp.dt = dt;
  sp.C = C;
  sp.first_stage = first;
  sp.flux = d->flux;
  // one element per CTA: prefetch half a wave of resident CTAs ahead (about
  // half a CTA lifetime before the element's CTA starts)
  sp.ahead = d->ks.nbuf == 1 ? d->ks.occ[mode] * d->sms / 2 : 0;
  DomainView v = view(d, in);
  v.dt = dt;
  // one launch per level; level l's elements after level l-1's
  for (int l = 0; l < d->nlevels; ++l)
  {
    int n = d->K;
    if (d->nlevels > 1)
    {
      v.elist = d->elist + d->level_off[l];
      n = d->level_off[l + 1] - d->level_off[l];
    }
    if (n == 0)
      continue;
    // two element buffers: a persistent grid (every resident CTA slot)
    // whose CTAs overlap the next element's loads with the current one; one
    // buffer: one CTA per element, balanced by the block scheduler
    const int64_t slots = (int64_t)d->ks.occ[mode] * d->sms;
    const int grid = d->ks.nbuf == 2 && n > slots ? (int)slots : n;
    // the first level has no coarse-side faces (unless faces glued to
    // another domain, which are lifted like them, sit there)
    const int m = mode == MODE_STAGE && l == 0 && !d->nglued ? MODE_STAGE_NC
                                                             : mode;
    bfam_gpu_domain::ProfLaunch pl{};
    if (d->prof)
    {
      for (cudaEvent_t *ev : {&pl.t0, &pl.t1})
      {
        if (d->prof_free.empty())
          CUDA_TRY(cudaEventCreate(ev));
        else
        {
          *ev = d->prof_free.back();
          d->prof_free.pop_back();
        }
      }
      // algorithmic bytes: q read and the new q written, dq written, and
      // after the first stage dq read (right-hand side: q read, rhs written)
      const double per_dof = mode == MODE_RHS ? 16.0 : (first ? 24.0 : 32.0);
      pl.level = l;
      pl.elements = n;
      pl.bytes = per_dof * (double)n * d->Np * d->NFLD;
      CUDA_TRY(cudaEventRecord(pl.t0, d->stream));
    }
    d->ks.launch(v, n, sp, d->hops.data(), m, grid, d->stream);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    CUDA_TRY(cudaGetLastError());
    if (d->prof)
    {
      CUDA_TRY(cudaEventRecord(pl.t1, d->stream));
      d->prof_pending.push_back(pl);
    }
  }
  return 0;
}

// Move the finished launches' times into the per-level totals.
int prof_drain(bfam_gpu_domain_t *d)
{
  for (auto &pl : d->prof_pending)
  {
    CUDA_TRY(cudaEventSynchronize(pl.t1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, pl.t0, pl.t1));
    if ((int)d->prof_ms.size() <= pl.level)
    {
      d->prof_ms.resize(pl.level + 1, 0.0);
      d->prof_bytes.resize(pl.level + 1, 0.0);
      d->prof_launches.resize(pl.level + 1, 0);
      d->prof_elements.resize(pl.level + 1, 0);
    }
    d->prof_ms[pl.level] += ms;
    d->prof_bytes[pl.level] += pl.bytes;
    d->prof_launches[pl.level] += 1;
    d->prof_elements[pl.level] += pl.elements;
    d->prof_free.push_back(pl.t0);
    d->prof_free.push_back(pl.t1);
  }
  d->prof_pending.clear();
  return 0;
}

} // namespace host
} // namespace bfam_b200

extern "C" {

int bfam_gpu_last_error(char *buf, size_t len)
{
  if (buf && len)
  {
    strncpy(buf, g_err.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return (int)g_err.size();
}

int bfam_gpu_domain_profile(bfam_gpu_domain_t *d, int enable)
{
  if (!d)
    return fail(BFAM_GPU_EINVAL, "domain is NULL");
  CUDA_TRY(cudaSetDevice(d->device));
  int rc = prof_drain(d);
  if (rc)
    return rc;
  d->prof = enable != 0;
  d->prof_ms.clear();
  d->prof_bytes.clear();
  d->prof_launches.clear();
  d->prof_elements.clear();
  return 0;
}

int bfam_gpu_domain_kernel_stats(bfam_gpu_domain_t *d,
                                 bfam_gpu_kernel_stat_t *out, int max_levels,
                                 int *nlevels)
{
  if (!d || !nlevels || (max_levels > 0 && !out))
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(d->device));
  int rc = prof_drain(d);
  if (rc)
    return rc;
  const int n = (int)d->prof_ms.size();
  *nlevels = n;
  for (int l = 0; l < n && l < max_levels; ++l)
  {
    out[l].level = l;
    out[l].launches = d->prof_launches[l];
    out[l].elements = d->prof_elements[l];
    out[l].ms = d->prof_ms[l];
    out[l].alg_bytes = d->prof_bytes[l];
    out[l].gbs = d->prof_ms[l] > 0 ? d->prof_bytes[l] / (d->prof_ms[l] * 1e6) : 0;
  }
  return 0;
}

int bfam_gpu_trim_pool(int device, size_t keep_bytes)
{
  cudaMemPool_t pool = library_pool(device);
  if (!pool)
    return fail(BFAM_GPU_EINVAL, "no memory pool for device %d", device);
  CUDA_TRY(cudaMemPoolTrimTo(pool, keep_bytes));
  return 0;
}

int bfam_gpu_record_error(int code, const char *msg)
{
  return fail(code, "%s", msg ? msg : "");
}

uint64_t bfam_gpu_launch_count(void) { return g_launches.load(); }

static int create_domain(const bfam_gpu_volume_t *vol,
                         const bfam_gpu_glue_t *glue,
                         const bfam_gpu_boundary_t *bnd,
                         const bfam_gpu_quadrants_t *quads,
                         const bfam_gpu_options_t *opts,
                         bfam_gpu_domain_t **out);

int bfam_gpu_domain_create(const bfam_gpu_volume_t *vol,
                           const bfam_gpu_glue_t *glue,
                           const bfam_gpu_options_t *opts,
                           bfam_gpu_domain_t **out)
{
  return bfam_gpu_domain_create_with_boundary(vol, glue, nullptr, opts, out);
}

int bfam_gpu_domain_create_with_boundary(const bfam_gpu_volume_t *vol,
                                         const bfam_gpu_glue_t *glue,
                                         const bfam_gpu_boundary_t *bnd,
                                         const bfam_gpu_options_t *opts,
                                         bfam_gpu_domain_t **out)
{
  return create_domain(vol, glue, bnd, nullptr, opts, out);
}

int bfam_gpu_domain_create_from_quadrants(const bfam_gpu_volume_t *vol,
                                          const bfam_gpu_glue_t *glue,
                                          const bfam_gpu_boundary_t *bnd,
                                          const bfam_gpu_quadrants_t *quads,
                                          const bfam_gpu_options_t *opts,
                                          bfam_gpu_domain_t **out)
{
  if (out)
    *out = nullptr;
  if (!quads)
    return fail(BFAM_GPU_EINVAL, "quads is NULL");
  return create_domain(vol, glue, bnd, quads, opts, out);
}

namespace
{

// quadrant data: trees are boxes, every element a quadrant of its tree
int check_quadrants(const bfam_gpu_quadrants_t *qd, int dim, int32_t K)
{
  if (!qd->tree_x0 || !qd->tree_h || !qd->quads)
    return fail(BFAM_GPU_EINVAL, "a required quadrant array is NULL");
  const int32_t root = qd->root_len;
  if (root < 1 || root > (1 << 30) || (root & (root - 1)))
    return fail(BFAM_GPU_EINVAL, "root_len %d is not a power of two <= 2^30",
                root);
  if (qd->num_trees < 1)
    return fail(BFAM_GPU_EINVAL, "num_trees must be positive (got %d)",
                qd->num_trees);
  for (int32_t t = 0; t < qd->num_trees; ++t)
    for (int a = 0; a < dim; ++a)
    {
      const double x = qd->tree_x0[3 * (size_t)t + a],
                   h = qd->tree_h[3 * (size_t)t + a];
      if (!std::isfinite(x) || !std::isfinite(h) || !(h > 0))
        return fail(BFAM_GPU_EINVAL, "tree %d: bad box on axis %d", t, a);
    }
  int maxlevel = 0;
  while ((1 << maxlevel) < root)
    ++maxlevel;
  for (int32_t e = 0; e < K; ++e)
  {
    const int32_t *q = qd->quads + BFAM_GPU_NQUAD * (size_t)e;
    if (q[0] < 0 || q[0] >= qd->num_trees)
      return fail(BFAM_GPU_EINVAL, "element %d: tree %d out of range", e,
                  q[0]);
    if (q[1] < 0 || q[1] > maxlevel)
      return fail(BFAM_GPU_EINVAL, "element %d: level %d out of [0, %d]", e,
                  q[1], maxlevel);
    const int32_t len = root >> q[1];
    for (int a = 0; a < dim; ++a)
      if (q[2 + a] < 0 || q[2 + a] >= root || q[2 + a] % len)
        return fail(BFAM_GPU_EINVAL,
                    "element %d: coordinate %d on axis %d is not a level-%d "
                    "quadrant corner in [0, %d)",
                    e, q[2 + a], a, q[1], root);
  }
  return 0;
}

} // namespace

static int create_domain(const bfam_gpu_volume_t *vol,
                         const bfam_gpu_glue_t *glue,
                         const bfam_gpu_boundary_t *bnd,
                         const bfam_gpu_quadrants_t *quads,
                         const bfam_gpu_options_t *opts,
                         bfam_gpu_domain_t **out)
{
  if (!out)
    return fail(BFAM_GPU_EINVAL, "out is NULL");
  *out = nullptr;
  if (!vol || !opts)
    return fail(BFAM_GPU_EINVAL, "vol/opts is NULL");
  const int dim = vol->dim, N = vol->N;
  if (dim != 2 && dim != 3)
    return fail(BFAM_GPU_EINVAL, "dim must be 2 or 3 (got %d)", dim);
  if (vol->K <= 0)
    return fail(BFAM_GPU_EINVAL, "K must be positive (got %d)", vol->K);
  if (opts->precision != BFAM_GPU_PRECISION_FP64 &&
      opts->precision != BFAM_GPU_PRECISION_FP32)
    return fail(BFAM_GPU_EINVAL, "unknown precision %d", opts->precision);
  KernelSet ks;
  if (!kernel_set(dim, N, opts->precision, &ks))
    return fail(BFAM_GPU_EUNSUPPORTED, "order N=%d in %dD is not compiled in",
                N, dim);
  if (!vol->r || !vol->w || !vol->Dr || !vol->vmapM || !vol->vmapP ||
      (!quads && (!vol->x0 || !vol->h)) || !vol->rho || !vol->lambda ||
      !vol->mu)
    return fail(BFAM_GPU_EINVAL, "a required volume array is NULL");
  if (quads && check_quadrants(quads, dim, vol->K))
    return BFAM_GPU_EINVAL;
  if (opts->flux != BFAM_GPU_FLUX_UPWIND && opts->flux != BFAM_GPU_FLUX_CENTRAL)
    return fail(BFAM_GPU_EINVAL, "unknown flux %d", opts->flux);

  const int Nq = N + 1;
  const int Np = dim == 3 ? Nq * Nq * Nq : Nq * Nq;
  const int Nfp = dim == 3 ? Nq * Nq : Nq;
  const int NF = 2 * dim;
  const int NFLD = dim == 3 ? 9 : 5;
  const int32_t K = vol->K;
  if ((int64_t)K * Np > INT32_MAX)
    return fail(BFAM_GPU_EINVAL, "K*Np exceeds the int32 node index range");
  const int nperm = dim == 3 ? 8 : 2;

  // face-node tables: gm[f][pn] = volume node of face f's node pn
  std::vector<int32_t> gm((size_t)NF * Nfp);
  for (int f = 0; f < NF; ++f)
    for (int pn = 0; pn < Nfp; ++pn)
      gm[(size_t)f * Nfp + pn] = gmask_host(dim, Nq, f, pn);

  // ---- vmapM must be bfam's canonical face mask layout
  const size_t nmap = (size_t)K * NF * Nfp;
  for (int32_t e = 0; e < K; ++e)
    for (int f = 0; f < NF; ++f)
      for (int pn = 0; pn < Nfp; ++pn)
      {
        const size_t id = ((size_t)e * NF + f) * Nfp + pn;
        if (vol->vmapM[id] != e * Np + gm[(size_t)f * Nfp + pn])
          return fail(BFAM_GPU_EINVAL,
                      "vmapM[%zu] = %d is not element %d face %d node %d",
                      id, vol->vmapM[id], e, f, pn);
      }

  // ---- vmapP -> neighbour across the opposite face, or glue face.  The
  // element metric is diagonal (affine boxes, every tree aligned with the
  // brick), so a face can only meet its neighbour's opposite face with the
  // nodes in the same order (bfam's orientation 0, src/bfam.c:3630-3712); any
  // other pairing comes from a rotated tree, which this metric cannot
  // represent, and is refused.
  std::vector<int32_t> nbr((size_t)K * NF);
  std::vector<int8_t> nbrf((size_t)K * NF, 0);
  for (int32_t e = 0; e < K; ++e)
    for (int f = 0; f < NF; ++f)
    {
      const int32_t *P = vol->vmapP + ((size_t)e * NF + f) * Nfp;
      const int32_t *M = vol->vmapM + ((size_t)e * NF + f) * Nfp;
      bool self = true;
      for (int pn = 0; pn < Nfp && self; ++pn)
        self = P[pn] == M[pn];
      if (self)
      {
        nbr[(size_t)e * NF + f] = INT32_MIN; // filled from the glue grid
        continue;
      }
      if (P[0] < 0 || P[0] >= K * Np)
        return fail(BFAM_GPU_EINVAL, "vmapP out of range at element %d face %d",
                    e, f);
      const int32_t nb = P[0] / Np;
      const int fn = f ^ 1;
      const int32_t *g = gm.data() + (size_t)fn * Nfp;
      bool ok = true;
      for (int pn = 0; pn < Nfp && ok; ++pn)
        ok = P[pn] == nb * Np + g[pn];
      if (!ok)
      {
        // name the pairing if vmapP is some face of nb at all
        for (int f2 = 0; f2 < NF; ++f2)
        {
          std::vector<int32_t> want(Nfp), have(P, P + Nfp);
          for (int pn = 0; pn < Nfp; ++pn)
            want[pn] = nb * Np + gm[(size_t)f2 * Nfp + pn];
          std::sort(want.begin(), want.end());
          std::sort(have.begin(), have.end());
          if (want == have)
            return fail(BFAM_GPU_EUNSUPPORTED,
                        "element %d face %d meets face %d of element %d "
                        "%s: only aligned trees are supported (opposite "
                        "faces, orientation 0; the element metric is "
                        "diagonal)",
                        e, f, f2, nb,
                        f2 == fn ? "with permuted nodes" : "");
        }
        return fail(BFAM_GPU_EINVAL,
                    "vmapP of element %d face %d is not a face of element %d",
                    e, f, nb);
      }
      nbr[(size_t)e * NF + f] = nb;
      nbrf[(size_t)e * NF + f] = (int8_t)fn;
    }

  // ---- glue grid
  const int32_t Kg = glue ? glue->K : 0;
  const int NPc = dim == 3 ? 4 : 2;
  if (Kg < 0)
    return fail(BFAM_GPU_EINVAL, "glue K is negative");
  if (Kg > 0 && (!glue->EToEp || !glue->EToHp || !glue->EToOp ||
                 !glue->EToEm || !glue->EToFm || !glue->EToHm))
    return fail(BFAM_GPU_EINVAL, "a required glue array is NULL");
  for (int32_t g = 0; g < Kg;)
  {
    const int32_t e = glue->EToEm[g];
    const int f = glue->EToFm[g];
    const int h = glue->EToHm[g];
    if (e < 0 || e >= K || f < 0 || f >= NF || h < 0 || h > NPc)
      return fail(BFAM_GPU_EINVAL, "glue element %d has bad (E, F, H) = "
                  "(%d, %d, %d)", g, e, f, h);
    if (nbr[(size_t)e * NF + f] != INT32_MIN)
      return fail(BFAM_GPU_EINVAL,
                  "glue element %d sits on element %d face %d whose vmapP "
                  "does not point to itself",
                  g, e, f);
    const int cnt = h == 0 ? 1 : NPc;
    if (g + cnt > Kg)
      return fail(BFAM_GPU_EINVAL, "glue grid ends inside a hanging face");
    for (int p = 0; p < cnt; ++p)
    {
      const int32_t gg = g + p;
      if (glue->EToEm[gg] != e || glue->EToFm[gg] != f ||
          glue->EToHm[gg] != (h == 0 ? 0 : p + 1))
        return fail(BFAM_GPU_EINVAL,
                    "glue elements of element %d face %d are not in receive "
                    "order (element, face, hanging number)",
                    e, f);
      const int32_t pg = glue->EToEp[gg];
      if (pg < 0 || pg >= Kg || glue->EToEp[pg] != gg)
        return fail(BFAM_GPU_EINVAL,
                    "glue EToEp is not an involution at %d (local glue grid)",
                    gg);
      if (glue->EToHp[gg] != glue->EToHm[pg])
        return fail(BFAM_GPU_EINVAL, "glue EToHp[%d] disagrees with the "
                    "partner's EToHm", gg);
      if (glue->EToHm[gg] > 0 && glue->EToHm[pg] != 0)
        return fail(BFAM_GPU_EINVAL, "hanging piece %d pairs with another "
                    "hanging piece", gg);
      if (glue->EToOp[gg] < 0 || glue->EToOp[gg] >= nperm)
        return fail(BFAM_GPU_EINVAL, "glue orientation %d out of range",
                    glue->EToOp[gg]);
      if (glue->EToOp[gg] != 0 || glue->EToFm[pg] != (f ^ 1))
        return fail(BFAM_GPU_EUNSUPPORTED,
                    "glue element %d pairs face %d with face %d under "
                    "orientation %d: only aligned trees are supported "
                    "(opposite faces, orientation 0; the element metric is "
                    "diagonal)",
                    gg, f, glue->EToFm[pg], glue->EToOp[gg]);
    }
    nbr[(size_t)e * NF + f] = -1 - g;
    g += cnt;
  }
  // ---- boundary faces: self-mapped and not in the glue grid
  constexpr int32_t BOUNDARY = INT32_MIN + 1;
  std::vector<int8_t> bctype(nbr.size(), -1);
  std::vector<int32_t> bentry(nbr.size(), -1); // boundary-list entry per face
  if (bnd && bnd->K > 0)
  {
    if (!bnd->EToE || !bnd->EToF || !bnd->type)
      return fail(BFAM_GPU_EINVAL, "a required boundary array is NULL");
    for (int32_t b = 0; b < bnd->K; ++b)
    {
      const int32_t e = bnd->EToE[b];
      const int f = bnd->EToF[b];
      const int ty = bnd->type[b];
      if (e < 0 || e >= K || f < 0 || f >= NF)
        return fail(BFAM_GPU_EINVAL, "boundary face %d has bad (E, F) = (%d, %d)",
                    b, e, f);
      if (ty != BFAM_GPU_BC_FREE_SURFACE && ty != BFAM_GPU_BC_ABSORBING &&
          ty != BFAM_GPU_BC_GLUED)
        return fail(BFAM_GPU_EINVAL, "boundary face %d has unknown type %d", b,
                    ty);
      if (nbr[(size_t)e * NF + f] != INT32_MIN)
        return fail(BFAM_GPU_EINVAL,
                    "boundary face %d (element %d face %d) has a neighbour, a "
                    "glue element or a second boundary entry",
                    b, e, f);
      nbr[(size_t)e * NF + f] = BOUNDARY;
      bctype[(size_t)e * NF + f] = (int8_t)ty;
      bentry[(size_t)e * NF + f] = b;
    }
  }
  for (size_t i = 0; i < nbr.size(); ++i)
    if (nbr[i] == INT32_MIN)
      return fail(BFAM_GPU_EINVAL,
                  "element %zu face %zu maps to itself but has no glue "
                  "element or boundary entry",
                  i / NF, i % NF);

  // ---- mortar buffer slots: one per coarse-side glue element (piece), in
  // glue order, so that a coarse face's pieces have consecutive slots
  std::vector<int32_t> mslot(Kg > 0 ? Kg : 1, -1);
  int32_t nslot = 0;
  for (int32_t g = 0; g < Kg; ++g)
    if (glue->EToHm[g] > 0)
      mslot[g] = nslot++;
  // then, per glued face in boundary-list order, as many slots as a coarse
  // face has pieces: the glue between domains writes the first, the others
  // stay zero, so that the stage kernel lifts it like a coarse face
  const int32_t nbnd = bnd ? bnd->K : 0;
  std::vector<int32_t> bslot(nbnd, -1);
  for (int32_t b = 0; b < nbnd; ++b)
    if (bnd->type[b] == BFAM_GPU_BC_GLUED)
    {
      bslot[b] = nslot;
      nslot += NPc;
    }

  // ---- compact descriptors read by the kernel (layout in dg_common.cuh)
  std::vector<int2> fdesc((size_t)K * NF);
  std::vector<int32_t> fslot((size_t)K * NF, -1);
  for (size_t i = 0; i < fdesc.size(); ++i)
  {
    const int32_t nb = nbr[i];
    if (nb >= 0)
    {
      fdesc[i] = make_int2(nb, 0 | (nbrf[i] << 2));
      continue;
    }
    if (nb == BOUNDARY)
    {
      if (bctype[i] == BFAM_GPU_BC_GLUED)
        fdesc[i] = make_int2(bslot[bentry[i]], 2);
      else
        fdesc[i] = make_int2((int32_t)(i / NF), 3 | (bctype[i] << 2));
      continue;
    }
    const int32_t g0 = -1 - nb;
    if (glue->EToHm[g0] == 0)
    {
      const int32_t pg = glue->EToEp[g0];
      fdesc[i] = make_int2(glue->EToEm[pg], 1 | (glue->EToFm[pg] << 2) |
                                                (glue->EToHm[pg] << 8));
      if (glue->EToHm[pg] > 0)
        fslot[i] = mslot[pg];
    }
    else
      fdesc[i] = make_int2(mslot[g0], 2);
  }

  // an element lies on the fine side of at most DIM hanging faces (the faces
  // on its parent's boundary); the kernel's mortar scratch is sized for that
  for (int32_t e = 0; e < K; ++e)
  {
    int nf = 0;
    for (int f = 0; f < NF; ++f)
      nf += fslot[(size_t)e * NF + f] >= 0;
    if (nf > dim)
      return fail(BFAM_GPU_EUNSUPPORTED,
                  "element %d is on the fine side of %d hanging faces (a 2:1 "
                  "balanced forest has at most %d)",
                  e, nf, dim);
  }

  // ---- launch levels: an element with coarse faces runs after the fine
  // elements across them (which write its mortar slots); level 0 has no
  // coarse face
  std::vector<int> level(K, 0);
  int nlevels = 1;
  for (bool changed = Kg > 0; changed;)
  {
    changed = false;
    for (int32_t e = 0; e < K; ++e)
      for (int f = 0; f < NF; ++f)
      {
        const int2 ds = fdesc[(size_t)e * NF + f];
        if ((ds.y & 3) != 2 || nbr[(size_t)e * NF + f] == BOUNDARY)
          continue; // not a hanging face (a glued face's slot is written
                    // before the stage's element launches)
        const int32_t g0 = -1 - nbr[(size_t)e * NF + f];
        for (int p = 0; p < NPc; ++p)
        {
          const int32_t fine = glue->EToEm[glue->EToEp[g0 + p]];
          if (level[e] < level[fine] + 1)
          {
            level[e] = level[fine] + 1;
            changed = true;
            if (level[e] >= K)
              return fail(BFAM_GPU_EINVAL,
                          "hanging faces form a cycle (element %d)", e);
          }
        }
      }
  }
  for (int32_t e = 0; e < K; ++e)
    nlevels = std::max(nlevels, level[e] + 1);
  std::vector<int32_t> elist, level_off(nlevels + 1, 0);
  if (nlevels > 1)
  {
    for (int32_t e = 0; e < K; ++e)
      ++level_off[level[e] + 1];
    for (int l = 0; l < nlevels; ++l)
      level_off[l + 1] += level_off[l];
    elist.resize(K);
    std::vector<int32_t> pos(level_off.begin(), level_off.end() - 1);
    for (int32_t e = 0; e < K; ++e)
      elist[pos[level[e]]++] = e;
  }

  // ---- operators: Dr | interp[3] | proj[3] | w
  std::vector<double> ops(7 * Nq * Nq + Nq, 0.0);
  std::memcpy(ops.data(), vol->Dr, sizeof(double) * Nq * Nq);
  for (int k = 0; k < 6; ++k)
  {
    const double *src = nullptr;
    if (glue && Kg > 0)
      src = k < 3 ? glue->interpolation[k] : glue->projection[k - 3];
    double *dst = ops.data() + (1 + k) * Nq * Nq;
    if (src)
      std::memcpy(dst, src, sizeof(double) * Nq * Nq);
    else
    {
      if (Kg > 0 && (k % 3) != 0)
        return fail(BFAM_GPU_EINVAL, "glue operator %s[%d] is NULL",
                    k < 3 ? "interpolation" : "projection", k % 3);
      for (int i = 0; i < Nq; ++i)
        dst[i + Nq * i] = 1.0;
    }
    if ((k % 3) == 0 && src)
      for (int i = 0; i < Nq * Nq; ++i)
        if (std::fabs(dst[i] - ((i % (Nq + 1)) == 0 ? 1.0 : 0.0)) > 1e-12)
          return fail(BFAM_GPU_EUNSUPPORTED,
                      "non-identity same-level operator (glue order differs "
                      "from the volume order) is not supported");
  }
  // the kernels apply the top-half operators as reflections of the
  // bottom-half ones: A_top(m, i) = A_bot(N - m, N - i)
  for (int k : {1, 4})
  {
    const double *bot = ops.data() + (1 + k) * Nq * Nq;
    const double *top = ops.data() + (2 + k) * Nq * Nq;
    double amax = 0;
    for (int i = 0; i < Nq * Nq; ++i)
      amax = std::fmax(amax, std::fabs(bot[i]));
    for (int m = 0; m < Nq; ++m)
      for (int i = 0; i < Nq; ++i)
        if (std::fabs(top[m + Nq * i] - bot[(N - m) + Nq * (N - i)]) >
            1e-13 * (amax > 1 ? amax : 1))
          return fail(BFAM_GPU_EUNSUPPORTED,
                      "glue %s operators are not reflections of each other "
                      "(non-LGL glue grid)",
                      k == 1 ? "interpolation" : "projection");
  }
  std::memcpy(ops.data() + 7 * Nq * Nq, vol->w, sizeof(double) * Nq);

  // ---- per-element geometry and material
  std::vector<ElemData> ed(K);
  for (int32_t e = 0; e < K; ++e)
  {
    const double rho = vol->rho[e], la = vol->lambda[e], mu = vol->mu[e];
    if (!(rho > 0) || !(mu > 0) || !(la + 2 * mu > 0))
      return fail(BFAM_GPU_EINVAL,
                  "element %d: need rho > 0, mu > 0, lambda + 2 mu > 0", e);
    ElemData &x = ed[e];
    x.irho = 1.0 / rho;
    x.lam = la;
    x.mu = mu;
    x.Zp = std::sqrt(rho * (la + 2 * mu));
    x.Zs = std::sqrt(rho * mu);
    if (quads)
      continue; // the metric comes from the device geometry kernel
    for (int a = 0; a < 3; ++a)
    {
      const double h = a < dim ? vol->h[3 * e + a] : 1.0;
      if (!(h > 0))
        return fail(BFAM_GPU_EINVAL, "element %d has edge %d <= 0", e, a);
      (&x.rx)[a] = 2.0 / h;
    }
  }

  // ---- upwind flux constants of every face and glue element
  auto fconst = [&](int32_t me, int32_t nb) {
    return make_double4(ed[nb].Zp, 1.0 / (ed[me].Zp + ed[nb].Zp), ed[nb].Zs,
                        1.0 / (ed[me].Zs + ed[nb].Zs));
  };
  std::vector<double4> fcE((size_t)K * NF, make_double4(0, 0, 0, 0));
  for (size_t i = 0; i < fcE.size(); ++i)
    if ((fdesc[i].y & 3) != 2) // boundary faces: the ghost has my material
      fcE[i] = fconst((int32_t)(i / NF), fdesc[i].x);

  // ---- device
  bfam_gpu_domain_t *d = new bfam_gpu_domain_t();
  d->dim = dim;
  d->N = N;
  d->Nq = Nq;
  d->Np = Np;
  d->Nfp = Nfp;
  d->NF = NF;
  d->NFLD = NFLD;
  d->K = K;
  d->Kg = Kg;
  d->fs = (size_t)K * Np;
  d->ks = ks;
  d->flux = opts->flux;
  d->precision = opts->precision;
  d->device = opts->device;
  d->budget = opts->mem_budget_bytes;
  int rc = 0;
#define TRY(x)                                                                 \
  do                                                                           \
  {                                                                            \
    rc = (x);                                                                  \
    if (rc)                                                                    \
    {                                                                          \
      release(d);                                                              \
      return rc;                                                               \
    }                                                                          \
  } while (0)
  {
    cudaError_t ce = cudaSetDevice(opts->device);
    if (ce != cudaSuccess)
    {
      release(d);
      return fail(BFAM_GPU_ECUDA, "cudaSetDevice(%d): %s", opts->device,
                  cudaGetErrorString(ce));
    }
    if (!d->budget)
      d->budget = free_device_bytes(opts->device);
    ce = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess)
    {
      release(d);
      return fail(BFAM_GPU_ECUDA, "stream: %s", cudaGetErrorString(ce));
    }
    d->own_stream = true;
    ce = ks.prepare(d->ks.occ);
    if (ce == cudaSuccess && (d->ks.occ[0] < 1 || d->ks.occ[1] < 1))
      ce = cudaErrorInvalidConfiguration;
    if (ce == cudaSuccess)
      ce = cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount,
                                  d->device);
    if (ce != cudaSuccess)
    {
      release(d);
      return fail(BFAM_GPU_ECUDA, "stage kernel setup: %s",
                  cudaGetErrorString(ce));
    }
  }
  d->hops = ops;
  const size_t state = (size_t)NFLD * d->fs * sizeof(double);
  TRY(dev_alloc(d, (void **)&d->q[0], state));
  TRY(dev_alloc(d, (void **)&d->q[1], state));
  TRY(dev_alloc(d, (void **)&d->dq, state));
  TRY(upload(d, &d->ed, ed.data(), ed.size()));
  TRY(upload(d, &d->fdesc, fdesc.data(), fdesc.size()));
  TRY(upload(d, &d->fcE, fcE.data(), fcE.size()));
  if (nslot > 0)
  {
    TRY(upload(d, &d->fslot, fslot.data(), fslot.size()));
    TRY(dev_alloc(d, (void **)&d->mbuf,
                  sizeof(double) * (size_t)nslot * 2 * dim * Nfp));
    // the unused pieces of glued faces stay zero
    if (cudaMemset(d->mbuf, 0, sizeof(double) * (size_t)nslot * 2 * dim *
                                   Nfp) != cudaSuccess)
    {
      release(d);
      return fail(BFAM_GPU_ECUDA, "mortar buffer memset failed");
    }
  }
  d->nlevels = nlevels;
  d->level_off = level_off;
  if (nlevels > 1)
    TRY(upload(d, &d->elist, elist.data(), elist.size()));
  d->helist = elist;
  TRY(upload(d, &d->ops, ops.data(), ops.size()));
  TRY(dev_alloc(d, (void **)&d->err, sizeof(int)));
  TRY(dev_alloc(d, (void **)&d->clock, sizeof(DomainClock)));
  if (quads)
  {
    // element boxes and metric on the device; the quadrant and tree tables
    // are needed only here
    int32_t *dq = nullptr;
    double *tx0 = nullptr, *th = nullptr;
    TRY(upload(d, &dq, quads->quads, (size_t)BFAM_GPU_NQUAD * K));
    TRY(upload(d, &tx0, quads->tree_x0, 3 * (size_t)quads->num_trees));
    TRY(upload(d, &th, quads->tree_h, 3 * (size_t)quads->num_trees));
    TRY(dev_alloc(d, (void **)&d->gx0, 3 * sizeof(double) * (size_t)K));
    TRY(dev_alloc(d, (void **)&d->gh, 3 * sizeof(double) * (size_t)K));
    dg_geometry_kernel<<<(K + 255) / 256, 256, 0, d->stream>>>(
        K, dim, dq, tx0, th, 1.0 / quads->root_len, d->ed, d->gx0, d->gh);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess)
      ce = cudaStreamSynchronize(d->stream);
    dev_free(d, dq);
    dev_free(d, tx0);
    dev_free(d, th);
    if (ce != cudaSuccess)
    {
      release(d);
      return fail(BFAM_GPU_ECUDA, "geometry kernel: %s",
                  cudaGetErrorString(ce));
    }
  }
#undef TRY
  // host copies for locating sources and receivers (device geometry: read
  // back when first needed)
  if (!quads)
  {
    d->hx0.assign(vol->x0, vol->x0 + 3 * (size_t)vol->K);
    d->hh.assign(vol->h, vol->h + 3 * (size_t)vol->K);
  }
  // boundary list (glued faces are joined to other domains later)
  d->bslot = bslot;
  d->bE.resize(nbnd);
  d->bF.resize(nbnd);
  for (int32_t b = 0; b < nbnd; ++b)
  {
    d->bE[b] = bnd->EToE[b];
    d->bF[b] = bnd->EToF[b];
    d->nglued += bslot[b] >= 0;
  }
  d->hr.assign(vol->r, vol->r + d->Nq);
  d->hw.assign(vol->w, vol->w + d->Nq);
  if (cudaMemset(d->q[0], 0, state) != cudaSuccess ||
      cudaMemset(d->q[1], 0, state) != cudaSuccess ||
      cudaMemset(d->dq, 0, state) != cudaSuccess ||
      cudaMemset(d->err, 0, sizeof(int)) != cudaSuccess ||
      cudaMemset(d->clock, 0, sizeof(DomainClock)) != cudaSuccess)
  {
    release(d);
    return fail(BFAM_GPU_ECUDA, "initial memset failed");
  }
  (void)nmap;
  *out = d;
  return 0;
}

int bfam_gpu_domain_get_geometry(bfam_gpu_domain_t *d, double *x0, double *h)
{
  if (!d)
    return fail(BFAM_GPU_EINVAL, "NULL domain");
  const int rc = host_geometry(d);
  if (rc)
    return rc;
  if (x0)
    std::memcpy(x0, d->hx0.data(), sizeof(double) * d->hx0.size());
  if (h)
    std::memcpy(h, d->hh.data(), sizeof(double) * d->hh.size());
  return 0;
}

int bfam_gpu_domain_launch_levels(const bfam_gpu_domain_t *d)
{
  return d ? d->nlevels : 0;
}

int bfam_gpu_domain_free(bfam_gpu_domain_t *d)
{
  release(d);
  return 0;
}

int bfam_gpu_domain_num_fields(const bfam_gpu_domain_t *d)
{
  return d ? d->NFLD : 0;
}

size_t bfam_gpu_domain_field_length(const bfam_gpu_domain_t *d)
{
  return d ? d->fs : 0;
}

size_t bfam_gpu_domain_device_bytes(const bfam_gpu_domain_t *d)
{
  return d ? d->bytes : 0;
}

int bfam_gpu_domain_set_stream(bfam_gpu_domain_t *d, void *stream)
{
  if (!d)
    return fail(BFAM_GPU_EINVAL, "domain is NULL");
  CUDA_TRY(cudaSetDevice(d->device));
  cudaStream_t next = (cudaStream_t)stream;
  if (next != d->stream)
  {
    // work queued on the old stream (asynchronous steps, stream-ordered
    // frees) comes before anything queued on the new one
    cudaEvent_t ev;
    CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, d->stream);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(next, ev, 0);
    cudaEventDestroy(ev);
    if (e != cudaSuccess)
    {
      cudaGetLastError();
      return fail(BFAM_GPU_ECUDA, "ordering the new stream after the old: %s",
                  cudaGetErrorString(e));
    }
    // a stream destroyed with work pending is released once that work ends
    if (d->own_stream && d->stream)
      cudaStreamDestroy(d->stream);
  }
  d->own_stream = false;
  d->stream = next;
  return 0;
}

int bfam_gpu_domain_sync(bfam_gpu_domain_t *d)
{
  if (!d)
    return fail(BFAM_GPU_EINVAL, "domain is NULL");
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  int err = 0;
  CUDA_TRY(cudaMemcpy(&err, d->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err)
  {
    CUDA_TRY(cudaMemset(d->err, 0, sizeof(int)));
    return fail(BFAM_GPU_ETIMEOUT,
                "a device-side wait on a bulk copy gave up (error flag %d)",
                err);
  }
  return 0;
}

int bfam_gpu_domain_set_fields(bfam_gpu_domain_t *d,
                               const double *const *fields)
{
  if (!d || !fields)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(d->device));
  for (int f = 0; f < d->NFLD; ++f)
  {
    if (!fields[f])
      return fail(BFAM_GPU_EINVAL, "field %d is NULL", f);
    CUDA_TRY(cudaMemcpyAsync(d->q[d->cur] + f * d->fs, fields[f],
                             d->fs * sizeof(double), cudaMemcpyHostToDevice,
                             d->stream));
  }
  return bfam_gpu_domain_sync(d);
}

int bfam_gpu_domain_get_fields(bfam_gpu_domain_t *d, double *const *fields)
{
  if (!d || !fields)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(d->device));
  for (int f = 0; f < d->NFLD; ++f)
  {
    if (!fields[f])
      return fail(BFAM_GPU_EINVAL, "field %d is NULL", f);
    CUDA_TRY(cudaMemcpyAsync(fields[f], d->q[d->cur] + f * d->fs,
                             d->fs * sizeof(double), cudaMemcpyDeviceToHost,
                             d->stream));
  }
  return bfam_gpu_domain_sync(d);
}

double *bfam_gpu_domain_field_device_ptr(bfam_gpu_domain_t *d, int f)
{
  if (!d || f < 0 || f >= d->NFLD)
    return nullptr;
  return d->q[d->cur] + f * d->fs;
}

int bfam_gpu_domain_rhs(bfam_gpu_domain_t *d, double *const *rhs)
{
  if (!d || !rhs)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  if (d->nglued)
    return fail(BFAM_GPU_EINVAL,
                "the domain has %d faces glued to another domain: step it "
                "in a batch with its glue",
                d->nglued);
  CUDA_TRY(cudaSetDevice(d->device));
  if (!d->rhs)
  {
    int rc = dev_alloc(d, (void **)&d->rhs,
                       (size_t)d->NFLD * d->fs * sizeof(double));
    if (rc)
      return rc;
  }
  int rc = launch_stage(d, d->cur, 0.0, 0.0, 0.0, 0.0, 1, MODE_RHS);
  if (rc)
    return rc;
  for (int f = 0; f < d->NFLD; ++f)
    CUDA_TRY(cudaMemcpyAsync(rhs[f], d->rhs + f * d->fs,
                             d->fs * sizeof(double), cudaMemcpyDeviceToHost,
                             d->stream));
  return bfam_gpu_domain_sync(d);
}

int bfam_gpu_domain_energy(bfam_gpu_domain_t *d, double *energy)
{
  if (!d || !energy)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(d->device));
  if (!d->energy)
  {
    int rc = dev_alloc(d, (void **)&d->energy, (d->K + 1) * sizeof(double));
    if (rc)
      return rc;
  }
  d->ks.energy<<<d->K, d->ks.NT, 0, d->stream>>>(d->q[d->cur], d->fs, d->ed,
                                                 d->ops, d->energy);
  sum_kernel<<<1, 1024, 0, d->stream>>>(d->energy, d->K, d->energy + d->K);
  g_launches.fetch_add(2, std::memory_order_relaxed);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(energy, d->energy + d->K, sizeof(double),
                           cudaMemcpyDeviceToHost, d->stream));
  return bfam_gpu_domain_sync(d);
}

} // extern "C"

namespace
{

// Fixed scratch for bfam_gpu_domain_energy_noalloc: one per-element energy
// slot per element plus the total.  In host code the array's name is only a
// stand-in; its device address comes from cudaGetSymbolAddress, once per
// device, and is cached below.
static __device__ __align__(256) double
    g_noalloc_energy[BFAM_GPU_NOALLOC_MAX_ELEMENTS + 1];

std::mutex g_noalloc_mu;
std::vector<double *> g_noalloc_ptr; // indexed by device ordinal

int noalloc_scratch(int device, double **out)
{
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if ((int)g_noalloc_ptr.size() <= device)
    g_noalloc_ptr.resize(device + 1, nullptr);
  if (!g_noalloc_ptr[device])
  {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_energy);
    if (e != cudaSuccess || !p)
      return fail(BFAM_GPU_ECUDA, "cudaGetSymbolAddress(noalloc scratch): %s",
                  cudaGetErrorString(e));
    g_noalloc_ptr[device] = static_cast<double *>(p);
  }
  *out = g_noalloc_ptr[device];
  return 0;
}

} // namespace

extern "C" {

int bfam_gpu_domain_energy_noalloc(bfam_gpu_domain_t *d, double *energy)
{
  if (!d || !energy)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  if (d->K > BFAM_GPU_NOALLOC_MAX_ELEMENTS)
    return fail(BFAM_GPU_EINVAL,
                "domain has %d elements; the allocation-free energy takes at "
                "most %d (BFAM_GPU_NOALLOC_MAX_ELEMENTS)",
                d->K, BFAM_GPU_NOALLOC_MAX_ELEMENTS);
  CUDA_TRY(cudaSetDevice(d->device));
  double *scratch = nullptr;
  int rc = noalloc_scratch(d->device, &scratch);
  if (rc)
    return rc;
  d->ks.energy<<<d->K, d->ks.NT, 0, d->stream>>>(d->q[d->cur], d->fs, d->ed,
                                                 d->ops, scratch);
  sum_kernel<<<1, 1024, 0, d->stream>>>(scratch, d->K, scratch + d->K);
  g_launches.fetch_add(2, std::memory_order_relaxed);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(energy, scratch + d->K, sizeof(double),
                           cudaMemcpyDeviceToHost, d->stream));
  return bfam_gpu_domain_sync(d);
}

int bfam_ts_lsrk_init(bfam_ts_lsrk_t **ts, bfam_gpu_domain_t *dom, int method,
                      double t0)
{
  if (!ts || !dom)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  *ts = nullptr;
  bfam_ts_lsrk_t *s = new bfam_ts_lsrk_t();
  s->dom = dom;
  s->t = t0;
  dom->clock_valid = false; // set from t0 before the first step that needs it
  switch (method)
  {
  case 0: // KC54: Carpenter & Kennedy five-stage fourth-order
    s->ns = 5;
    s->A[0] = 0.0;
    s->A[1] = (double)(-567301805773.0L / 1357537059087.0L);
    s->A[2] = (double)(-2404267990393.0L / 2016746695238.0L);
    s->A[3] = (double)(-3550918686646.0L / 2091501179385.0L);
    s->A[4] = (double)(-1275806237668.0L / 842570457699.0L);
    s->B[0] = (double)(1432997174477.0L / 9575080441755.0L);
    s->B[1] = (double)(5161836677717.0L / 13612068292357.0L);
    s->B[2] = (double)(1720146321549.0L / 2090206949498.0L);
    s->B[3] = (double)(3134564353537.0L / 4481467310338.0L);
    s->B[4] = (double)(2277821191437.0L / 14882151754819.0L);
    s->C[0] = 0.0;
    s->C[1] = (double)(1432997174477.0L / 9575080441755.0L);
    s->C[2] = (double)(2526269341429.0L / 6820363962896.0L);
    s->C[3] = (double)(2006345519317.0L / 3224310063776.0L);
    s->C[4] = (double)(2802321613138.0L / 2924317926251.0L);
    s->C[5] = 1.0;
    break;
  case 1: // forward Euler
    s->ns = 1;
    s->B[0] = 1.0;
    s->C[1] = 1.0;
    break;
  case 2: // Heun
    s->ns = 2;
    s->A[1] = -1.0;
    s->B[0] = 1.0;
    s->B[1] = 0.5;
    s->C[1] = 1.0;
    s->C[2] = 1.0;
    break;
  case 3: // Williamson three-stage third-order
    s->ns = 3;
    s->A[1] = (double)(-5.0L / 9.0L);
    s->A[2] = (double)(-153.0L / 128.0L);
    s->B[0] = (double)(1.0L / 3.0L);
    s->B[1] = (double)(15.0L / 16.0L);
    s->B[2] = (double)(8.0L / 15.0L);
    s->C[1] = (double)(1.0L / 3.0L);
    s->C[2] = (double)(3.0L / 4.0L);
    s->C[3] = 1.0;
    break;
  default:
    delete s;
    return fail(BFAM_GPU_EINVAL, "unknown LSRK method %d", method);
  }
  *ts = s;
  return 0;
}

int bfam_ts_lsrk_step(bfam_ts_lsrk_t *ts, double dt, int nsteps, int use_graph)
{
  if (!ts || nsteps < 0)
    return fail(BFAM_GPU_EINVAL, "bad arguments");
  bfam_gpu_domain_t *d = ts->dom;
  if (d->nglued)
    return fail(BFAM_GPU_EINVAL,
                "the domain has %d faces glued to another domain: step it "
                "in a batch with its glue",
                d->nglued);
  CUDA_TRY(cudaSetDevice(d->device));
  // a point source or receivers need the device clock, advanced once per
  // step by the post-step kernel
  const bool post = has_extras(d);
  if (post && !d->clock_valid)
  {
    int rc = set_clock(d, ts->t, 0);
    if (rc)
      return rc;
  }
  // one step starting from state buffer c0
  auto issue = [&](int c0) -> int {
    int in = c0;
    static const char *const stage_name[] = {"lsrk stage 0", "lsrk stage 1",
                                             "lsrk stage 2", "lsrk stage 3",
                                             "lsrk stage 4", "lsrk stage 5"};
    for (int s = 0; s < ts->ns; ++s, in ^= 1)
    {
      nvtxRangePushA(stage_name[s < 6 ? s : 5]);
      int rc = launch_stage(d, in, ts->A[s], ts->B[s], ts->C[s], dt, s == 0,
                            MODE_STAGE);
      nvtxRangePop();
      if (rc)
        return rc;
    }
    return post ? launch_post(d, in, dt) : 0;
  };
  const int per_step = ts->ns * d->nlevels + (post ? 1 : 0);
  // per-launch timing needs eager launches
  if (d->prof)
    use_graph = 0;
  struct NvtxRange
  {
    NvtxRange() { nvtxRangePushA("bfam_ts_lsrk_step"); }
    ~NvtxRange() { nvtxRangePop(); }
  } nvtx_range;
  for (int st = 0; st < nsteps; ++st)
  {
    const int c0 = d->cur;
    if (use_graph && d->stream)
    {
      if (!ts->graph[c0] || ts->graph_dt[c0] != dt ||
          ts->graph_post[c0] != post || ts->graph_gen[c0] != d->extras_gen)
      {
        if (ts->graph[c0])
          cudaGraphExecDestroy(ts->graph[c0]);
        ts->graph[c0] = nullptr;
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(d->stream,
                                        cudaStreamCaptureModeThreadLocal));
        const int rc = issue(c0);
        cudaError_t ce = cudaStreamEndCapture(d->stream, &g);
        if (rc)
          return rc;
        if (ce != cudaSuccess)
          return fail(BFAM_GPU_ECUDA, "graph capture: %s",
                      cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&ts->graph[c0], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess)
          return fail(BFAM_GPU_ECUDA, "graph instantiate: %s",
                      cudaGetErrorString(ce));
        ts->graph_dt[c0] = dt;
        ts->graph_post[c0] = post;
        ts->graph_gen[c0] = d->extras_gen;
        // capture counted the launches once; replays are counted below
        g_launches.fetch_sub(per_step, std::memory_order_relaxed);
      }
      CUDA_TRY(cudaGraphLaunch(ts->graph[c0], d->stream));
      g_launches.fetch_add(per_step, std::memory_order_relaxed);
    }
    else
    {
      const int rc = issue(c0);
      if (rc)
        return rc;
    }
    d->cur = (ts->ns & 1) ? c0 ^ 1 : c0;
    ts->t += dt;
  }
  if (!post && nsteps > 0)
    d->clock_valid = false;
  return 0;
}

int bfam_ts_lsrk_time(const bfam_ts_lsrk_t *ts, double *t)
{
  if (!ts || !t)
    return fail(BFAM_GPU_EINVAL, "NULL argument");
  *t = ts->t;
  return 0;
}

int bfam_ts_lsrk_free(bfam_ts_lsrk_t *ts)
{
  if (!ts)
    return 0;
  for (int i = 0; i < 2; ++i)
    if (ts->graph[i])
      cudaGraphExecDestroy(ts->graph[i]);
  delete ts;
  return 0;
}

} // extern "C"
