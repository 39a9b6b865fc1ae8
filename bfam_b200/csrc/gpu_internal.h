// Host-side declarations shared by the translation units of the bfam_gpu
// C-ABI (internal; the public interface is include/bfam_gpu.h).
#pragma once

#include "bfam_gpu.h"
#include "dg_common.cuh"

#include <atomic>
#include <cstdint>
#include <vector>

namespace bfam_b200
{
namespace host
{

// records the message for bfam_gpu_last_error and returns code
int fail(int code, const char *fmt, ...);
// kernels launched by the library (bfam_gpu_launch_count)
extern std::atomic<uint64_t> g_launches;

#define CUDA_TRY(call)                                                         \
  do                                                                           \
  {                                                                            \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return fail(BFAM_GPU_ECUDA, "%s: %s (%s:%d)", #call,                     \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                 \
  } while (0)

// per-order launchers (the kernels' parameter lists depend on the order)
typedef void (*stage_launch_fn)(const DomainView &, int n,
                                const StageParams &, const double *D,
                                int mode, int grid, cudaStream_t);
typedef cudaError_t (*prepare_fn)(int *occ);
typedef void (*energy_fn)(const double *, size_t, const ElemData *,
                          const double *, double *);

struct KernelSet
{
  stage_launch_fn launch = nullptr;
  prepare_fn prepare = nullptr;
  energy_fn energy = nullptr;
  int NT = 0;
  size_t smem = 0;
  int occ[2] = {0, 0}; // resident CTAs per SM of the stage and rhs kernels
  int nbuf = 1;        // element buffers per CTA
};

// the kernels of one (dim, order, precision)
bool kernel_set(int dim, int N, int precision, KernelSet *out);

// hops: host copy of the operator block Dr | interp[3] | proj[3] | w
template <int N, typename CT>
DiffOp<N, CT> make_diffop(const double *hops)
{
  constexpr int n2 = (N + 1) * (N + 1);
  DiffOp<N, CT> dop;
  for (int i = 0; i < n2; ++i)
  {
    dop.D[i] = CT(hops[i]);
    dop.Ib[i] = CT(hops[2 * n2 + i]); // interpolation[1]: refine to bottom
    dop.Pb[i] = hops[5 * n2 + i];     // projection[1]: coarsen from bottom
  }
  dop.iwend = 1.0 / hops[7 * n2];
  return dop;
}

} // namespace host
} // namespace bfam_b200

struct bfam_gpu_domain
{
  int dim = 0, N = 0, Nq = 0, Np = 0, Nfp = 0, NF = 0, NFLD = 0;
  int32_t K = 0, Kg = 0;
  int device = 0, sms = 0;
  int flux = 0, precision = 0;
  size_t fs = 0;
  bfam_b200::host::KernelSet ks;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double *q[2] = {nullptr, nullptr};
  double *dq = nullptr;
  double *rhs = nullptr;
  double *energy = nullptr;
  bfam_b200::ElemData *ed = nullptr;
  int2 *fdesc = nullptr;
  double4 *fcE = nullptr;
  int *fslot = nullptr;  // [K][NF] mortar slot of each fine face (-1: none)
  double *mbuf = nullptr; // [slots][2 dim][Nfp] projected coarse-side jumps
  // launch levels (meshes with hanging faces): elements of level l are
  // elist[level_off[l] .. level_off[l+1])
  int nlevels = 1;
  std::vector<int32_t> level_off;
  int32_t *elist = nullptr;
  std::vector<int32_t> helist; // host copy of elist
  double *ops = nullptr;
  // host copy of Dr | interp[3] | proj[3] | w; the 1-D operators are passed
  // by value (kernel parameter bank) to each launch
  std::vector<double> hops;
  int *err = nullptr;
  int cur = 0;
  size_t bytes = 0, budget = 0;
  std::vector<void *> allocs;
  std::vector<size_t> alloc_bytes;
  // host copies for locating sources and receivers: element lower corners
  // and edge lengths [K][3], LGL nodes and weights [Nq]
  std::vector<double> hx0, hh, hr, hw;
  // element boxes computed on the device from quadrant data ([K][3] each;
  // null when the boxes came from the host)
  double *gx0 = nullptr, *gh = nullptr;
  // boundary list: element, face and (glued faces) mortar slot per entry;
  // glued faces are filled by the glue between domains
  std::vector<int32_t> bE, bslot;
  std::vector<int8_t> bF;
  int nglued = 0;
  // time-dependent extras: device clock, Ricker point source, receivers
  bfam_b200::DomainClock *clock = nullptr;
  bool clock_valid = false; // device clock holds the stepper's time
  bfam_b200::PointSource src{-1, nullptr, {0, 0, 0}, 0, 0};
  void *src_w_alloc = nullptr; // device copy of src.w
  int nrecv = 0, max_samples = 0;
  int *recv_elem = nullptr;
  double *recv_w = nullptr;
  double *seis = nullptr;
  unsigned extras_gen = 0;   // bumped when the source or receivers change
  // opt-in per-launch timing (bfam_gpu_domain_profile): an event pair
  // around every stage launch, drained into per-level totals
  bool prof = false;
  struct ProfLaunch
  {
    cudaEvent_t t0, t1;
    int level;
    double bytes; // algorithmic bytes of the launch
    int64_t elements;
  };
  std::vector<ProfLaunch> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  std::vector<double> prof_ms, prof_bytes;
  std::vector<int64_t> prof_launches, prof_elements;
};

struct bfam_ts_lsrk
{
  bfam_gpu_domain_t *dom = nullptr;
  int ns = 0;
  double A[6] = {0}, B[6] = {0}, C[7] = {0};
  double t = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt[2] = {0, 0};
  bool graph_post[2] = {false, false};
  unsigned graph_gen[2] = {0, 0};
};

namespace bfam_b200
{
namespace host
{

// device allocation counted against the domain's budget, freed with it
int dev_alloc(bfam_gpu_domain_t *d, void **p, size_t bytes);
// the library's own stream-ordered memory pool of a device (created once,
// keeps freed blocks for reuse), and an allocation from it on a stream
cudaMemPool_t library_pool(int device);
cudaError_t pool_alloc(void **p, size_t bytes, int device, cudaStream_t stream);
// fills the host copies of the element boxes (read back from the device
// when the domain computed them from quadrant data)
int host_geometry(bfam_gpu_domain_t *d);
// frees one allocation made by dev_alloc before the domain is freed
void dev_free(bfam_gpu_domain_t *d, void *p);

template <typename T>
int upload(bfam_gpu_domain_t *d, T **dst, const T *src, size_t n)
{
  int rc = dev_alloc(d, (void **)dst, n * sizeof(T));
  if (rc)
    return rc;
  if (n)
    CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// the stage kernel's view of a domain whose stage input is q[in]
DomainView view(bfam_gpu_domain_t *d, int in);
int launch_stage(bfam_gpu_domain_t *d, int in, double A, double B, double C,
                 double dt, int first, int mode);

// point source or receivers present
inline bool has_extras(const bfam_gpu_domain_t *d)
{
  return d->src.elem >= 0 || d->nrecv > 0;
}
// set the device clock to t (and reset the sample count), on the domain's
// stream
int set_clock(bfam_gpu_domain_t *d, double t, int reset);
// the post-step kernel of one domain whose state after the step is q[cur]
int launch_post(bfam_gpu_domain_t *d, int cur, double dt);

} // namespace host
} // namespace bfam_b200
