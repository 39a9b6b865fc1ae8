// Once-per-step work beside the stage kernels: receiver sampling and the
// per-domain clock that the point source reads.
#pragma once

#include "dg_common.cuh"

namespace bfam_b200
{

// What the post-step kernel needs of one domain.
struct PostView
{
  const double *__restrict__ q; // state after the step
  size_t fs;                    // field stride K*Np
  int Np, nfld;
  int nrecv, max_samples;
  const int *__restrict__ relem; // [nrecv] element holding receiver r
  const double *__restrict__ rw; // [nrecv][Np] Lagrange weights phi_n(x_r)
  double *__restrict__ seis;     // [max_samples][nrecv][nfld]
  DomainClock *clock;
  double dt;
};

// One CTA per domain: sample every field at every receiver (one warp per
// (receiver, field) pair, lane-strided dot product with the element's
// Lagrange weights, then a butterfly sum: deterministic for a fixed block
// size), then advance the domain's clock by dt.  Samples beyond
// max_samples are dropped; the clock still advances.
__device__ __forceinline__ void post_step(const PostView &p)
{
  const int s = p.clock->nsamp;
  if (s < p.max_samples)
  {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5,
              nw = blockDim.x >> 5;
    for (int w = wid; w < p.nrecv * p.nfld; w += nw)
    {
      const int r = w / p.nfld, c = w % p.nfld;
      const double *x = p.q + c * p.fs + (size_t)p.relem[r] * p.Np;
      const double *wt = p.rw + (size_t)r * p.Np;
      double acc = 0;
      for (int n = lane; n < p.Np; n += 32)
        acc += wt[n] * x[n];
#pragma unroll
      for (int o = 16; o; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0)
        p.seis[((size_t)s * p.nrecv + r) * p.nfld + c] = acc;
    }
  }
  __syncthreads(); // every warp has read the clock
  if (threadIdx.x == 0)
  {
    p.clock->time += p.dt;
    p.clock->nsamp = s + 1;
  }
}

constexpr int POST_THREADS = 256;

// batches: one CTA per domain of the array
__global__ void __launch_bounds__(POST_THREADS)
    dg_post_step_kernel(const PostView *__restrict__ pv)
{
  post_step(pv[blockIdx.x]);
}

// one domain, its view in the parameter bank (captured by value in graphs)
__global__ void __launch_bounds__(POST_THREADS)
    dg_post_step_one(const __grid_constant__ PostView p)
{
  post_step(p);
}

// what & 1: set the time to t; what & 2: restart the sample count
__global__ void dg_set_clock_kernel(DomainClock *clock, double t, int what)
{
  if (what & 1)
    clock->time = t;
  if (what & 2)
    clock->nsamp = 0;
}

} // namespace bfam_b200
