// Discrete energy of a domain's state (FP64): per-element sums and a
// deterministic reduction.
#pragma once

#include "dg_common.cuh"

namespace bfam_b200
{

// Per-element discrete energy (FP64), one element per CTA.
template <int DIM, int N>
__global__ void __launch_bounds__(Shape<DIM, N>::NT)
    dg_energy_kernel(const double *__restrict__ q, size_t fs,
                     const ElemData *__restrict__ ed,
                     const double *__restrict__ ops, double *__restrict__ out)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, NT = S::NT;
  __shared__ double red[NT / 32];
  const int e = blockIdx.x, t = threadIdx.x;
  const double *w = ops + 7 * Nq * Nq;
  const ElemData me = ed[e];
  double val = 0;
  // NT may be below Np (N = 7 in 3D): a thread sums several nodes
  for (int n = t; n < Np; n += NT)
  {
    const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
    const double wn = w[i] * w[j] * (DIM == 3 ? w[k] : 1.0);
    const size_t id = (size_t)e * Np + n;
    const double rho = 1.0 / me.irho, la = me.lam, mu = me.mu;
    double kin = 0, pot = 0;
    for (int a = 0; a < DIM; ++a)
      kin += q[a * fs + id] * q[a * fs + id];
    kin *= rho;
    if (DIM == 3)
    {
      const double sxx = q[3 * fs + id], syy = q[4 * fs + id],
                   szz = q[5 * fs + id];
      const double tr = sxx + syy + szz;
      pot = (sxx * sxx + syy * syy + szz * szz -
             la / (3 * la + 2 * mu) * tr * tr) /
            (2 * mu);
      for (int c = 6; c < 9; ++c)
        pot += q[c * fs + id] * q[c * fs + id] / mu;
    }
    else
    {
      const double sxx = q[2 * fs + id], syy = q[3 * fs + id],
                   sxy = q[4 * fs + id];
      const double aa = la + 2 * mu, bb = la, det = aa * aa - bb * bb;
      pot = (aa * sxx * sxx - 2 * bb * sxx * syy + aa * syy * syy) / det +
            sxy * sxy / mu;
    }
    val += wn * (kin + pot);
  }
  for (int o = 16; o > 0; o >>= 1)
    val += __shfl_down_sync(0xffffffffu, val, o);
  if ((t & 31) == 0)
    red[t >> 5] = val;
  __syncthreads();
  if (t == 0)
  {
    double s = 0;
    for (int wi = 0; wi < NT / 32; ++wi)
      s += red[wi];
    double J = 1;
    J = (2.0 / me.rx) * (2.0 / me.ry) * (DIM == 3 ? (2.0 / me.rz) : 1.0);
    J *= DIM == 3 ? 0.125 : 0.25;
    out[e] = 0.5 * J * s;
  }
}

// Deterministic sum of n values by one CTA of 1024 threads.
__global__ void __launch_bounds__(1024)
    sum_kernel(const double *__restrict__ v, int64_t n, double *__restrict__ out)
{
  __shared__ double red[32];
  double s = 0;
  for (int64_t i = threadIdx.x; i < n; i += 1024)
    s += v[i];
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double tt = 0;
    for (int i = 0; i < 32; ++i)
      tt += red[i];
    *out = tt;
  }
}

} // namespace bfam_b200
