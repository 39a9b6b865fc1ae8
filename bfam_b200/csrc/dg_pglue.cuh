// Glue between two domains (faces of different orders): the coupling
// kernel run once per LSRK stage before the stage's element launches.
#pragma once

#include "dg_common.cuh"

namespace bfam_b200
{

constexpr int PGLUE_MAXQ = 8;  // highest compiled order 7
constexpr int PGLUE_THREADS = 64;

// One side of a glue: its domain's stage input, element tables and mortar
// buffer, the glued face of every pair and its mortar slot, and its 1-D
// operators to and from the glue grid (column-major; NULL: identity).
struct PGlueSide
{
  const double *__restrict__ q;
  size_t fs;
  int N;
  const ElemData *__restrict__ ed;
  double *mbuf;
  const int32_t *__restrict__ elem;
  const int8_t *__restrict__ face;
  const int32_t *__restrict__ slot;
  const double *__restrict__ I; // (Ng+1) x (N+1)
  const double *__restrict__ P; // (N+1) x (Ng+1)
};

struct PGlueView
{
  PGlueSide s[2];
  int32_t K;
  int Ng, flux;
};

// volume node of face node (a, b) on face f of an order-N element
template <int DIM>
__device__ __forceinline__ int gmask_rt(int N, int f, int a, int b)
{
  const int Nq = N + 1;
  if (DIM == 2)
    return f == 0 ? a * Nq : (f == 1 ? a * Nq + N : (f == 2 ? a : N * Nq + a));
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

// out[i + mo b'] = sum A(i, a) v[a + mi b] along the first face axis (A is
// mo x mi column-major, A == NULL: copy), for the n2 lines b of nf fields;
// `stride` separates the fields in both arrays
__device__ __forceinline__ void pglue_axis0(const double *A, int mo, int mi,
                                            int n2, int nf, int stride,
                                            const double *v, double *out)
{
  for (int w = threadIdx.x; w < nf * mo * n2; w += blockDim.x)
  {
    const int c = w / (mo * n2), r = w % (mo * n2);
    const int i = r % mo, b = r / mo;
    const double *x = v + c * stride + mi * b;
    double s = 0;
    if (A)
      for (int a = 0; a < mi; ++a)
        s += A[i + mo * a] * x[a];
    else
      s = x[i];
    out[c * stride + i + mo * b] = s;
  }
}

// the same along the second face axis: out[a + m0 i] = sum A(i, b) v[a + m0 b]
__device__ __forceinline__ void pglue_axis1(const double *A, int mo, int mi,
                                            int m0, int nf, int stride,
                                            const double *v, double *out)
{
  for (int w = threadIdx.x; w < nf * m0 * mo; w += blockDim.x)
  {
    const int c = w / (m0 * mo), r = w % (m0 * mo);
    const int a = r % m0, i = r / m0;
    const double *x = v + c * stride + a;
    double s = 0;
    if (A)
      for (int b = 0; b < mi; ++b)
        s += A[i + mo * b] * x[m0 * b];
    else
      s = x[m0 * i];
    out[c * stride + a + m0 * i] = s;
  }
}

// One CTA per glued pair (minus side s[0], plus side s[1], opposite faces of
// one axis, face nodes in the same tangential order):
//  1. each side's trace (velocity and the stress row of the face axis) is
//     gathered and interpolated to the order-Ng glue grid;
//  2. at every glue node the Riemann problem gives each side's jumps
//     (T* - T-, v* - v-) from its own outward normal and impedances;
//  3. each side's jumps are L2-projected back to its order and stored in
//     its mortar slot, [2 dim][Nfp] in that side's face-node order, which
//     the side's stage kernel lifts like a coarse face with one piece.
template <int DIM>
__global__ void __launch_bounds__(PGLUE_THREADS) dg_pglue_kernel(const PGlueView v)
{
  constexpr int NTF = 2 * DIM, NJ = 2 * DIM;
  constexpr int MF = DIM == 3 ? PGLUE_MAXQ * PGLUE_MAXQ : PGLUE_MAXQ;
  __shared__ double tr[2][NTF][MF]; // traces, then glue-grid values
  __shared__ double tmp[NTF][MF];
  __shared__ double J[2][NJ][MF];
  const int k = blockIdx.x, t = threadIdx.x;
  if (k >= v.K)
    return;
  const int Ngq = v.Ng + 1;
  const int nfg = DIM == 3 ? Ngq * Ngq : Ngq;
  const int f0 = v.s[0].face[k];
  const int ax = f0 >> 1;

  // 1. traces to the glue grid
  for (int sd = 0; sd < 2; ++sd)
  {
    const PGlueSide &S = v.s[sd];
    const int N = S.N, Nq = N + 1, nf = DIM == 3 ? Nq * Nq : Nq;
    const int e = S.elem[k], f = S.face[k];
    const size_t eoff = (size_t)e * (DIM == 3 ? Nq * Nq * Nq : Nq * Nq);
    for (int w = t; w < NTF * nf; w += blockDim.x)
    {
      const int c = w / nf, pn = w % nf;
      tr[sd][c][pn] = S.q[trace_field<DIM>(ax, c) * S.fs + eoff +
                          gmask_rt<DIM>(N, f, pn % Nq, pn / Nq)];
    }
    __syncthreads();
    if (DIM == 3)
    {
      pglue_axis0(S.I, Ngq, Nq, Nq, NTF, MF, &tr[sd][0][0], &tmp[0][0]);
      __syncthreads();
      pglue_axis1(S.I, Ngq, Nq, Ngq, NTF, MF, &tmp[0][0], &tr[sd][0][0]);
    }
    else
    {
      pglue_axis0(S.I, Ngq, Nq, 1, NTF, MF, &tr[sd][0][0], &tmp[0][0]);
      __syncthreads();
      for (int w = t; w < NTF * Ngq; w += blockDim.x)
        tr[sd][w / Ngq][w % Ngq] = tmp[w / Ngq][w % Ngq];
    }
    __syncthreads();
  }

  // 2. jumps of both sides at the glue nodes
  {
    const ElemData &m0 = v.s[0].ed[v.s[0].elem[k]];
    const ElemData &m1 = v.s[1].ed[v.s[1].elem[k]];
    const double fc0[4] = {m1.Zp, 1.0 / (m0.Zp + m1.Zp), m1.Zs,
                           1.0 / (m0.Zs + m1.Zs)};
    const double fc1[4] = {m0.Zp, 1.0 / (m1.Zp + m0.Zp), m0.Zs,
                           1.0 / (m1.Zs + m0.Zs)};
    const double sg = (f0 & 1) ? 1.0 : -1.0;
    for (int pg = t; pg < nfg; pg += blockDim.x)
    {
      double dq[NTF], dqn[NTF], Jm[6], Jp[6];
#pragma unroll
      for (int c = 0; c < NTF; ++c)
      {
        dq[c] = tr[1][c][pg] - tr[0][c][pg];
        dqn[c] = -dq[c];
      }
      flux_jumps<DIM, double>(dq, ax, sg, m0.Zp, m0.Zs, fc0, v.flux, Jm);
      flux_jumps<DIM, double>(dqn, ax, -sg, m1.Zp, m1.Zs, fc1, v.flux, Jp);
#pragma unroll
      for (int c = 0; c < NJ; ++c)
      {
        J[0][c][pg] = Jm[jslot<DIM>(c)];
        J[1][c][pg] = Jp[jslot<DIM>(c)];
      }
    }
    __syncthreads();
  }

  // 3. projection to each side's order, into its mortar slot
  for (int sd = 0; sd < 2; ++sd)
  {
    const PGlueSide &S = v.s[sd];
    const int Nq = S.N + 1, nf = DIM == 3 ? Nq * Nq : Nq;
    double *out = S.mbuf + (size_t)S.slot[k] * NJ * nf;
    if (DIM == 3)
    {
      pglue_axis0(S.P, Nq, Ngq, Ngq, NJ, MF, &J[sd][0][0], &tmp[0][0]);
      __syncthreads();
      pglue_axis1(S.P, Nq, Ngq, Nq, NJ, MF, &tmp[0][0], &tr[0][0][0]);
    }
    else
    {
      pglue_axis0(S.P, Nq, Ngq, 1, NJ, MF, &J[sd][0][0], &tr[0][0][0]);
    }
    __syncthreads();
    for (int w = t; w < NJ * nf; w += blockDim.x)
      out[w] = tr[0][w / nf][w % nf];
    __syncthreads();
  }
}

} // namespace bfam_b200
