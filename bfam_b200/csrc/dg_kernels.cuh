// Fused DG stage kernel for the isotropic velocity-stress elastic system on
// affine Cartesian elements (sm_100a).
//
// One launch per LSRK stage does, per element:
//   volume  : tensor-product LGL derivative along each axis from shared
//             memory (the BFAM_KRON_* contractions, src/bfam.c:3137-3624);
//   face    : upwind flux on neighbour traces gathered through the compact
//             neighbour table (the on-device replacement of vmapP and of the
//             bfam_communicator ghost exchange, src/bfam.c:6783-6877,
//             2418-2679), lifted with the lumped LGL mass;
//   mortar  : for faces that go through the glue grid (2:1 hanging faces,
//             src/bfam.c:7328-7520) the traces are interpolated to each
//             half-size mortar piece (interpolation[1..2]), the flux is
//             evaluated there and L2-projected back (projection[1..2]);
//   update  : the 2N-storage LSRK stage dq = A dq + dt rhs, q' = q + B dq
//             (bfamo_lsrk_t, src/bfam.h:1840-1846) in the tail, writing the
//             new state to the other state buffer so that neighbours of
//             every element read the stage input unchanged.
//
// State layout in HBM: field-major, element, node (bfam's per-field arrays
// stacked): q[f * K * Np + e * Np + n], n = i + Nq (j + Nq k).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bfam_b200
{

struct ElemData
{
  double irho, lam, mu, Zp, Zs, rx, ry, rz; // rx = 2/hx, ...
};

struct DomainView
{
  int32_t K;
  size_t fs; // field stride K*Np
  const double *__restrict__ qin;
  double *__restrict__ qout;
  double *__restrict__ dq;
  double *__restrict__ rhs; // right-hand-side output (rhs mode)
  const ElemData *__restrict__ ed;
  const int32_t *__restrict__ nbr; // [K][NF] >= 0 neighbour, < 0 -(1 + glue)
  const int8_t *__restrict__ nbrf; // [K][NF] neighbour face + NF * perm code
  const int32_t *__restrict__ gEm;
  const int32_t *__restrict__ gEp;
  const int8_t *__restrict__ gFm;
  const int8_t *__restrict__ gHm;
  const int8_t *__restrict__ gOp;
  const double *__restrict__ ops; // Dr | interp[3] | proj[3] | w
  int *err;
};

struct StageParams
{
  double A, B, dt;
  int first_stage; // A == 0: dq is not read
  int flux;        // 0 upwind, 1 central
};

enum
{
  MODE_STAGE = 0,
  MODE_RHS = 1
};

template <int DIM, int N> struct Shape
{
  static constexpr int Nq = N + 1;
  static constexpr int Np = DIM == 3 ? Nq * Nq * Nq : Nq * Nq;
  static constexpr int Nfp = DIM == 3 ? Nq * Nq : Nq;
  static constexpr int NF = 2 * DIM;
  static constexpr int NFLD = DIM == 3 ? 9 : 5;
  static constexpr int NJ = 6; // (T* - T-, v* - v-), 3 components each
  static constexpr int NP = DIM == 3 ? 4 : 2; // mortar pieces per coarse face
  static constexpr int work = (Np > NF * Nfp ? Np : NF * Nfp);
  static constexpr int NT = ((work + 31) / 32) * 32 > 1024
                                ? 1024
                                : ((work + 31) / 32) * 32;
  static constexpr int OPS = 7 * Nq * Nq + Nq;
  static constexpr int OPS_PAD = (OPS + 1) & ~1; // keep 16-byte alignment
  // shared memory in doubles
  static constexpr int SM_QS = NFLD * Np;
  static constexpr int SM_JF = NF * NJ * Nfp;
  // mortar buffers hold either NFLD traces or NJ jump components
  static constexpr int SM_MB = (NFLD > NJ ? NFLD : NJ) * Nfp;
  static constexpr int SM_TOTAL = OPS_PAD + SM_QS + SM_JF + 3 * SM_MB + 2;
  static constexpr bool TMA = (Np % 2) == 0; // 16-byte aligned element rows
};

// ------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::"
               "bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Wait on phase `parity`; gives up after ~2 s of wall time and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it)
  {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(a), "r"(parity)
                 : "memory");
    if (done)
      return true;
    if (it == 0)
      t0 = global_ns();
    else if ((it & 63) == 0 && global_ns() - t0 > 2000000000ull)
      return false;
  }
}

// --------------------------------------------------------- index helpers

// volume node of face node pn on face f (bfam face masks)
template <int DIM, int N> __device__ __forceinline__ int gmask(int f, int pn)
{
  constexpr int Nq = N + 1;
  if (DIM == 2)
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

// neighbour face-node of my face node pn under permutation code ns
// (bfam_subdomain_dgx_buildmaps, src/bfam.c:6823-6866)
template <int DIM, int N> __device__ __forceinline__ int face_perm(int ns, int pn)
{
  constexpr int Nq = N + 1;
  if (DIM == 2)
    return ns ? N - pn : pn;
  const int i = pn % Nq, j = pn / Nq, ir = N - i, jr = N - j;
  switch (ns)
  {
  case 0: return i + j * Nq;
  case 1: return j + i * Nq;
  case 2: return ir + j * Nq;
  case 3: return jr + i * Nq;
  case 4: return j + ir * Nq;
  case 5: return i + jr * Nq;
  case 6: return jr + ir * Nq;
  default: return ir + jr * Nq;
  }
}

// glue orientation map mapOp[o][n] (src/bfam.c:7430-7461)
template <int DIM, int N> __device__ __forceinline__ int map_op(int o, int pn)
{
  constexpr int Nq = N + 1;
  if (DIM == 2)
    return o ? N - pn : pn;
  const int i = pn % Nq, j = pn / Nq, ir = N - i, jr = N - j;
  switch (o)
  {
  case 0: return i + j * Nq;
  case 1: return j + i * Nq;
  case 2: return ir + j * Nq;
  case 3: return j + ir * Nq;
  case 4: return jr + i * Nq;
  case 5: return i + jr * Nq;
  case 6: return jr + ir * Nq;
  default: return ir + jr * Nq;
  }
}

// ------------------------------------------------------------- physics

// Jump terms (T* - T-, v* - v-) at one face point.  qm/qp hold the point's
// fields (velocity then stress, bfam field order); nx,ny,nz is the minus
// side's outward unit normal.  Upwind: exact Riemann solution of the normal
// (P, impedance Zp) and tangential (S, impedance Zs) problems; T - Z v
// travels out of the minus side, T + Z v out of the plus side.
template <int DIM, typename CT>
__device__ __forceinline__ void flux_jumps(const CT *qm, const CT *qp, CT nx,
                                           CT ny, CT nz, CT Zpm, CT Zsm, CT Zpp,
                                           CT Zsp, int flux, CT *J)
{
  CT vm[3], vp[3], Tm[3], Tp[3];
  if (DIM == 3)
  {
    vm[0] = qm[0]; vm[1] = qm[1]; vm[2] = qm[2];
    vp[0] = qp[0]; vp[1] = qp[1]; vp[2] = qp[2];
    Tm[0] = qm[3] * nx + qm[6] * ny + qm[7] * nz;
    Tm[1] = qm[6] * nx + qm[4] * ny + qm[8] * nz;
    Tm[2] = qm[7] * nx + qm[8] * ny + qm[5] * nz;
    Tp[0] = qp[3] * nx + qp[6] * ny + qp[7] * nz;
    Tp[1] = qp[6] * nx + qp[4] * ny + qp[8] * nz;
    Tp[2] = qp[7] * nx + qp[8] * ny + qp[5] * nz;
  }
  else
  {
    vm[0] = qm[0]; vm[1] = qm[1]; vm[2] = 0;
    vp[0] = qp[0]; vp[1] = qp[1]; vp[2] = 0;
    Tm[0] = qm[2] * nx + qm[4] * ny;
    Tm[1] = qm[4] * nx + qm[3] * ny;
    Tm[2] = 0;
    Tp[0] = qp[2] * nx + qp[4] * ny;
    Tp[1] = qp[4] * nx + qp[3] * ny;
    Tp[2] = 0;
  }
  const CT n[3] = {nx, ny, nz};
  if (flux == 1)
  {
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      J[a] = CT(0.5) * (Tp[a] - Tm[a]);
      J[3 + a] = CT(0.5) * (vp[a] - vm[a]);
    }
    return;
  }
  const CT vnm = vm[0] * nx + vm[1] * ny + vm[2] * nz;
  const CT vnp = vp[0] * nx + vp[1] * ny + vp[2] * nz;
  const CT Tnm = Tm[0] * nx + Tm[1] * ny + Tm[2] * nz;
  const CT Tnp = Tp[0] * nx + Tp[1] * ny + Tp[2] * nz;
  const CT dvn = (Zpp * (vnp - vnm) + (Tnp - Tnm)) / (Zpm + Zpp);
  const CT dTn = Zpm * dvn;
  const CT isz = CT(1) / (Zsm + Zsp);
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    const CT dvt =
        (Zsp * ((vp[a] - vnp * n[a]) - (vm[a] - vnm * n[a])) +
         ((Tp[a] - Tnp * n[a]) - (Tm[a] - Tnm * n[a]))) *
        isz;
    J[a] = dTn * n[a] + Zsm * dvt;
    J[3 + a] = dvn * n[a] + dvt;
  }
}

// --------------------------------------------------- mortar tensor passes

// dst[c][m + Nq*b] = sum_i A(m,i) src[c][i + Nq*b]  (face axis 0), or for
// axis 1: dst[c][a + Nq*m] = sum_i A(m,i) src[c][a + Nq*i].  1-D faces (2D
// volumes) only have axis 0.  A is column-major A(m,i) = A[m + Nq*i].
template <int DIM, int N, int NT>
__device__ __forceinline__ void face_pass(const double *A, const double *src,
                                          double *dst, int nc, int axis,
                                          bool accumulate)
{
  constexpr int Nq = N + 1;
  constexpr int Nfp = DIM == 3 ? Nq * Nq : Nq;
  for (int w = threadIdx.x; w < nc * Nfp; w += NT)
  {
    const int c = w / Nfp, p = w % Nfp;
    const int a = p % Nq, b = p / Nq;
    const double *s = src + c * Nfp;
    double acc = 0;
    if (axis == 0)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        acc += A[a + Nq * i] * s[i + Nq * b];
    }
    else
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        acc += A[b + Nq * i] * s[a + Nq * i];
    }
    if (accumulate)
      dst[w] += acc;
    else
      dst[w] = acc;
  }
}

// ------------------------------------------------------------ the kernel

template <int DIM, int N, int MODE>
__global__ void __launch_bounds__(Shape<DIM, N>::NT)
    dg_stage_kernel(DomainView d, StageParams sp)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, Nfp = S::Nfp, NF = S::NF,
                NFLD = S::NFLD, NJ = S::NJ, NT = S::NT;
  extern __shared__ __align__(16) double smem[];
  double *sops = smem;
  double *qs = smem + S::OPS_PAD;
  double *jf = qs + S::SM_QS;
  double *mb0 = jf + S::SM_JF;
  double *mb1 = mb0 + S::SM_MB;
  double *mb2 = mb1 + S::SM_MB;
  uint64_t *bar = reinterpret_cast<uint64_t *>(mb2 + S::SM_MB);
  const double *sD = sops;
  const double *sI = sops + Nq * Nq;     // interp[0..2]
  const double *sP = sops + 4 * Nq * Nq; // proj[0..2]
  const double *sw = sops + 7 * Nq * Nq;

  const int e = blockIdx.x;
  const int t = threadIdx.x;
  const size_t fs = d.fs;
  const size_t eoff = (size_t)e * Np;

  // ---- stage the element's state into shared memory
  if constexpr (S::TMA)
  {
    if (t == 0)
      mbar_init(bar, 1);
    __syncthreads();
    if (t == 0)
    {
      mbar_expect_tx(bar, NFLD * Np * sizeof(double));
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        bulk_g2s(qs + c * Np, d.qin + c * fs + eoff, Np * sizeof(double), bar);
    }
  }
  else
  {
    for (int w = t; w < NFLD * Np; w += NT)
      qs[w] = d.qin[(w / Np) * fs + eoff + (w % Np)];
  }
  for (int w = t; w < S::OPS; w += NT)
    sops[w] = d.ops[w];
  double dqr[NFLD];
  if (MODE == MODE_STAGE && t < Np)
  {
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
      dqr[c] = sp.first_stage ? 0.0 : d.dq[c * fs + eoff + t];
  }
  const ElemData me = d.ed[e];
  if constexpr (S::TMA)
  {
    if (!mbar_wait(bar, 0))
      atomicExch(d.err, 1);
  }
  __syncthreads();

  // ---- volume: gradients from shared memory
  double rv[NFLD];
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    if constexpr (DIM == 3)
    {
      double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; // d(v_c)/d(x_a): g[3c + a]
      double sx[3] = {0, 0, 0}, sy[3] = {0, 0, 0}, sz[3] = {0, 0, 0};
#pragma unroll
      for (int m = 0; m < Nq; ++m)
      {
        const double Dx = sD[i + Nq * m], Dy = sD[j + Nq * m],
                     Dz = sD[k + Nq * m];
        const int nx = m + Nq * (j + Nq * k), ny = i + Nq * (m + Nq * k),
                  nz = i + Nq * (j + Nq * m);
#pragma unroll
        for (int c = 0; c < 3; ++c)
        {
          g[3 * c + 0] += Dx * qs[c * Np + nx];
          g[3 * c + 1] += Dy * qs[c * Np + ny];
          g[3 * c + 2] += Dz * qs[c * Np + nz];
        }
        // rows of div S: x (sxx, sxy, sxz), y (sxy, syy, syz), z (sxz, syz, szz)
        sx[0] += Dx * qs[3 * Np + nx];
        sy[0] += Dy * qs[6 * Np + ny];
        sz[0] += Dz * qs[7 * Np + nz];
        sx[1] += Dx * qs[6 * Np + nx];
        sy[1] += Dy * qs[4 * Np + ny];
        sz[1] += Dz * qs[8 * Np + nz];
        sx[2] += Dx * qs[7 * Np + nx];
        sy[2] += Dy * qs[8 * Np + ny];
        sz[2] += Dz * qs[5 * Np + nz];
      }
      const double rx = me.rx, ry = me.ry, rz = me.rz;
#pragma unroll
      for (int c = 0; c < 3; ++c)
      {
        g[3 * c + 0] *= rx;
        g[3 * c + 1] *= ry;
        g[3 * c + 2] *= rz;
        rv[c] = me.irho * (rx * sx[c] + ry * sy[c] + rz * sz[c]);
      }
      const double div = g[0] + g[4] + g[8];
      rv[3] = me.lam * div + 2 * me.mu * g[0];
      rv[4] = me.lam * div + 2 * me.mu * g[4];
      rv[5] = me.lam * div + 2 * me.mu * g[8];
      rv[6] = me.mu * (g[1] + g[3]);
      rv[7] = me.mu * (g[2] + g[6]);
      rv[8] = me.mu * (g[5] + g[7]);
    }
    else
    {
      double g[4] = {0, 0, 0, 0};
      double sx[2] = {0, 0}, sy[2] = {0, 0};
#pragma unroll
      for (int m = 0; m < Nq; ++m)
      {
        const double Dx = sD[i + Nq * m], Dy = sD[j + Nq * m];
        const int nx = m + Nq * j, ny = i + Nq * m;
        g[0] += Dx * qs[0 * Np + nx];
        g[1] += Dy * qs[0 * Np + ny];
        g[2] += Dx * qs[1 * Np + nx];
        g[3] += Dy * qs[1 * Np + ny];
        sx[0] += Dx * qs[2 * Np + nx];
        sy[0] += Dy * qs[4 * Np + ny];
        sx[1] += Dx * qs[4 * Np + nx];
        sy[1] += Dy * qs[3 * Np + ny];
      }
      const double rx = me.rx, ry = me.ry;
      g[0] *= rx;
      g[1] *= ry;
      g[2] *= rx;
      g[3] *= ry;
      rv[0] = me.irho * (rx * sx[0] + ry * sy[0]);
      rv[1] = me.irho * (rx * sx[1] + ry * sy[1]);
      const double div = g[0] + g[3];
      rv[2] = me.lam * div + 2 * me.mu * g[0];
      rv[3] = me.lam * div + 2 * me.mu * g[3];
      rv[4] = me.mu * (g[1] + g[2]);
    }
  }

  // ---- conforming faces: one work item per face node
  for (int w = t; w < NF * Nfp; w += NT)
  {
    const int f = w / Nfp, pn = w % Nfp;
    const int32_t nb = d.nbr[(size_t)e * NF + f];
    if (nb < 0)
      continue;
    const int code = d.nbrf[(size_t)e * NF + f];
    const int fn = code % NF, ns = code / NF;
    const int vm = gmask<DIM, N>(f, pn);
    const int vp = gmask<DIM, N>(fn, face_perm<DIM, N>(ns, pn));
    const size_t noff = (size_t)nb * Np + vp;
    double qm[NFLD], qp[NFLD];
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
    {
      qm[c] = qs[c * Np + vm];
      qp[c] = d.qin[c * fs + noff];
    }
    const ElemData ne = d.ed[nb];
    const int ax = f >> 1;
    const double sg = (f & 1) ? 1.0 : -1.0;
    double J[NJ];
    flux_jumps<DIM, double>(qm, qp, ax == 0 ? sg : 0.0, ax == 1 ? sg : 0.0,
                            ax == 2 ? sg : 0.0, me.Zp, me.Zs, ne.Zp, ne.Zs,
                            sp.flux, J);
#pragma unroll
    for (int c = 0; c < NJ; ++c)
      jf[(f * NJ + c) * Nfp + pn] = J[c];
  }

  // ---- faces through the glue grid (mortars)
  for (int f = 0; f < NF; ++f)
  {
    const int32_t nb = d.nbr[(size_t)e * NF + f];
    if (nb >= 0)
      continue; // uniform across the CTA
    const int32_t g0 = -1 - nb;
    const int hm0 = d.gHm[g0];
    const int ax = f >> 1;
    const double sg = (f & 1) ? 1.0 : -1.0;
    const double nx = ax == 0 ? sg : 0.0, ny = ax == 1 ? sg : 0.0,
                 nz = ax == 2 ? sg : 0.0;
    double *jff = jf + f * NJ * Nfp;
    if (hm0 == 0)
    {
      // same-size or fine side: one glue element covering the whole face
      const int32_t pg = d.gEp[g0];
      const int32_t ep = d.gEm[pg];
      const int fp = d.gFm[pg], hp = d.gHm[pg], o = d.gOp[g0];
      __syncthreads();
      for (int w = t; w < NFLD * Nfp; w += NT)
      {
        const int c = w / Nfp, pn = w % Nfp;
        mb0[w] = d.qin[c * fs + (size_t)ep * Np + gmask<DIM, N>(fp, pn)];
      }
      __syncthreads();
      const double *src = mb0;
      if (hp > 0)
      {
        const int a = (hp - 1) & 1, b = (hp - 1) >> 1;
        face_pass<DIM, N, NT>(sI + (1 + a) * Nq * Nq, mb0,
                              DIM == 3 ? mb2 : mb1, NFLD, 0, false);
        if (DIM == 3)
        {
          __syncthreads();
          face_pass<DIM, N, NT>(sI + (1 + b) * Nq * Nq, mb2, mb1, NFLD, 1,
                                false);
        }
        __syncthreads();
        src = mb1;
      }
      const ElemData ne = d.ed[ep];
      for (int pn = t; pn < Nfp; pn += NT)
      {
        const int vm = gmask<DIM, N>(f, pn);
        const int pp = map_op<DIM, N>(o, pn);
        double qm[NFLD], qp[NFLD], J[NJ];
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
        {
          qm[c] = qs[c * Np + vm];
          qp[c] = src[c * Nfp + pp];
        }
        flux_jumps<DIM, double>(qm, qp, nx, ny, nz, me.Zp, me.Zs, ne.Zp, ne.Zs,
                                sp.flux, J);
#pragma unroll
        for (int c = 0; c < NJ; ++c)
          jff[c * Nfp + pn] = J[c];
      }
    }
    else
    {
      // coarse side: S::NP half-size pieces, projected back and summed
      __syncthreads();
      for (int w = t; w < NJ * Nfp; w += NT)
        jff[w] = 0;
      for (int piece = 0; piece < S::NP; ++piece)
      {
        const int32_t g = g0 + piece;
        const int h = d.gHm[g];
        const int a = (h - 1) & 1, b = (h - 1) >> 1;
        const int32_t pg = d.gEp[g];
        const int32_t ep = d.gEm[pg];
        const int fp = d.gFm[pg], o = d.gOp[g];
        __syncthreads();
        for (int w = t; w < NFLD * Nfp; w += NT)
        {
          const int c = w / Nfp, pn = w % Nfp;
          mb0[w] = d.qin[c * fs + (size_t)ep * Np + gmask<DIM, N>(fp, pn)];
          mb1[w] = qs[c * Np + gmask<DIM, N>(f, pn)];
        }
        __syncthreads();
        face_pass<DIM, N, NT>(sI + (1 + a) * Nq * Nq, mb1, mb2, NFLD, 0,
                              false);
        __syncthreads();
        const double *qmi = mb2;
        if (DIM == 3)
        {
          face_pass<DIM, N, NT>(sI + (1 + b) * Nq * Nq, mb2, mb1, NFLD, 1,
                                false);
          __syncthreads();
          qmi = mb1;
        }
        const ElemData ne = d.ed[ep];
        // jump terms go to the buffer that holds neither trace
        double *Jm = DIM == 3 ? mb2 : mb1;
        for (int pn = t; pn < Nfp; pn += NT)
        {
          const int pp = map_op<DIM, N>(o, pn);
          double qm[NFLD], qp[NFLD], J[NJ];
#pragma unroll
          for (int c = 0; c < NFLD; ++c)
          {
            qm[c] = qmi[c * Nfp + pn];
            qp[c] = mb0[c * Nfp + pp];
          }
          flux_jumps<DIM, double>(qm, qp, nx, ny, nz, me.Zp, me.Zs, ne.Zp,
                                  ne.Zs, sp.flux, J);
#pragma unroll
          for (int c = 0; c < NJ; ++c)
            Jm[c * Nfp + pn] = J[c];
        }
        __syncthreads();
        if (DIM == 3)
        {
          face_pass<DIM, N, NT>(sP + (1 + a) * Nq * Nq, Jm, mb0, NJ, 0, false);
          __syncthreads();
          face_pass<DIM, N, NT>(sP + (1 + b) * Nq * Nq, mb0, jff, NJ, 1, true);
        }
        else
        {
          face_pass<DIM, N, NT>(sP + (1 + a) * Nq * Nq, Jm, jff, NJ, 0, true);
        }
      }
    }
  }
  __syncthreads();

  // ---- lift (lumped LGL mass), combine, stage update
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    const double iwend = 1.0 / sw[0];
    const double r3[3] = {me.rx, me.ry, me.rz};
#pragma unroll
    for (int f = 0; f < NF; ++f)
    {
      const int ax = f >> 1, side = f & 1;
      const int idx = ax == 0 ? i : (ax == 1 ? j : k);
      if (idx != (side ? N : 0))
        continue;
      const int pn = DIM == 3 ? (ax == 0 ? j + Nq * k
                                         : (ax == 1 ? i + Nq * k : i + Nq * j))
                              : (ax == 0 ? j : i);
      const double L = r3[ax] * iwend;
      const double sg = side ? 1.0 : -1.0;
      const double *Jf = jf + f * NJ * Nfp + pn;
      const double dT0 = Jf[0 * Nfp], dT1 = Jf[1 * Nfp], dT2 = Jf[2 * Nfp];
      const double dv0 = Jf[3 * Nfp], dv1 = Jf[4 * Nfp], dv2 = Jf[5 * Nfp];
      const double dvv[3] = {dv0, dv1, dv2};
      const double dvn = sg * dvv[ax];
      if constexpr (DIM == 3)
      {
        rv[0] += L * me.irho * dT0;
        rv[1] += L * me.irho * dT1;
        rv[2] += L * me.irho * dT2;
        const double ll = L * me.lam * dvn, lm = L * me.mu * sg;
        rv[3] += ll + (ax == 0 ? 2 * lm * dv0 : 0.0);
        rv[4] += ll + (ax == 1 ? 2 * lm * dv1 : 0.0);
        rv[5] += ll + (ax == 2 ? 2 * lm * dv2 : 0.0);
        rv[6] += lm * (ax == 1 ? dv0 : 0.0) + lm * (ax == 0 ? dv1 : 0.0);
        rv[7] += lm * (ax == 2 ? dv0 : 0.0) + lm * (ax == 0 ? dv2 : 0.0);
        rv[8] += lm * (ax == 2 ? dv1 : 0.0) + lm * (ax == 1 ? dv2 : 0.0);
      }
      else
      {
        rv[0] += L * me.irho * dT0;
        rv[1] += L * me.irho * dT1;
        const double ll = L * me.lam * dvn, lm = L * me.mu * sg;
        rv[2] += ll + (ax == 0 ? 2 * lm * dv0 : 0.0);
        rv[3] += ll + (ax == 1 ? 2 * lm * dv1 : 0.0);
        rv[4] += lm * (ax == 1 ? dv0 : 0.0) + lm * (ax == 0 ? dv1 : 0.0);
      }
    }
    if constexpr (MODE == MODE_STAGE)
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
      {
        const double dqn = sp.A * dqr[c] + sp.dt * rv[c];
        d.dq[c * fs + eoff + t] = dqn;
        d.qout[c * fs + eoff + t] = qs[c * Np + t] + sp.B * dqn;
      }
    }
    else
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        d.rhs[c * fs + eoff + t] = rv[c];
    }
  }
}

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
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    const double wn = w[i] * w[j] * (DIM == 3 ? w[k] : 1.0);
    const size_t id = (size_t)e * Np + t;
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
    val = wn * (kin + pot);
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
