// Fused DG stage kernel for the isotropic velocity-stress elastic system on
// affine Cartesian elements (sm_100a).
//
// One launch per LSRK stage does, per element (one CTA per element):
//   gather  : every global read of the element is issued up front -- its own
//             state q (and dq) by TMA bulk copies into shared memory, the
//             neighbours' face traces by 8-byte cp.async gathers straight into
//             shared memory.  This gather is the on-device replacement of
//             vmapP and of the bfam_communicator ghost exchange
//             (src/bfam.c:6783-6877, 2418-2679);
//   face    : upwind flux on the gathered traces (conforming faces and the
//             fine side of hanging faces);
//   mortar  : faces that go through the glue grid (2:1 hanging faces,
//             src/bfam.c:7328-7520): on the fine side the coarse neighbour's
//             trace is interpolated to this element's mortar piece
//             (interpolation[1..2]); on the coarse side the element's own trace
//             is interpolated to the four (2D: two) pieces, the flux evaluated
//             there against each fine neighbour and L2-projected back
//             (projection[1..2]) -- all pieces of a face at once;
//   volume  : tensor-product LGL derivative along each axis from shared memory
//             (the BFAM_KRON_* contractions, src/bfam.c:3137-3624);
//   update  : the 2N-storage LSRK stage dq = A dq + dt rhs, q' = q + B dq
//             (bfamo_lsrk_t, src/bfam.h:1840-1846) in the tail, writing the new
//             state to the other state buffer so that every element's
//             neighbours read the stage input unchanged.
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
  // stored jump components: (T* - T-)[0..DIM), (v* - v-)[0..DIM)
  static constexpr int NJ = 2 * DIM;
  static constexpr int NPC = DIM == 3 ? 4 : 2; // mortar pieces per coarse face
  static constexpr int ROWS = DIM == 3 ? Nq : 1; // rows of a face
  static constexpr int work = (Np > NF * Nfp ? Np : NF * Nfp);
  static constexpr int NT = ((work + 31) / 32) * 32 > 1024
                                ? 1024
                                : ((work + 31) / 32) * 32;
  // CTAs per SM the register allocation is sized for (about 96 registers)
  static constexpr int MINB_RAW = 65536 / (NT * 96);
  static constexpr int MINB = MINB_RAW < 1 ? 1 : (MINB_RAW > 8 ? 8 : MINB_RAW);
  static constexpr int OPS = 7 * Nq * Nq + Nq;
  static constexpr int OPS_PAD = (OPS + 1) & ~1; // keep 16-byte alignment
  static constexpr bool TMA = (Np % 2) == 0;     // 16-byte aligned element rows
  static constexpr bool DQ_SMEM = NFLD * Np * 8 <= 20 * 1024;
  // shared memory regions in doubles (all even, so 16-byte aligned)
  static constexpr int SM_QS = NFLD * Np + (NFLD * Np) % 2;
  static constexpr int SM_DQ = DQ_SMEM ? SM_QS : 0;
  static constexpr int SM_PT = NF * NFLD * Nfp + (NF * NFLD * Nfp) % 2;
  static constexpr int SM_OI = NPC * NFLD * Nfp + (NPC * NFLD * Nfp) % 2;
  static constexpr int SM_FC = 4 * (NF + NPC);
  static constexpr int SM_TOTAL =
      OPS_PAD + SM_QS + SM_DQ + SM_PT + 2 * SM_OI + SM_FC + 4;
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

// 8-byte asynchronous gather global -> shared (completes with the group)
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)),
               "l"(src)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int NPENDING> __device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;" ::"n"(NPENDING) : "memory");
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

// Jump terms J = (T* - T-, v* - v-) at one face point.  qm/qp hold the
// point's fields (velocity then stress, bfam field order); n = e_axis * sg is
// the minus side's outward unit normal.  Upwind: exact Riemann solution of
// the normal (P, impedance Zp) and tangential (S, impedance Zs) problems;
// T - Z v travels out of the minus side, T + Z v out of the plus side:
//   v*_n - v-_n = (Zp+ [v_n] + [T_n]) / (Zp- + Zp+),  T*_n - T-_n = Zp- (..)
//   v*_t - v-_t = (Zs+ [v_t] + [T_t]) / (Zs- + Zs+),  T*_t - T-_t = Zs- (..)
// fc = {Zp+, 1/(Zp- + Zp+), Zs+, 1/(Zs- + Zs+)}, computed once per face.
template <int DIM>
__device__ __forceinline__ void flux_jumps(const double *qm, const double *qp,
                                           int ax, double sg, double Zpm,
                                           double Zsm, const double *fc,
                                           int flux, double *J)
{
  double vm[3], vp[3], Tm[3], Tp[3];
  // traction S n with n = sg e_ax: column ax of S times sg (selects, so the
  // field arrays stay in registers)
  const bool x = ax == 0, y = ax == 1;
  if (DIM == 3)
  {
    vm[0] = qm[0]; vm[1] = qm[1]; vm[2] = qm[2];
    vp[0] = qp[0]; vp[1] = qp[1]; vp[2] = qp[2];
    Tm[0] = sg * (x ? qm[3] : (y ? qm[6] : qm[7]));
    Tm[1] = sg * (x ? qm[6] : (y ? qm[4] : qm[8]));
    Tm[2] = sg * (x ? qm[7] : (y ? qm[8] : qm[5]));
    Tp[0] = sg * (x ? qp[3] : (y ? qp[6] : qp[7]));
    Tp[1] = sg * (x ? qp[6] : (y ? qp[4] : qp[8]));
    Tp[2] = sg * (x ? qp[7] : (y ? qp[8] : qp[5]));
  }
  else
  {
    vm[0] = qm[0]; vm[1] = qm[1]; vm[2] = 0;
    vp[0] = qp[0]; vp[1] = qp[1]; vp[2] = 0;
    Tm[0] = sg * (x ? qm[2] : qm[4]);
    Tm[1] = sg * (x ? qm[4] : qm[3]);
    Tm[2] = 0;
    Tp[0] = sg * (x ? qp[2] : qp[4]);
    Tp[1] = sg * (x ? qp[4] : qp[3]);
    Tp[2] = 0;
  }
  if (flux == 1)
  {
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      J[a] = 0.5 * (Tp[a] - Tm[a]);
      J[3 + a] = 0.5 * (vp[a] - vm[a]);
    }
    return;
  }
  double dv[3], dT[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    dv[a] = vp[a] - vm[a];
    dT[a] = Tp[a] - Tm[a];
  }
  // normal parts
  const double dvn = sg * (x ? dv[0] : (y ? dv[1] : dv[2]));
  const double dTn = sg * (x ? dT[0] : (y ? dT[1] : dT[2]));
  const double un = (fc[0] * dvn + dTn) * fc[1];
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    const double na = a == ax ? sg : 0.0;
    const double ut = (fc[2] * (dv[a] - dvn * na) + (dT[a] - dTn * na)) * fc[3];
    J[a] = Zpm * un * na + Zsm * ut;
    J[3 + a] = un * na + ut;
  }
}

__device__ __forceinline__ void face_constants(const ElemData &me,
                                               const ElemData &ne, double *fc)
{
  fc[0] = ne.Zp;
  fc[1] = 1.0 / (me.Zp + ne.Zp);
  fc[2] = ne.Zs;
  fc[3] = 1.0 / (me.Zs + ne.Zs);
}

// slot in the 6-component jump vector of stored component c
template <int DIM> __device__ __forceinline__ constexpr int jslot(int c)
{
  return c < DIM ? c : 3 + (c - DIM);
}

// In-place 1-D operator pass on a face array x[m0 + Nq*m1]:
// axis 0: x[:, m1] <- A x[:, m1];  axis 1: x[m0, :] <- A x[m0, :].
// A is column-major A(m,i) = A[m + Nq*i].  One thread owns one line.
template <int N>
__device__ __forceinline__ void line_apply(const double *A, double *x,
                                           int stride)
{
  constexpr int Nq = N + 1;
  double v[Nq], o[Nq];
#pragma unroll
  for (int i = 0; i < Nq; ++i)
    v[i] = x[i * stride];
#pragma unroll
  for (int m = 0; m < Nq; ++m)
  {
    double s = 0;
#pragma unroll
    for (int i = 0; i < Nq; ++i)
      s += A[m + Nq * i] * v[i];
    o[m] = s;
  }
#pragma unroll
  for (int m = 0; m < Nq; ++m)
    x[m * stride] = o[m];
}

// ------------------------------------------------------------ the kernel

template <int DIM, int N, int MODE>
__global__ void __launch_bounds__(Shape<DIM, N>::NT, Shape<DIM, N>::MINB)
    dg_stage_kernel(DomainView d, StageParams sp)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, Nfp = S::Nfp, NF = S::NF,
                NFLD = S::NFLD, NJ = S::NJ, NT = S::NT, NPC = S::NPC,
                ROWS = S::ROWS;
  extern __shared__ __align__(16) double smem[];
  double *sops = smem;
  double *qs = sops + S::OPS_PAD;
  double *dqs = qs + S::SM_QS;
  double *pt = dqs + S::SM_DQ; // [NF][NFLD][Nfp] plus traces, then jumps
  double *oi = pt + S::SM_PT;  // [NPC][NFLD][Nfp] own trace on mortar pieces
  double *ms = oi + S::SM_OI;  // [NPC][NFLD][Nfp] fine partners' traces
  double *fcf = ms + S::SM_OI; // [NF][4] face flux constants
  double *fcp = fcf + 4 * NF;  // [NPC][4] mortar piece flux constants
  uint64_t *bar = reinterpret_cast<uint64_t *>(fcp + 4 * NPC);
  const double *sD = sops;
  const double *sI = sops + Nq * Nq;     // interp[0..2]
  const double *sP = sops + 4 * Nq * Nq; // proj[0..2]
  const double *sw = sops + 7 * Nq * Nq;

  const int e = blockIdx.x;
  const int t = threadIdx.x;
  const size_t fs = d.fs;
  const size_t eoff = (size_t)e * Np;
  const bool load_dq = MODE == MODE_STAGE && !sp.first_stage;
  const ElemData me = d.ed[e];

  // face kinds: 0 conforming, 1 glue (same size or fine side), 2 coarse side
  int kinds = 0; // 2 bits per face
  int coarse_mask = 0, fine_mask = 0;
#pragma unroll
  for (int f = 0; f < NF; ++f)
  {
    const int32_t nb = d.nbr[(size_t)e * NF + f];
    int k = 0;
    if (nb < 0)
      k = d.gHm[-1 - nb] == 0 ? 1 : 2;
    kinds |= k << (2 * f);
    coarse_mask |= (k == 2) << f;
    fine_mask |= (k == 1) << f;
  }

  // ---------------------------------------------------------- phase 0: issue
  if constexpr (S::TMA)
  {
    if (t == 0)
    {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
    }
    __syncthreads();
    if (t == 0)
    {
      mbar_expect_tx(&bar[0], NFLD * Np * sizeof(double));
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        bulk_g2s(qs + c * Np, d.qin + c * fs + eoff, Np * sizeof(double),
                 &bar[0]);
      if (S::DQ_SMEM && load_dq)
      {
        mbar_expect_tx(&bar[1], NFLD * Np * sizeof(double));
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
          bulk_g2s(dqs + c * Np, d.dq + c * fs + eoff, Np * sizeof(double),
                   &bar[1]);
      }
    }
  }
  else
  {
    for (int w = t; w < NFLD * Np; w += NT)
    {
      cp_async8(qs + w, d.qin + (w / Np) * fs + eoff + (w % Np));
      if (S::DQ_SMEM && load_dq)
        cp_async8(dqs + w, d.dq + (w / Np) * fs + eoff + (w % Np));
    }
  }
  for (int w = t; w < S::OPS; w += NT)
    sops[w] = d.ops[w];

  // neighbour traces of conforming faces and coarse partners of fine-side
  // glue faces, gathered into pt in this element's face-node order
  for (int w = t; w < NF * Nfp; w += NT)
  {
    const int f = w / Nfp, pn = w % Nfp;
    const int k = (kinds >> (2 * f)) & 3;
    if (k == 2)
      continue;
    const int32_t nb = d.nbr[(size_t)e * NF + f];
    int32_t src_e;
    int src_n;
    if (k == 0)
    {
      const int code = d.nbrf[(size_t)e * NF + f];
      src_e = nb;
      src_n = gmask<DIM, N>(code % NF, face_perm<DIM, N>(code / NF, pn));
    }
    else
    {
      const int32_t pg = d.gEp[-1 - nb];
      src_e = d.gEm[pg];
      src_n = gmask<DIM, N>(d.gFm[pg], pn);
    }
    const double *src = d.qin + (size_t)src_e * Np + src_n;
    double *dst = pt + f * NFLD * Nfp + pn;
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
      cp_async8(dst + c * Nfp, src + c * fs);
    if (pn == 0)
      face_constants(me, d.ed[src_e], fcf + 4 * f);
  }
  cp_async_commit(); // group: q (non-TMA path), dq, face traces

  // fine partners of the first coarse-side face
  auto issue_coarse = [&](int f) {
    const int32_t g0 = -1 - d.nbr[(size_t)e * NF + f];
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int32_t pg = d.gEp[g0 + p];
      const int32_t ep = d.gEm[pg];
      const double *src = d.qin + (size_t)ep * Np + gmask<DIM, N>(d.gFm[pg], pn);
      double *dst = ms + p * NFLD * Nfp + pn;
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        cp_async8(dst + c * Nfp, src + c * fs);
      if (pn == 0)
        face_constants(me, d.ed[ep], fcp + 4 * p);
    }
    cp_async_commit();
  };
  int next_coarse = coarse_mask ? __ffs(coarse_mask) - 1 : -1;
  if (next_coarse >= 0)
    issue_coarse(next_coarse);
  else
    cp_async_commit(); // keep the group count uniform

  // ------------------------------------------------- phase 1: faces, mortars
  if constexpr (S::TMA)
  {
    if (!mbar_wait(&bar[0], 0))
      atomicExch(d.err, 1);
  }
  cp_async_wait<1>();
  __syncthreads();

  // fine side: coarse partner trace -> my piece, in place (rows, then columns)
  if (fine_mask)
  {
    for (int pass = 0; pass < (DIM == 3 ? 2 : 1); ++pass)
    {
      for (int w = t; w < NF * NFLD * ROWS; w += NT)
      {
        const int f = w / (NFLD * ROWS), r = w % (NFLD * ROWS);
        if (!((fine_mask >> f) & 1))
          continue;
        const int hp = d.gHm[d.gEp[-1 - d.nbr[(size_t)e * NF + f]]];
        if (hp == 0)
          continue; // same-size glue face: no interpolation
        const int c = r / ROWS, line = r % ROWS;
        const int half = pass == 0 ? (hp - 1) & 1 : (hp - 1) >> 1;
        double *x = pt + (f * NFLD + c) * Nfp;
        if (pass == 0)
          line_apply<N>(sI + (1 + half) * Nq * Nq, x + Nq * line, 1);
        else
          line_apply<N>(sI + (1 + half) * Nq * Nq, x + line, Nq);
      }
      __syncthreads();
    }
  }

  // flux on conforming and fine-side faces: read, barrier, write in place
  {
    double J[6];
    int my_f = -1, my_pn = 0;
    if (t < NF * Nfp)
    {
      const int f = t / Nfp, pn = t % Nfp;
      const int k = (kinds >> (2 * f)) & 3;
      if (k != 2)
      {
        my_f = f;
        my_pn = pn;
        const int vm = gmask<DIM, N>(f, pn);
        int pp = pn;
        if (k == 1)
          pp = map_op<DIM, N>(d.gOp[-1 - d.nbr[(size_t)e * NF + f]], pn);
        double qm[NFLD], qp[NFLD];
        const double *x = pt + f * NFLD * Nfp;
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
        {
          qm[c] = qs[c * Np + vm];
          qp[c] = x[c * Nfp + pp];
        }
        flux_jumps<DIM>(qm, qp, f >> 1, (f & 1) ? 1.0 : -1.0, me.Zp, me.Zs,
                        fcf + 4 * f, sp.flux, J);
      }
    }
    __syncthreads();
    if (my_f >= 0)
    {
#pragma unroll
      for (int c = 0; c < NJ; ++c)
        pt[(my_f * NFLD + c) * Nfp + my_pn] = J[jslot<DIM>(c)];
    }
  }

  // coarse side: all pieces of one face at a time
  while (next_coarse >= 0)
  {
    const int f = next_coarse;
    coarse_mask &= ~(1 << f);
    next_coarse = coarse_mask ? __ffs(coarse_mask) - 1 : -1;
    const int32_t g0 = -1 - d.nbr[(size_t)e * NF + f];
    cp_async_wait<0>();
    __syncthreads(); // ms holds this face's partners; oi is free
    // own face trace -> pieces, along face axis 0
    for (int w = t; w < NPC * NFLD * ROWS; w += NT)
    {
      const int p = w / (NFLD * ROWS), r = w % (NFLD * ROWS);
      const int c = r / ROWS, line = r % ROWS;
      const int h = d.gHm[g0 + p];
      const double *A = sI + (1 + ((h - 1) & 1)) * Nq * Nq;
      double v[Nq];
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        v[i] = qs[c * Np + gmask<DIM, N>(f, i + Nq * line)];
      double *x = oi + (p * NFLD + c) * Nfp + Nq * line;
#pragma unroll
      for (int m = 0; m < Nq; ++m)
      {
        double s = 0;
#pragma unroll
        for (int i = 0; i < Nq; ++i)
          s += A[m + Nq * i] * v[i];
        x[m] = s;
      }
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NFLD * Nq; w += NT)
      {
        const int p = w / (NFLD * Nq), r = w % (NFLD * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = d.gHm[g0 + p];
        line_apply<N>(sI + (1 + ((h - 1) >> 1)) * Nq * Nq,
                      oi + (p * NFLD + c) * Nfp + col, Nq);
      }
      __syncthreads();
    }
    // flux on the pieces; jumps overwrite the own trace in place
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int pp = map_op<DIM, N>(d.gOp[g0 + p], pn);
      double qm[NFLD], qp[NFLD], J[6];
      double *x = oi + p * NFLD * Nfp;
      const double *y = ms + p * NFLD * Nfp;
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
      {
        qm[c] = x[c * Nfp + pn];
        qp[c] = y[c * Nfp + pp];
      }
      flux_jumps<DIM>(qm, qp, f >> 1, (f & 1) ? 1.0 : -1.0, me.Zp, me.Zs,
                      fcp + 4 * p, sp.flux, J);
#pragma unroll
      for (int c = 0; c < NJ; ++c)
        x[c * Nfp + pn] = J[jslot<DIM>(c)];
    }
    __syncthreads(); // ms and fcp free: fetch the next face's partners
    if (next_coarse >= 0)
      issue_coarse(next_coarse);
    // L2 projection back to the coarse face: axis 0, (axis 1), sum of pieces
    for (int w = t; w < NPC * NJ * ROWS; w += NT)
    {
      const int p = w / (NJ * ROWS), r = w % (NJ * ROWS);
      const int c = r / ROWS, line = r % ROWS;
      const int h = d.gHm[g0 + p];
      line_apply<N>(sP + (1 + ((h - 1) & 1)) * Nq * Nq,
                    oi + (p * NFLD + c) * Nfp + Nq * line, 1);
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NJ * Nq; w += NT)
      {
        const int p = w / (NJ * Nq), r = w % (NJ * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = d.gHm[g0 + p];
        line_apply<N>(sP + (1 + ((h - 1) >> 1)) * Nq * Nq,
                      oi + (p * NFLD + c) * Nfp + col, Nq);
      }
      __syncthreads();
    }
    for (int w = t; w < NJ * Nfp; w += NT)
    {
      const int c = w / Nfp, pn = w % Nfp;
      double s = 0;
#pragma unroll
      for (int p = 0; p < NPC; ++p)
        s += oi[(p * NFLD + c) * Nfp + pn];
      pt[(f * NFLD + c) * Nfp + pn] = s;
    }
  }
  __syncthreads();

  // --------------------------------------------- phase 2: volume and update
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    double rv[NFLD];
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

    // lift of the face jump terms with the lumped LGL mass
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
      const double *Jf = pt + f * NFLD * Nfp + pn;
      const double dT0 = Jf[0 * Nfp], dT1 = Jf[1 * Nfp];
      const double dT2 = DIM == 3 ? Jf[2 * Nfp] : 0.0;
      const double dv0 = Jf[DIM * Nfp], dv1 = Jf[(DIM + 1) * Nfp];
      const double dv2 = DIM == 3 ? Jf[5 * Nfp] : 0.0;
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
      double dqo[NFLD];
      if (load_dq)
      {
        if constexpr (S::DQ_SMEM)
        {
          if constexpr (S::TMA)
          {
            if (!mbar_wait(&bar[1], 0))
              atomicExch(d.err, 2);
          }
#pragma unroll
          for (int c = 0; c < NFLD; ++c)
            dqo[c] = dqs[c * Np + t];
        }
        else
        {
#pragma unroll
          for (int c = 0; c < NFLD; ++c)
            dqo[c] = d.dq[c * fs + eoff + t];
        }
      }
      else
      {
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
          dqo[c] = 0.0;
      }
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
      {
        const double dqn = sp.A * dqo[c] + sp.dt * rv[c];
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
