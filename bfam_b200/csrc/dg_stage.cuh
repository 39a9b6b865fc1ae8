// Fused DG stage kernel for the isotropic velocity-stress elastic system on
// affine Cartesian elements (sm_100a).
//
// One launch per LSRK stage does, per element (one CTA per element):
//   issue   : every global read of the element is issued up front -- its own
//             q and dq by TMA bulk copies into shared memory, the neighbours'
//             face traces by 8-byte cp.async gathers straight into shared
//             memory, addressed from a per-face descriptor.  This is the
//             on-device replacement of vmapP and of the bfam_communicator
//             ghost exchange (src/bfam.c:6783-6877, 2418-2679);
//   face    : upwind flux on the gathered traces (conforming faces and the
//             fine side of hanging faces), lifted with the lumped LGL mass to
//             per-node field contributions;
//   mortar  : faces that go through the glue grid (2:1 hanging faces,
//             src/bfam.c:7328-7520): on the fine side the coarse neighbour's
//             trace is interpolated to this element's mortar piece
//             (interpolation[1..2]); on the coarse side the element's own trace
//             is interpolated to the four (2D: two) pieces, the flux evaluated
//             there against each fine neighbour and L2-projected back
//             (projection[1..2]) -- all pieces of a face at once;
//   volume  : one thread per node, the tensor-product LGL derivative along each
//             axis (the BFAM_KRON_IXIXA / IXAXI / AXIXI contractions of
//             src/bfam.c:3519-3624 at one node), plus the node's face
//             contributions;
//   update  : the 2N-storage LSRK stage dq = A dq + dt rhs, q' = q + B dq
//             (bfamo_lsrk_t, src/bfam.h:1840-1846), writing the new state to
//             the other state buffer so that every element's neighbours read
//             the stage input unchanged.
//
// State layout in HBM: field-major, element, node (bfam's per-field arrays
// stacked): q[f * K * Np + e * Np + n], n = i + Nq (j + Nq k).
#pragma once

#include "dg_common.cuh"
#include "dg_volume.cuh"

namespace bfam_b200
{

template <int DIM, int N, int MODE>
__global__ void __launch_bounds__(Shape<DIM, N>::NT, Shape<DIM, N>::MINB)
    dg_stage_kernel(DomainView d, StageParams sp, DiffOp<N> dop)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, Nfp = S::Nfp, NF = S::NF,
                NFLD = S::NFLD, NJ = S::NJ, NT = S::NT, NPC = S::NPC,
                ROWS = S::ROWS, NTF = S::NTF;
  extern __shared__ __align__(16) double smem[];
  double *qs = smem;
  double *R = qs + S::SM_QS;   // dq tile, becomes A dq + s rhs
  double *pt = R + S::SM_DQ;   // [NF][NFLD][Nfp] plus traces, then jumps
  double *oi = pt + S::SM_PT;  // [NPC][NFLD][Nfp] own trace on mortar pieces
  double *ms = oi + S::SM_OI;  // [NPC][NFLD][Nfp] fine partners' traces
  double *fcf = oi + S::SM_MOR; // [NF][4] face flux constants
  double *fcp = fcf + 4 * NF;   // [NPC][4] piece flux constants
  double *sD = fcp + 4 * NPC;   // differentiation matrix
  uint64_t *bar = reinterpret_cast<uint64_t *>(sD + S::SM_IP);

  const int e = blockIdx.x;
  const int t = threadIdx.x;
  const size_t fs = d.fs;
  const size_t eoff = (size_t)e * Np;
  // R = a dq + s rhs: the stage update (A, dt) or the plain right-hand side
  const bool rd = MODE == MODE_STAGE && !sp.first_stage;
  const double a = MODE == MODE_STAGE ? sp.A : 0.0;
  const double s = MODE == MODE_STAGE ? sp.dt : 1.0;
  const ElemData me = d.ed[e];
  const int2 *desc = d.fdesc + (size_t)e * NF;

  int kinds = 0, coarse_mask = 0, fine_mask = 0;
#pragma unroll
  for (int f = 0; f < NF; ++f)
  {
    const int k = desc[f].y & 3;
    kinds |= k << (2 * f);
    coarse_mask |= (k == 2) << f;
    fine_mask |= (k == 1 && ((desc[f].y >> 8) & 7) != 0) << f;
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
      if (rd)
      {
        mbar_expect_tx(&bar[1], NFLD * Np * sizeof(double));
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
          bulk_g2s(R + c * Np, d.dq + c * fs + eoff, Np * sizeof(double),
                   &bar[1]);
      }
    }
  }
  else
  {
    for (int w = t; w < NFLD * Np; w += NT)
    {
      cp_async8(qs + w, d.qin + (w / Np) * fs + eoff + (w % Np));
      if (rd)
        cp_async8(R + w, d.dq + (w / Np) * fs + eoff + (w % Np));
    }
    cp_async_commit(); // own state
  }

  // neighbour traces of conforming faces and coarse partners of fine-side
  // glue faces, gathered into pt in this element's face-node order
  for (int w = t; w < NF * Nfp; w += NT)
  {
    const int f = w / Nfp, pn = w % Nfp;
    const int2 ds = desc[f];
    const int k = ds.y & 3;
    if (k == 2)
      continue;
    const int nface = (ds.y >> 2) & 7;
    const int src_n = k == 0 ? gmask<DIM, N>(nface, face_perm<DIM, N>((ds.y >> 5) & 7, pn))
                             : gmask<DIM, N>(nface, pn);
    const double *src = d.qin + (size_t)ds.x * Np + src_n;
    double *dst = pt + f * NFLD * Nfp + pn;
#pragma unroll
    for (int c = 0; c < NTF; ++c)
      cp_async8(dst + c * Nfp, src + trace_field<DIM>(f >> 1, c) * fs);
    if (pn == 0)
    {
      const double *fc = reinterpret_cast<const double *>(d.fcE + (size_t)e * NF + f);
      cp_async16(fcf + 4 * f, fc);
      cp_async16(fcf + 4 * f + 2, fc + 2);
    }
  }
  cp_async_commit(); // face traces, flux constants

  // fine partners of one coarse-side face
  auto issue_coarse = [&](int f) {
    const int32_t g0 = desc[f].x;
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int2 gp = d.gpart[g0 + p];
      const double *src = d.qin + (size_t)gp.x * Np + gmask<DIM, N>(gp.y & 7, pn);
      double *dst = ms + p * NTF * Nfp + pn;
#pragma unroll
      for (int c = 0; c < NTF; ++c)
        cp_async8(dst + c * Nfp, src + trace_field<DIM>(f >> 1, c) * fs);
      if (pn == 0)
      {
        const double *fc = reinterpret_cast<const double *>(d.fcG + g0 + p);
        cp_async16(fcp + 4 * p, fc);
        cp_async16(fcp + 4 * p + 2, fc + 2);
      }
    }
    cp_async_commit();
  };
  int next_coarse = coarse_mask ? __ffs(coarse_mask) - 1 : -1;
  if (next_coarse >= 0)
    issue_coarse(next_coarse);
  else
    cp_async_commit(); // keep the group count uniform

  // differentiation matrix into shared memory (indexed per thread later)
  for (int w = t; w < Nq * Nq; w += NT)
    sD[w] = dop.D[w];

  // ------------------------------------------------- phase 1: faces, mortars
  if constexpr (S::TMA)
  {
    if (!mbar_wait(&bar[0], 0))
      atomicExch(d.err, 1);
  }
  cp_async_wait<1>(); // own state (non-TMA path), face traces
  __syncthreads();
  // lift factor of face axis ax: s (2/h_ax) / w_0
  const double Lx = s * me.rx * dop.iwend, Ly = s * me.ry * dop.iwend,
               Lz = s * me.rz * dop.iwend;
  auto lfac = [&](int ax) { return ax == 0 ? Lx : (ax == 1 ? Ly : Lz); };

  // fine side: coarse partner trace -> my piece, in place (rows, then columns)
  if (fine_mask)
  {
    for (int pass = 0; pass < (DIM == 3 ? 2 : 1); ++pass)
    {
      for (int w = t; w < NF * NTF * ROWS; w += NT)
      {
        const int f = w / (NTF * ROWS), r = w % (NTF * ROWS);
        if (!((fine_mask >> f) & 1))
          continue;
        const int hp = (desc[f].y >> 8) & 7;
        const int c = r / ROWS, line = r % ROWS;
        const int half = pass == 0 ? (hp - 1) & 1 : (hp - 1) >> 1;
        double *x = pt + (f * NFLD + c) * Nfp;
        if (pass == 0)
          line_apply<N, false>(dop, half, x + Nq * line, 1);
        else
          line_apply<N, false>(dop, half, x + line, Nq);
      }
      __syncthreads();
    }
  }

  // flux on conforming and fine-side faces, lifted to the face node's field
  // contributions: read, barrier, write in place
  {
    double lc[NFLD];
    int my_f = -1, my_pn = 0;
    if (t < NF * Nfp)
    {
      const int f = t / Nfp, pn = t % Nfp;
      const int y = desc[f].y;
      const int k = y & 3;
      if (k != 2)
      {
        my_f = f;
        my_pn = pn;
        const int vm = gmask<DIM, N>(f, pn);
        const int pp = k == 1 ? map_op<DIM, N>((y >> 5) & 7, pn) : pn;
        double qm[NTF], qp[NTF], J[6];
        const double *x = pt + f * NFLD * Nfp;
#pragma unroll
        for (int c = 0; c < NTF; ++c)
        {
          qm[c] = qs[trace_field<DIM>(f >> 1, c) * Np + vm];
          qp[c] = x[c * Nfp + pp];
        }
        const double sg = (f & 1) ? 1.0 : -1.0;
        flux_jumps<DIM>(qm, qp, f >> 1, sg, me.Zp, me.Zs, fcf + 4 * f, sp.flux,
                        J);
        lift_face<DIM>(J, f >> 1, sg, lfac(f >> 1), me, lc);
      }
    }
    __syncthreads();
    if (my_f >= 0)
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        pt[(my_f * NFLD + c) * Nfp + my_pn] = lc[c];
    }
  }

  // coarse side: all pieces of one face at a time
  while (next_coarse >= 0)
  {
    const int f = next_coarse;
    coarse_mask &= ~(1 << f);
    next_coarse = coarse_mask ? __ffs(coarse_mask) - 1 : -1;
    const int32_t g0 = desc[f].x;
    cp_async_wait<0>();
    __syncthreads(); // ms holds this face's partners; oi is free
    // own face trace -> pieces, along face axis 0
    for (int w = t; w < NPC * NTF * ROWS; w += NT)
    {
      const int p = w / (NTF * ROWS), r = w % (NTF * ROWS);
      const int c = r / ROWS, line = r % ROWS;
      const int h = (d.gpart[g0 + p].y >> 6) & 7;
      const double *src = qs + trace_field<DIM>(f >> 1, c) * Np;
      double v[Nq];
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        v[i] = src[gmask<DIM, N>(f, i + Nq * line)];
      apply_half<N, false>(dop, (h - 1) & 1, v, v);
      double *x = oi + (p * NTF + c) * Nfp + Nq * line;
#pragma unroll
      for (int m = 0; m < Nq; ++m)
        x[m] = v[m];
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NTF * Nq; w += NT)
      {
        const int p = w / (NTF * Nq), r = w % (NTF * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = (d.gpart[g0 + p].y >> 6) & 7;
        line_apply<N, false>(dop, (h - 1) >> 1, oi + (p * NTF + c) * Nfp + col,
                             Nq);
      }
      __syncthreads();
    }
    // flux on the pieces; jumps overwrite the own trace in place
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int pp = map_op<DIM, N>((d.gpart[g0 + p].y >> 3) & 7, pn);
      double qm[NTF], qp[NTF], J[6];
      double *x = oi + p * NTF * Nfp;
      const double *y = ms + p * NTF * Nfp;
#pragma unroll
      for (int c = 0; c < NTF; ++c)
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
      const int h = (d.gpart[g0 + p].y >> 6) & 7;
      line_apply<N, true>(dop, (h - 1) & 1, oi + (p * NTF + c) * Nfp + Nq * line,
                          1);
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NJ * Nq; w += NT)
      {
        const int p = w / (NJ * Nq), r = w % (NJ * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = (d.gpart[g0 + p].y >> 6) & 7;
        line_apply<N, true>(dop, (h - 1) >> 1, oi + (p * NTF + c) * Nfp + col,
                            Nq);
      }
      __syncthreads();
    }
    for (int pn = t; pn < Nfp; pn += NT)
    {
      double J[6] = {0, 0, 0, 0, 0, 0}, lc[NFLD];
#pragma unroll
      for (int c = 0; c < NJ; ++c)
      {
        double sum = 0;
#pragma unroll
        for (int p = 0; p < NPC; ++p)
          sum += oi[(p * NTF + c) * Nfp + pn];
        J[jslot<DIM>(c)] = sum;
      }
      lift_face<DIM>(J, f >> 1, (f & 1) ? 1.0 : -1.0, lfac(f >> 1), me, lc);
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        pt[(f * NFLD + c) * Nfp + pn] = lc[c];
    }
  }
  __syncthreads();

  // ------------------------ phase 2: volume, face contributions and update
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    double rv[NFLD];
    volume_node<DIM, N>(qs, sD, me, s, i, j, k, rv);

    // lifted face contributions of the faces this node lies on
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
      const double *lc = pt + f * NFLD * Nfp + pn;
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        rv[c] += lc[c * Nfp];
    }

    if constexpr (MODE == MODE_STAGE)
    {
      if (rd)
      {
        if constexpr (S::TMA)
        {
          if (!mbar_wait(&bar[1], 0))
            atomicExch(d.err, 2);
        }
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
          rv[c] += a * R[c * Np + t];
      }
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
      {
        d.dq[c * fs + eoff + t] = rv[c];
        d.qout[c * fs + eoff + t] = qs[c * Np + t] + sp.B * rv[c];
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

} // namespace bfam_b200
