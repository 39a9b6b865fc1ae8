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
//   volume  : while the gathers are in flight: the tensor-product LGL
//             derivative, one pass per axis with one thread per (line, field)
//             -- the BFAM_KRON_IXIXA / IXAXI / AXIXI contractions of
//             src/bfam.c:3519-3624 restated per line -- accumulated straight
//             into A dq + dt rhs in the dq tile;
//   face    : upwind flux on the gathered traces (conforming faces and the
//             fine side of hanging faces);
//   mortar  : faces that go through the glue grid (2:1 hanging faces,
//             src/bfam.c:7328-7520): on the fine side the coarse neighbour's
//             trace is interpolated to this element's mortar piece
//             (interpolation[1..2]); on the coarse side the element's own trace
//             is interpolated to the four (2D: two) pieces, the flux evaluated
//             there against each fine neighbour and L2-projected back
//             (projection[1..2]) -- all pieces of a face at once;
//   update  : lift of the face terms with the lumped LGL mass and the 2N-storage
//             LSRK stage dq = A dq + dt rhs, q' = q + B dq (bfamo_lsrk_t,
//             src/bfam.h:1840-1846), writing the new state to the other state
//             buffer so that every element's neighbours read the stage input
//             unchanged.
//
// State layout in HBM: field-major, element, node (bfam's per-field arrays
// stacked): q[f * K * Np + e * Np + n], n = i + Nq (j + Nq k).
#pragma once

#include "dg_common.cuh"

namespace bfam_b200
{

// One axis of the volume operator for one (line, field) work item: the
// derivative along the line (constant-bank D) and its contributions to the
// right-hand-side fields, accumulated into R = A dq + s rhs (the first axis
// initialises R from a * dq when rd, from zero otherwise).
//   rho dv/dt = div S,  dS/dt = lambda div(v) I + mu (grad v + grad v^T)
template <int DIM, int N, int AXIS>
__device__ __forceinline__ void volume_axis(const DiffOp<N> &dop,
                                            const double *qs, double *R,
                                            const ElemData &me, int w,
                                            double a, double s, bool rd)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, NL = S::NL;
  const int line = w % NL, fsel = w / NL;
  int base, stride;
  if (AXIS == 0)
  {
    base = line * Nq;
    stride = 1;
  }
  else if (AXIS == 1)
  {
    base = (line % Nq) + Nq * Nq * (line / Nq);
    stride = Nq;
  }
  else
  {
    base = line;
    stride = Nq * Nq;
  }
  const double r = s * (AXIS == 0 ? me.rx : (AXIS == 1 ? me.ry : me.rz));
  // differentiated field per (axis, fsel), bfam field order:
  // 3D x: vx vy vz sxx sxy sxz | y: vx vy vz sxy syy syz | z: vx vy vz sxz syz szz
  // 2D x: vx vy sxx sxy        | y: vx vy sxy syy
  int c;
  if (DIM == 3)
  {
    const int k = fsel - 3;
    if (fsel < 3)
      c = fsel;
    else if (AXIS == 0)
      c = k == 0 ? 3 : (k == 1 ? 6 : 7);
    else if (AXIS == 1)
      c = k == 0 ? 6 : (k == 1 ? 4 : 8);
    else
      c = k == 0 ? 7 : (k == 1 ? 8 : 5);
  }
  else
  {
    if (fsel < 2)
      c = fsel;
    else if (AXIS == 0)
      c = fsel == 2 ? 2 : 4;
    else
      c = fsel == 2 ? 4 : 3;
  }
  double v[Nq], dv[Nq];
  const double *src = qs + c * Np + base;
#pragma unroll
  for (int m = 0; m < Nq; ++m)
    v[m] = src[m * stride];
#pragma unroll
  for (int i = 0; i < Nq; ++i)
  {
    double acc = 0;
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      acc += dop.D[i + Nq * m] * v[m];
    dv[i] = r * acc;
  }
  const double l2m = me.lam + 2 * me.mu;
  auto put = [&](int tgt, double coef) {
    double *dst = R + tgt * Np + base;
#pragma unroll
    for (int i = 0; i < Nq; ++i)
    {
      if (AXIS == 0)
        dst[i * stride] = (rd ? a * dst[i * stride] : 0.0) + coef * dv[i];
      else
        dst[i * stride] += coef * dv[i];
    }
  };
  if (DIM == 3)
  {
    if (fsel < 3)
    {
      if (fsel == AXIS)
      {
        put(3, AXIS == 0 ? l2m : me.lam);
        put(4, AXIS == 1 ? l2m : me.lam);
        put(5, AXIS == 2 ? l2m : me.lam);
      }
      else
      {
        // shear: d v_fsel / d x_AXIS -> S_{fsel,AXIS}
        const int lo = fsel < AXIS ? fsel : AXIS, hi = fsel < AXIS ? AXIS : fsel;
        put((lo == 0 && hi == 1) ? 6 : ((lo == 0) ? 7 : 8), me.mu);
        if (AXIS == 0 && fsel == 2)
        {
          // syz gets nothing along x: start it from A dq here
          double *dst = R + 8 * Np + base;
#pragma unroll
          for (int i = 0; i < Nq; ++i)
            dst[i * stride] = rd ? a * dst[i * stride] : 0.0;
        }
      }
    }
    else
      put(fsel - 3, me.irho); // rows of div S -> vx, vy, vz
  }
  else
  {
    if (fsel < 2)
    {
      if (fsel == AXIS)
      {
        put(2, AXIS == 0 ? l2m : me.lam);
        put(3, AXIS == 1 ? l2m : me.lam);
      }
      else
        put(4, me.mu);
    }
    else
      put(fsel - 2, me.irho);
  }
}

template <int DIM, int N, int MODE>
__global__ void __launch_bounds__(Shape<DIM, N>::NT, Shape<DIM, N>::MINB)
    dg_stage_kernel(DomainView d, StageParams sp, DiffOp<N> dop)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, Nfp = S::Nfp, NF = S::NF,
                NFLD = S::NFLD, NJ = S::NJ, NT = S::NT, NPC = S::NPC,
                ROWS = S::ROWS, NL = S::NL, NDF = S::NDF;
  extern __shared__ __align__(16) double smem[];
  double *qs = smem;
  double *R = qs + S::SM_QS;   // dq tile, becomes A dq + s rhs
  double *pt = R + S::SM_DQ;   // [NF][NFLD][Nfp] plus traces, then jumps
  double *oi = pt + S::SM_PT;  // [NPC][NFLD][Nfp] own trace on mortar pieces
  double *ms = oi + S::SM_OI;  // [NPC][NFLD][Nfp] fine partners' traces
  double *fcf = oi + S::SM_MOR; // [NF][4] face flux constants
  double *fcp = fcf + 4 * NF;   // [NPC][4] piece flux constants
  double *sIP = fcp + 4 * NPC;  // interp to bottom/top, proj from bottom/top
  uint64_t *bar = reinterpret_cast<uint64_t *>(sIP + S::SM_IP);
  const double *sIb = sIP, *sIt = sIP + Nq * Nq;
  const double *sPb = sIP + 2 * Nq * Nq, *sPt = sIP + 3 * Nq * Nq;

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
    for (int c = 0; c < NFLD; ++c)
      cp_async8(dst + c * Nfp, src + c * fs);
    if (pn == 0)
    {
      const double *fc = reinterpret_cast<const double *>(d.fcE + (size_t)e * NF + f);
      cp_async16(fcf + 4 * f, fc);
      cp_async16(fcf + 4 * f + 2, fc + 2);
    }
  }
  // mortar operators: interpolation[1..2], projection[1..2]
  for (int w = t; w < 4 * Nq * Nq; w += NT)
  {
    const int which = w / (Nq * Nq), idx = w % (Nq * Nq);
    cp_async8(sIP + w, d.ops + (which < 2 ? 2 + which : 3 + which) * Nq * Nq + idx);
  }
  cp_async_commit(); // face traces, flux constants, mortar operators

  // fine partners of one coarse-side face
  auto issue_coarse = [&](int f) {
    const int32_t g0 = desc[f].x;
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int2 gp = d.gpart[g0 + p];
      const double *src = d.qin + (size_t)gp.x * Np + gmask<DIM, N>(gp.y & 7, pn);
      double *dst = ms + p * NFLD * Nfp + pn;
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        cp_async8(dst + c * Nfp, src + c * fs);
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

  // ------------------------------- phase 1: volume while the gathers fly
  if constexpr (S::TMA)
  {
    if (!mbar_wait(&bar[0], 0))
      atomicExch(d.err, 1);
    if (rd && !mbar_wait(&bar[1], 0))
      atomicExch(d.err, 2);
  }
  else
  {
    cp_async_wait<2>(); // own state (face-trace groups may still fly)
  }
  __syncthreads();
  for (int w = t; w < NL * NDF; w += NT)
    volume_axis<DIM, N, 0>(dop, qs, R, me, w, a, s, rd);
  __syncthreads();
  for (int w = t; w < NL * NDF; w += NT)
    volume_axis<DIM, N, 1>(dop, qs, R, me, w, a, s, rd);
  if (DIM == 3)
  {
    __syncthreads();
    for (int w = t; w < NL * NDF; w += NT)
      volume_axis<DIM, N, (DIM == 3 ? 2 : 1)>(dop, qs, R, me, w, a, s, rd);
  }

  // ------------------------------------------------- phase 2: faces, mortars
  cp_async_wait<1>(); // face traces
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
        const int hp = (desc[f].y >> 8) & 7;
        const int c = r / ROWS, line = r % ROWS;
        const int half = pass == 0 ? (hp - 1) & 1 : (hp - 1) >> 1;
        double *x = pt + (f * NFLD + c) * Nfp;
        if (pass == 0)
          line_apply<N>(half ? sIt : sIb, x + Nq * line, 1);
        else
          line_apply<N>(half ? sIt : sIb, x + line, Nq);
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
      const int y = desc[f].y;
      const int k = y & 3;
      if (k != 2)
      {
        my_f = f;
        my_pn = pn;
        const int vm = gmask<DIM, N>(f, pn);
        const int pp = k == 1 ? map_op<DIM, N>((y >> 5) & 7, pn) : pn;
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
    const int32_t g0 = desc[f].x;
    cp_async_wait<0>();
    __syncthreads(); // ms holds this face's partners; oi is free
    // own face trace -> pieces, along face axis 0
    for (int w = t; w < NPC * NFLD * ROWS; w += NT)
    {
      const int p = w / (NFLD * ROWS), r = w % (NFLD * ROWS);
      const int c = r / ROWS, line = r % ROWS;
      const int h = (d.gpart[g0 + p].y >> 6) & 7;
      double v[Nq], o[Nq];
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        v[i] = qs[c * Np + gmask<DIM, N>(f, i + Nq * line)];
      apply_smem<N>(((h - 1) & 1) ? sIt : sIb, v, o);
      double *x = oi + (p * NFLD + c) * Nfp + Nq * line;
#pragma unroll
      for (int m = 0; m < Nq; ++m)
        x[m] = o[m];
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NFLD * Nq; w += NT)
      {
        const int p = w / (NFLD * Nq), r = w % (NFLD * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = (d.gpart[g0 + p].y >> 6) & 7;
        line_apply<N>(((h - 1) >> 1) ? sIt : sIb, oi + (p * NFLD + c) * Nfp + col,
                      Nq);
      }
      __syncthreads();
    }
    // flux on the pieces; jumps overwrite the own trace in place
    for (int w = t; w < NPC * Nfp; w += NT)
    {
      const int p = w / Nfp, pn = w % Nfp;
      const int pp = map_op<DIM, N>((d.gpart[g0 + p].y >> 3) & 7, pn);
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
      const int h = (d.gpart[g0 + p].y >> 6) & 7;
      line_apply<N>(((h - 1) & 1) ? sPt : sPb,
                    oi + (p * NFLD + c) * Nfp + Nq * line, 1);
    }
    __syncthreads();
    if (DIM == 3)
    {
      for (int w = t; w < NPC * NJ * Nq; w += NT)
      {
        const int p = w / (NJ * Nq), r = w % (NJ * Nq);
        const int c = r / Nq, col = r % Nq;
        const int h = (d.gpart[g0 + p].y >> 6) & 7;
        line_apply<N>(((h - 1) >> 1) ? sPt : sPb,
                      oi + (p * NFLD + c) * Nfp + col, Nq);
      }
      __syncthreads();
    }
    for (int w = t; w < NJ * Nfp; w += NT)
    {
      const int c = w / Nfp, pn = w % Nfp;
      double sum = 0;
#pragma unroll
      for (int p = 0; p < NPC; ++p)
        sum += oi[(p * NFLD + c) * Nfp + pn];
      pt[(f * NFLD + c) * Nfp + pn] = sum;
    }
  }
  __syncthreads();

  // --------------------------------------- phase 3: lift, combine and update
  if (t < Np)
  {
    const int i = t % Nq, j = (t / Nq) % Nq, k = t / (Nq * Nq);
    double rv[NFLD];
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
      rv[c] = R[c * Np + t];

    // lift of the face jump terms with the lumped LGL mass
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
      const double L = s * r3[ax] * dop.iwend;
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
