// Fused DG stage kernel for the isotropic velocity-stress elastic system on
// affine Cartesian elements (sm_100a).
//
// One element per CTA iteration does:
//   issue   : every global read of the element is issued up front -- its own
//             q (and dq, where the shape stages it; else an L2 prefetch of
//             it) and its faces' flux constants by TMA bulk copies into
//             shared memory, the neighbours' face traces by 8-byte cp.async
//             gathers straight into shared memory, addressed from a
//             per-face descriptor.  This is the
//             on-device replacement of vmapP and of the bfam_communicator
//             ghost exchange (src/bfam.c:6783-6877, 2418-2679).  Only the six
//             trace fields the flux uses are gathered (velocity and the stress
//             row of the face normal);
//   face    : upwind flux on the gathered traces (conforming faces and the
//             fine side of hanging faces): six jumps per face node, stored
//             in place of its trace;
//   mortar  : faces that go through the glue grid (2:1 hanging faces,
//             src/bfam.c:7328-7520).  The fine element interpolates the coarse
//             neighbour's trace to its mortar piece (interpolation[1..2]) and
//             evaluates the flux there; from the same Riemann solution it
//             forms the coarse side's jumps on the piece, L2-projects them to
//             the coarse face (projection[1..2]) and stores them in a mortar
//             buffer slot.  The coarse element, launched after its fine
//             neighbours (elements are launched by level), sums its pieces'
//             projected jumps;
//   volume  : one thread per node, the tensor-product LGL derivative along each
//             axis (the BFAM_KRON_IXIXA / IXAXI / AXIXI contractions of
//             src/bfam.c:3519-3624 at one node), plus the jumps of the faces
//             the node lies on, lifted with the lumped LGL mass;
//   update  : the 2N-storage LSRK stage dq = A dq + dt rhs, q' = q + B dq
//             (bfamo_lsrk_t, src/bfam.h:1840-1846) in FP64, writing the new
//             state to the other state buffer so that every element's
//             neighbours read the stage input unchanged.
//
// Template parameters: NT threads per CTA and MINB CTAs per SM targeted by the
// register allocation (the tile shape chosen per order), MODE (stage update or
// right-hand side only) and CT, the arithmetic of the right-hand side (double
// for the plain form; float for the precision form, where the volume
// derivative, flux, lift and mortar interpolation run in FP32 while the state,
// dq, the mortar L2 projection and the update stay FP64; the face jumps and
// lifts stay FP32 until one widening per field).
//
// State layout in HBM: field-major, element, node (bfam's per-field arrays
// stacked): q[f * K * Np + e * Np + n], n = i + Nq (j + Nq k).
#pragma once

#include "dg_common.cuh"
#include "dg_volume.cuh"

namespace bfam_b200
{

// index of the i-th set bit of m
__device__ __forceinline__ int nth_bit(int m, int i)
{
  for (; i > 0; --i)
    m &= m - 1;
  return __ffs(m) - 1;
}

// Node of thread t in the volume/update pass.  Nodes go in order (i
// fastest), except in 3D when a k-plane holds between 32 and 64 nodes (N = 5,
// 6): then warp w < Nq takes the first 32 nodes of plane w and the remaining
// warps the rest of every plane, so that the lines along y a warp reads lie
// in one plane (two planes per warp put lines of both at the same shared
// memory banks).  Threads past the last node get Np.
template <int DIM, int N, int NT>
__device__ __forceinline__ int node_of_thread(int t)
{
  constexpr int Nq = N + 1, P = Nq * Nq, Np = DIM == 3 ? P * Nq : P;
  if constexpr (DIM == 3 && P > 32 && P < 64 && NT >= Np)
  {
    if (t < 32 * Nq)
      return (t >> 5) * P + (t & 31);
    const int r = t - 32 * Nq;
    constexpr int REST = P - 32;
    return r < REST * Nq ? (r / REST) * P + 32 + r % REST : Np;
  }
  else
    return t < Np ? t : Np;
}

// A face node's flux jump in its trace slot (one double): stored at the
// precision of the right-hand side (a float in the slot's first four bytes
// in the precision form), so that it is never widened and narrowed again.
template <typename CT> __device__ __forceinline__ void put_jump(double *slot, CT v)
{
  *reinterpret_cast<CT *>(slot) = v;
}
template <typename CT> __device__ __forceinline__ CT get_jump(const double *slot)
{
  return *reinterpret_cast<const CT *>(slot);
}

// Shared-memory layout of one CTA (in doubles, every region 16-byte
// aligned).  NBUF element buffers (state, dq, face traces / flux jumps, face
// flux constants) let the loads of the next element fly
// while the current one is computed; the mortar scratch, the differentiation
// matrix, the mbarriers (q and dq per buffer) and the precision form's FP32 tile are
// single.
template <int DIM, int N, typename CT, int NBUF, bool DQS = true> struct Tile
{
  using S = Shape<DIM, N>;
  // DQS: the element's dq rows are staged in shared memory (TMA); otherwise
  // they are prefetched into L2 and read from global memory by the update
  static constexpr int BUF =
      S::SM_QS + (DQS ? S::SM_DQ : 0) + S::SM_PT + 4 * S::NF;
  static constexpr int OFF_MJ = NBUF * BUF;
  static constexpr int OFF_OPS = OFF_MJ + S::SM_MJ;
  static constexpr int OFF_BAR = OFF_OPS + S::SM_IP;
  static constexpr int OFF_QV = OFF_BAR + 2 * NBUF;
  static constexpr bool NARROW = sizeof(CT) < sizeof(double);
  static constexpr int TOTAL = OFF_QV + (NARROW ? S::SM_QF : 0);
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(double);
};

// the shape's register budget in resident CTAs per SM for arithmetic CT
template <int DIM, int N, typename CT> __host__ __device__ constexpr int shape_minb()
{
  return sizeof(CT) < sizeof(double) ? Shape<DIM, N>::MINB_NARROW
                                     : Shape<DIM, N>::MINB;
}

// CTAs per SM that the shape's register budget and NBUF buffers admit
// (228 KB of shared memory per SM, 1 KB reserved per CTA)
template <int DIM, int N, typename CT, int NBUF, bool DQS = true>
__host__ __device__ constexpr int resident_ctas()
{
  constexpr size_t bytes = Tile<DIM, N, CT, NBUF, DQS>::BYTES;
  constexpr int by_smem = bytes > 227 * 1024 ? 0 : (int)(233472 / (bytes + 1024));
  constexpr int m = shape_minb<DIM, N, CT>();
  return m < by_smem ? m : by_smem;
}

// dq staged in shared memory (TMA) unless the shape reads it from L2 in the
// update (Shape::DQ_L2 / DQ_L2_NARROW: 3D N=7, and the precision form at
// 3D N=5, where staging measured 9 % slower; the rows are prefetched into
// L2 when the element's loads are issued), or unless leaving it out admits
// more resident CTAs (the plain form at 3D N=5: five CTAs instead of four)
template <int DIM, int N, typename CT> __host__ __device__ constexpr bool stage_dqs()
{
  if (Shape<DIM, N>::DQ_L2 ||
      (Shape<DIM, N>::DQ_L2_NARROW && sizeof(CT) < sizeof(double)))
    return false;
  return resident_ctas<DIM, N, CT, 1, true>() >=
         resident_ctas<DIM, N, CT, 1, false>();
}

// Two buffers (a persistent grid; the loads of the next element overlap the
// current one) only where one buffer leaves fewer than four resident CTAs
// per SM and the second buffer costs none.  With four or more one-element
// CTAs per SM the block scheduler's balancing of the uneven element costs
// wins (3D N=3: 105.8 vs 91.5 G DOF-updates/s, N=4: 83.7 vs 72.0, 2D N=3:
// 54.0 vs 51.3; 3D N=2: 57.5 vs 61.0 in FP64 but 66.6 vs 59.2 in the
// precision form; 2D N=5: 61.8 vs 70.5), and a second buffer that costs
// resident CTAs loses (N=5: three CTAs of 7 warps with one buffer, two with
// two).
template <int DIM, int N, typename CT> __host__ __device__ constexpr int nbuf()
{
  constexpr bool DQS = stage_dqs<DIM, N, CT>();
  constexpr int one = resident_ctas<DIM, N, CT, 1, DQS>(),
                two = resident_ctas<DIM, N, CT, 2, DQS>();
  return one < 4 && two >= one && two > 0 ? 2 : 1;
}

// Elements per CTA: a CTA of EPC * NT threads holds EPC sub-elements of NT
// threads, each with its own shared-memory tile (Tile::TOTAL doubles, one
// after the other) and its own barrier -- the CTA's barrier when EPC = 1, the
// warp's when NT = 32, else named barrier 1 + sub -- so that sub-elements
// whose branches differ (fine or coarse faces) never wait for each other.
template <int NT, int EPC> struct Sub
{
  static_assert(EPC >= 1 && (EPC == 1 || NT == 32 || EPC <= 15),
                "named barriers 1..15");
  static_assert(NT % 32 == 0, "whole warps per sub-element");
  __device__ __forceinline__ static int t()
  {
    return EPC == 1 ? (int)threadIdx.x : (int)threadIdx.x % NT;
  }
  __device__ __forceinline__ static int id()
  {
    return EPC == 1 ? 0 : (int)threadIdx.x / NT;
  }
  __device__ __forceinline__ static void sync()
  {
    if constexpr (EPC == 1)
      __syncthreads();
    else if constexpr (NT == 32)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(1 + id()), "n"(NT) : "memory");
  }
};

// shared-memory tile of this thread's sub-element
template <typename T, int NT, int EPC>
__device__ __forceinline__ double *sub_smem()
{
  extern __shared__ __align__(16) double smem[];
  return EPC == 1 ? smem : smem + Sub<NT, EPC>::id() * T::TOTAL;
}

// Element buffer b of the tile.
template <int DIM, int N, typename CT, int NBUF, int NT = 32, int EPC = 1>
struct TileBuf
{
  double *qs, *R, *pt, *fcf;
  uint64_t *bq, *bdq;
  __device__ __forceinline__ explicit TileBuf(int b)
  {
    using S = Shape<DIM, N>;
    constexpr bool DQS = stage_dqs<DIM, N, CT>();
    using T = Tile<DIM, N, CT, NBUF, DQS>;
    double *smem = sub_smem<T, NT, EPC>();
    qs = smem + b * T::BUF;
    R = qs + S::SM_QS;
    pt = R + (DQS ? S::SM_DQ : 0);
    fcf = pt + S::SM_PT;
    bq = reinterpret_cast<uint64_t *>(smem + T::OFF_BAR) + 2 * b;
    bdq = bq + 1;
  }
};

// Issue every global read of element e into buffer b: q and (after the first
// stage) dq by TMA bulk copies completing on the buffer's mbarriers, the
// neighbours' face traces and the face flux constants by cp.async, as one
// commit group.
template <int DIM, int N, int NT, int MODE, typename CT, int NBUF,
          int EPC = 1>
__device__ __forceinline__ void issue_element(const DomainView &d,
                                              const StageParams &sp, int e,
                                              int b)
{
  using S = Shape<DIM, N>;
  constexpr int Np = S::Np, Nfp = S::Nfp, NF = S::NF, NFLD = S::NFLD,
                NTF = S::NTF;
  const TileBuf<DIM, N, CT, NBUF, NT, EPC> tb(b);
  double *qs = tb.qs, *R = tb.R, *pt = tb.pt, *fcf = tb.fcf;
  uint64_t *bar_q = tb.bq, *bar_dq = tb.bdq;
  const int t = Sub<NT, EPC>::t();
  const size_t fs = d.fs;
  const size_t eoff = (size_t)e * Np;
  const bool rd = MODE != MODE_RHS && !sp.first_stage;
  const int2 *desc = d.fdesc + (size_t)e * NF;
  if constexpr (S::TMA)
  {
    if (t == 0)
    {
      fence_proxy_async(); // shared memory of the previous element is free
      mbar_expect_tx(bar_q, NFLD * Np * sizeof(double) + NF * sizeof(double4));
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        bulk_g2s(qs + c * Np, d.qin + c * fs + eoff, Np * sizeof(double),
                 bar_q);
      // the face flux constants with the state, so that no thread needs
      // another thread's copies before the face phase
      bulk_g2s(fcf, d.fcE + (size_t)e * NF, NF * sizeof(double4), bar_q);
      if (rd)
      {
        if constexpr (stage_dqs<DIM, N, CT>())
        {
          mbar_expect_tx(bar_dq, NFLD * Np * sizeof(double));
#pragma unroll
          for (int c = 0; c < NFLD; ++c)
            bulk_g2s(R + c * Np, d.dq + c * fs + eoff, Np * sizeof(double),
                     bar_dq);
        }
        else
        {
#pragma unroll
          for (int c = 0; c < NFLD; ++c)
            bulk_prefetch_l2(d.dq + c * fs + eoff, Np * sizeof(double));
        }
      }
    }
  }
  else
  {
    for (int w = t; w < NFLD * Np; w += NT)
    {
      cp_async8(qs + w, d.qin + (w / Np) * fs + eoff + (w % Np));
      if (stage_dqs<DIM, N, CT>() && rd)
        cp_async8(R + w, d.dq + (w / Np) * fs + eoff + (w % Np));
    }
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
    if (k != 3) // a boundary face's ghost trace comes from the element itself
    {
      // the neighbour's opposite face, nodes in the same order (aligned
      // trees: the host refuses any other pairing or orientation)
      const int src_n = gmask<DIM, N>((ds.y >> 2) & 7, pn);
      const double *src = d.qin + (size_t)ds.x * Np + src_n;
#pragma unroll
      for (int c = 0; c < NTF; ++c)
      {
        const int g = f * NTF + c;
        cp_async8(pt + g * Nfp + fpos<DIM, N>(g, pn),
                  src + trace_field<DIM>(f >> 1, c) * fs);
      }
    }
    if (!S::TMA && pn == 0)
    {
      const double *fc =
          reinterpret_cast<const double *>(d.fcE + (size_t)e * NF + f);
      cp_async16(fcf + 4 * f, fc);
      cp_async16(fcf + 4 * f + 2, fc + 2);
    }
  }
  cp_async_commit(); // own state and constants (non-TMA path), face traces

}

// L2 prefetch of everything issue_element will read of element e itself
// (state rows, dq rows after the first stage, face descriptors, element
// data, flux constants); one thread, no completion to wait for.
template <int DIM, int N, int MODE>
__device__ __forceinline__ void prefetch_element(const DomainView &d,
                                                 const StageParams &sp, int e)
{
  using S = Shape<DIM, N>;
  if constexpr (S::TMA)
  {
    constexpr int Np = S::Np, NF = S::NF, NFLD = S::NFLD;
    const size_t eoff = (size_t)e * Np;
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
      bulk_prefetch_l2(d.qin + c * d.fs + eoff, Np * sizeof(double));
    if (MODE != MODE_RHS && !sp.first_stage)
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        bulk_prefetch_l2(d.dq + c * d.fs + eoff, Np * sizeof(double));
    }
    bulk_prefetch_l2(d.fdesc + (size_t)e * NF, NF * sizeof(int2));
    bulk_prefetch_l2(d.ed + e, sizeof(ElemData));
    bulk_prefetch_l2(d.fcE + (size_t)e * NF, NF * sizeof(double4));
    if constexpr (MODE != MODE_STAGE_NC)
    {
      // the mortar slots of its coarse faces (written by an earlier launch)
      constexpr int NJ = S::NJ, Nfp = S::Nfp, NPC = S::NPC;
#pragma unroll 1
      for (int f = 0; f < NF; ++f)
      {
        const int2 ds = d.fdesc[(size_t)e * NF + f];
        if ((ds.y & 3) == 2)
          bulk_prefetch_l2(d.mbuf + (size_t)ds.x * NJ * Nfp,
                           NPC * NJ * Nfp * sizeof(double));
      }
    }
  }
}

// Compute element e from buffer b (its loads issued by issue_element; `par`
// is the buffer's mbarrier phase parity).
template <int DIM, int N, int NT, int MODE, typename CT, int NBUF,
          int EPC = 1>
__device__ __forceinline__ void compute_element(const DomainView &d,
                                                const StageParams &sp,
                                                const DiffOp<N, CT> &dop,
                                                int e, int b, unsigned par)
{
  using S = Shape<DIM, N>;
  using T = Tile<DIM, N, CT, NBUF, stage_dqs<DIM, N, CT>()>;
  constexpr int Nq = S::Nq, Np = S::Np, Nfp = S::Nfp, NF = S::NF,
                NFLD = S::NFLD, NJ = S::NJ, NPC = S::NPC, ROWS = S::ROWS,
                NTF = S::NTF;
  // this sub-element's tile, derived from the dynamic shared array itself
  // (not a pointer parameter), so that all accesses stay in the shared
  // window with 32-bit addressing
  double *smem = sub_smem<T, NT, EPC>();
  const TileBuf<DIM, N, CT, NBUF, NT, EPC> tb(b);
  double *qs = tb.qs, *R = tb.R, *pt = tb.pt, *fcf = tb.fcf;
  uint64_t *bar_q = tb.bq, *bar_dq = tb.bdq;
  double *mj = smem + T::OFF_MJ; // [DIM][NJ][Nfp] coarse-side jumps, by fine rank
  const CT *sD = reinterpret_cast<const CT *>(smem + T::OFF_OPS); // D
  // the volume pass's copy of q: q itself in the plain form; in the
  // precision form FP32 q minus the element's first node per field (the
  // derivative of a constant is zero), so that rounding is relative to the
  // variation inside the element
  constexpr bool NARROW = T::NARROW;
  CT *qv;
  if constexpr (NARROW)
    qv = reinterpret_cast<CT *>(smem + T::OFF_QV);
  else
    qv = qs;

  const int t = Sub<NT, EPC>::t();
  const size_t fs = d.fs;
  const size_t eoff = (size_t)e * Np;
  // the update is dq = a dq + s rhs; the right-hand-side mode uses a = 0, s = 1
  const bool rd = MODE != MODE_RHS && !sp.first_stage;
  const double a = MODE != MODE_RHS ? sp.A : 0.0;
  const double s = MODE != MODE_RHS ? d.dt : 1.0;
  const ElemData me = d.ed[e];
  const int2 *desc = d.fdesc + (size_t)e * NF;

  int coarse_mask = 0, fine_mask = 0;
#pragma unroll
  for (int f = 0; f < NF; ++f)
  {
    const int y = desc[f].y;
    coarse_mask |= ((y & 3) == 2) << f;
    fine_mask |= ((y & 3) == 1 && ((y >> 8) & 7) != 0) << f;
  }
  const int ncoarse = __popc(coarse_mask), nfine = __popc(fine_mask);

  // ------------------------------------------------- phase 1: faces, mortars
  if constexpr (S::TMA)
  {
    if (!mbar_wait(bar_q, par))
      atomicExch(d.err, 1);
  }
  cp_async_wait<NBUF - 1>(); // this element's group (the next one may fly)
  if constexpr (NARROW && !S::TMA)
    Sub<NT, EPC>::sync(); // other threads' cp.async writes of q
  if constexpr (NARROW)
  {
    for (int n = t; n < Np; n += NT)
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        qv[c * Np + n] = CT(qs[c * Np + n] - qs[c * Np]);
    }
  }
  // With the state and flux constants by TMA, a thread's face pass reads
  // only its own gathered trace slots (its own cp.async group), so only the
  // fine-side interpolation, which reads whole lines, needs the barrier.
  if (!S::TMA || nfine)
    Sub<NT, EPC>::sync();
  // lift factor of face axis ax: s (2/h_ax) / w_0
  CT lfac[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    lfac[ax] =
        CT(s * (ax == 0 ? me.rx : (ax == 1 ? me.ry : me.rz)) * dop.iwend);

  // fine side: coarse partner trace -> my piece, in place (rows, then columns)
  if (nfine)
  {
    for (int pass = 0; pass < (DIM == 3 ? 2 : 1); ++pass)
    {
      for (int w = t; w < nfine * NTF * ROWS; w += NT)
      {
        const int f = nth_bit(fine_mask, w / (NTF * ROWS)),
                  r = w % (NTF * ROWS);
        const int hp = (desc[f].y >> 8) & 7;
        const int c = r / ROWS, line = r % ROWS;
        const int half = pass == 0 ? (hp - 1) & 1 : (hp - 1) >> 1;
        const int g = f * NTF + c;
        if (pass == 0)
          line_apply<DIM, N, true, false, CT, CT>(dop, half, pt + g * Nfp, g, line);
        else
          line_apply<DIM, N, false, false, CT, CT>(dop, half, pt + g * Nfp, g, line);
      }
      Sub<NT, EPC>::sync();
    }
  }

  // flux on conforming and fine-side faces: the face node's jumps (T* - T-,
  // v* - v-), written in place over the node's own trace slots (a thread
  // reads only its own node's slots: partners' face nodes are in the same
  // order on aligned trees) and lifted by the node pass.  On a fine face
  // the coarse side's jumps follow from the same Riemann solution (star
  // state v*, S* n shared by both sides, coarse normal -n):
  //   coarse (T* - T-) = -(fine J_T) + [T],  coarse (v* - v-) = fine J_v - [v]
  // with [.] = coarse - fine as seen from the fine side; they go to mj in the
  // coarse piece's node order.
  for (int w = t; w < NF * Nfp; w += NT)
  {
    {
      const int f = w / Nfp, pn = w % Nfp;
      const int y = desc[f].y;
      const int k = y & 3;
      if (k != 2)
      {
        const int vm = gmask<DIM, N>(f, pn);
        const int pp = pn;
        CT dq[NTF], J[6];
        // boundary faces: ghost state v+ = v-, S+ = -S- (free surface) or
        // q+ = 0 (absorbing)
        const bool free_surface = k == 3 && ((y >> 2) & 3) == 0;
#pragma unroll
        for (int c = 0; c < NTF; ++c)
        {
          const double qm = qs[trace_field<DIM>(f >> 1, c) * Np + vm];
          const int g = f * NTF + c;
          const double qp = k != 3 ? pt[g * Nfp + fpos<DIM, N>(g, pp)]
                                   : (free_surface ? (c < DIM ? qm : -qm) : 0.0);
          dq[c] = CT(qp - qm);
        }
        const CT sg = (f & 1) ? CT(1) : CT(-1);
        flux_jumps<DIM, CT>(dq, f >> 1, sg, CT(me.Zp), CT(me.Zs),
                            fcf + 4 * f, sp.flux, J);
        if ((fine_mask >> f) & 1)
        {
          // rank of f among the fine faces (an element has at most DIM)
          const int fr = __popc(fine_mask & ((1 << f) - 1));
#pragma unroll
          for (int c = 0; c < NJ; ++c)
          {
            const int sl = jslot<DIM>(c);
            const CT v = sl < 3 ? sg * dq[DIM + sl] - J[sl] : J[sl] - dq[sl - 3];
            const int g = fr * NJ + c;
            mj[g * Nfp + fpos<DIM, N>(g, pp)] = double(v);
          }
        }
#pragma unroll
        for (int c = 0; c < NJ; ++c)
        {
          const int g = f * NTF + c;
          put_jump<CT>(pt + g * Nfp + fpos<DIM, N>(g, pp), J[jslot<DIM>(c)]);
        }
      }
    }
  }

  // coarse side: the pieces' projected jumps, summed in glue order (stored
  // at the precision of the right-hand side, like the flux jumps)
  for (int w = t; MODE != MODE_STAGE_NC && w < ncoarse * Nfp; w += NT)
  {
    const int f = nth_bit(coarse_mask, w / Nfp), pn = w % Nfp;
    const double *mb = d.mbuf + (size_t)desc[f].x * NJ * Nfp + pn;
#pragma unroll
    for (int c = 0; c < NJ; ++c)
    {
      double sum = 0;
#pragma unroll
      for (int p = 0; p < NPC; ++p)
        sum += mb[(p * NJ + c) * Nfp];
      const int g = f * NTF + c;
      put_jump<CT>(pt + g * Nfp + fpos<DIM, N>(g, pn), CT(sum));
    }
  }

  // fine side: L2 projection of the coarse-side jumps to the coarse face
  // (FP64), then out to the mortar buffer for the coarse element
  if (nfine)
  {
    Sub<NT, EPC>::sync();
    for (int w = t; w < nfine * NJ * ROWS; w += NT)
    {
      const int fr = w / (NJ * ROWS), r = w % (NJ * ROWS);
      const int hp = (desc[nth_bit(fine_mask, fr)].y >> 8) & 7;
      const int g = fr * NJ + r / ROWS, line = r % ROWS;
      line_apply<DIM, N, true, true, double, CT>(
          dop, (hp - 1) & 1, mj + g * Nfp, g, line);
    }
    Sub<NT, EPC>::sync();
    if (DIM == 3)
    {
      for (int w = t; w < nfine * NJ * Nq; w += NT)
      {
        const int fr = w / (NJ * Nq), r = w % (NJ * Nq);
        const int hp = (desc[nth_bit(fine_mask, fr)].y >> 8) & 7;
        const int g = fr * NJ + r / Nq, col = r % Nq;
        line_apply<DIM, N, false, true, double, CT>(
            dop, (hp - 1) >> 1, mj + g * Nfp, g, col);
      }
      Sub<NT, EPC>::sync();
    }
    for (int w = t; w < nfine * NJ * Nfp; w += NT)
    {
      const int fr = w / (NJ * Nfp), r = w % (NJ * Nfp);
      const int f = nth_bit(fine_mask, fr), g = fr * NJ + r / Nfp;
      d.mbuf[(size_t)d.fslot[(size_t)e * NF + f] * NJ * Nfp + r] =
          mj[g * Nfp + fpos<DIM, N>(g, r % Nfp)];
    }
  }
  Sub<NT, EPC>::sync();

  // ------------------------ phase 2: volume, face contributions and update
  constexpr bool DQS = stage_dqs<DIM, N, CT>();
  if (MODE != MODE_RHS && rd && DQS)
  {
    if constexpr (S::TMA)
    {
      if (!mbar_wait(bar_dq, par))
        atomicExch(d.err, 2);
    }
  }
  constexpr int NODE_ITERS = (Np + NT - 1) / NT;
#pragma unroll 1
  for (int it = 0; it < NODE_ITERS; ++it)
  {
    const int n = node_of_thread<DIM, N, NT>(t + it * NT);
    if (n >= Np)
      break;
    const int i = n % Nq, j = (n / Nq) % Nq, k = n / (Nq * Nq);
    // s times the right-hand side in CT: the volume term, then the lifted
    // jumps of the faces this node lies on (at most one per axis, in face
    // order); widened to FP64 once for the update
    CT rv[NFLD];
    volume_node<DIM, N, CT>(qv, sD, dop, me, s, i, j, k, rv);
#pragma unroll
    for (int ax = 0; ax < DIM; ++ax)
    {
      const int idx = ax == 0 ? i : (ax == 1 ? j : k);
      if (idx != 0 && idx != N)
        continue;
      const int side = idx == N;
      const int pn = DIM == 3 ? (ax == 0 ? j + Nq * k
                                         : (ax == 1 ? i + Nq * k : i + Nq * j))
                              : (ax == 0 ? j : i);
      const int g0 = (2 * ax + side) * NTF;
      CT J[6] = {0, 0, 0, 0, 0, 0}, lc[NFLD];
#pragma unroll
      for (int c = 0; c < NJ; ++c)
        J[jslot<DIM>(c)] =
            get_jump<CT>(pt + (g0 + c) * Nfp + fpos<DIM, N>(g0 + c, pn));
      lift_face<DIM, CT>(J, ax, side ? CT(1) : CT(-1), lfac[ax], me, lc);
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        rv[c] += lc[c];
    }
    double acc[NFLD];
#pragma unroll
    for (int c = 0; c < NFLD; ++c)
      acc[c] = double(rv[c]);

    // point source on the velocity: s f(t_stage) F phi_n(x_s) / (rho w_n J)
    if (e == d.src.elem)
    {
      const double ts = d.clock->time + sp.C * d.dt;
      const double g = s * ricker(ts, d.src.f0, d.src.t0) * d.src.w[n] * me.irho;
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        acc[c] += g * d.src.force[c];
    }

    if constexpr (MODE != MODE_RHS)
    {
      if (rd)
      {
#pragma unroll
        for (int c = 0; c < NFLD; ++c)
          acc[c] += a * (DQS ? R[c * Np + n] : d.dq[c * fs + eoff + n]);
      }
      // streaming stores: the next stage reads these rows a whole stage
      // later (from DRAM), so they should not push the lines in reuse out
      // of L2 (+0.3-0.8 % at cfg1)
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
      {
        __stcs(d.dq + c * fs + eoff + n, acc[c]);
        __stcs(d.qout + c * fs + eoff + n, qs[c * Np + n] + sp.B * acc[c]);
      }
    }
    else
    {
#pragma unroll
      for (int c = 0; c < NFLD; ++c)
        d.rhs[c * fs + eoff + n] = acc[c];
    }
  }
}


// The launch's work items: item.view(idx) and item.elem(idx) give item idx's
// domain view and element.  With one buffer every CTA does one item (the
// grid covers them all); with two buffers the grid is persistent (items
// blockIdx.x, blockIdx.x + gridDim.x, ...) and the loads of the next item
// are issued before the current one is computed.
template <int DIM, int N, int NT, int MODE, typename CT, int NBUF,
          typename Item, int EPC = 1>
__device__ __forceinline__ void stage_loop(const Item &item, int n,
                                           const StageParams &sp,
                                           const DiffOp<N, CT> &dop)
{
  using T = Tile<DIM, N, CT, NBUF, stage_dqs<DIM, N, CT>()>;
  using SB = Sub<NT, EPC>;
  static_assert(EPC == 1 || NBUF == 1, "sub-elements use one buffer each");
  constexpr int Nq = N + 1;
  double *smem = sub_smem<T, NT, EPC>();
  const int lt = SB::t();
  if (lt == 0)
  {
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::OFF_BAR);
    for (int i = 0; i < 2 * NBUF; ++i)
      mbar_init(&bar[i], 1);
  }
  // the differentiation matrix into shared memory (rows indexed per
  // thread in the volume pass; the mortar operators are read from the
  // parameter bank at unrolled indices)
  {
    CT *sD = reinterpret_cast<CT *>(smem + T::OFF_OPS);
    for (int w = lt; w < Nq * Nq; w += NT)
      sD[w] = dop.D[w];
  }
  SB::sync();
  int idx = (int)blockIdx.x * EPC + SB::id();
  if (idx >= n)
    return;
  if constexpr (NBUF == 1)
  {
    // one element per sub-element (the grid covers every item)
    issue_element<DIM, N, NT, MODE, CT, 1, EPC>(item.view(idx), sp,
                                                item.elem(idx), 0);
    // a thread of another warp than the TMA issuer prefetches a later
    // item's element while this one's loads fly
    const int ia = idx + sp.ahead;
    if (sp.ahead > 0 && ia < n && lt == (NT > 32 ? 32 : 0))
      prefetch_element<DIM, N, MODE>(item.view(ia), sp, item.elem(ia));
    compute_element<DIM, N, NT, MODE, CT, 1, EPC>(item.view(idx), sp, dop,
                                                  item.elem(idx), 0, 0);
    return;
  }
  issue_element<DIM, N, NT, MODE, CT, NBUF>(item.view(idx), sp,
                                            item.elem(idx), 0);
#pragma unroll 1
  for (unsigned it = 0; idx < n; ++it)
  {
    const int b = (int)(it & 1u);
    const unsigned par = (it >> 1) & 1u;
    const int nidx = idx + (int)gridDim.x;
    if (nidx < n)
      issue_element<DIM, N, NT, MODE, CT, NBUF>(item.view(nidx), sp,
                                                item.elem(nidx), b ^ 1);
    else
      cp_async_commit(); // keep one group per iteration
    compute_element<DIM, N, NT, MODE, CT, NBUF>(item.view(idx), sp, dop,
                                                item.elem(idx), b, par);
    __syncthreads(); // buffer b is free
    idx = nidx;
  }
}

// one domain: item idx is element idx, or the idx-th of an element list
struct SingleItems
{
  const DomainView &d;
  __device__ __forceinline__ const DomainView &view(int) const { return d; }
  __device__ __forceinline__ int elem(int idx) const
  {
    return d.elist ? d.elist[idx] : idx;
  }
};

// many domains: item idx is work[idx] = (domain, element)
struct BatchItems
{
  const DomainView *__restrict__ views;
  const int2 *__restrict__ work;
  __device__ __forceinline__ const DomainView &view(int idx) const
  {
    return views[work[idx].x];
  }
  __device__ __forceinline__ int elem(int idx) const { return work[idx].y; }
};

// One domain: item idx is element idx, or the idx-th of the launch's
// element list (meshes with hanging faces launch their elements by level).
template <int DIM, int N, int NT, int MINB, int MODE, typename CT, int NBUF>
__global__ void __launch_bounds__(NT, MINB)
    dg_stage_kernel(DomainView d, int n, StageParams sp,
                    const __grid_constant__ DiffOp<N, CT> dop)
{
  stage_loop<DIM, N, NT, MODE, CT, NBUF>(SingleItems{d}, n, sp, dop);
}

// Many domains of the same order: item idx is work[idx] = (domain, element),
// each domain with its own arrays and time step.  EPC elements per CTA of
// EPC * NT threads (one buffer each).
template <int DIM, int N, int NT, int MINB, int MODE, typename CT, int NBUF,
          int EPC = 1>
__global__ void __launch_bounds__(NT *EPC, MINB)
    dg_stage_batch_kernel(const DomainView *__restrict__ views,
                          const int2 *__restrict__ work, int nwork,
                          StageParams sp,
                          const __grid_constant__ DiffOp<N, CT> dop)
{
  stage_loop<DIM, N, NT, MODE, CT, NBUF, BatchItems, EPC>(
      BatchItems{views, work}, nwork, sp, dop);
}

// dynamic shared memory of one CTA of the stage kernels (EPC sub-elements of
// one buffer each when EPC > 1)
template <int DIM, int N, typename CT, int EPC = 1>
__host__ __device__ constexpr size_t stage_smem_bytes()
{
  return EPC == 1
             ? Tile<DIM, N, CT, nbuf<DIM, N, CT>(), stage_dqs<DIM, N, CT>()>::BYTES
             : EPC * Tile<DIM, N, CT, 1, stage_dqs<DIM, N, CT>()>::BYTES;
}

// resident CTAs per SM the register budget is sized for: the shape's choice,
// capped by what the shared memory allows (228 KB per SM, 1 KB reserved per
// CTA)
template <int DIM, int N, typename CT>
__host__ __device__ constexpr int stage_min_ctas()
{
  constexpr int by_smem = (int)(233472 / (stage_smem_bytes<DIM, N, CT>() + 1024));
  constexpr int m = shape_minb<DIM, N, CT>() < by_smem ? shape_minb<DIM, N, CT>() : by_smem;
  return m < 1 ? 1 : m;
}

} // namespace bfam_b200
