// Shared definitions of the sm_100a kernels: device-side views of a domain,
// per-order shapes, PTX wrappers (TMA bulk copies, cp.async, mbarrier),
// bfam's face numbering, the elastic upwind flux and small 1-D operator
// passes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bfam_b200
{

struct ElemData
{
  double irho, lam, mu, Zp, Zs, rx, ry, rz; // rx = 2/hx, ...
};

// Face descriptor, one per (element, face), built on the host from vmapP and
// the glue grid.  b & 3 is the kind:
//   0 conforming:        a = neighbour element, b>>2 & 7 = its face (the
//                        opposite one: trees are aligned, orientation 0)
//   1 glue, whole face:  a = partner element (same size or coarse),
//                        b>>2 & 7 = partner face,
//                        b>>8 & 7 = partner's hanging piece (0: same size)
//   3 boundary:          a = the element, b>>2 & 3 = condition
//                        (0 free surface, 1 absorbing)
//   2 glue, coarse side: a = mortar buffer slot of the face's first piece
//                        (the pieces' slots are consecutive, in glue order;
//                        a face glued to another domain has its jumps in
//                        the first, written by the coupling kernel, and
//                        zeros in the others)
// A fine face (kind 1 with a hanging piece) writes its projected coarse-side
// jumps to mortar slot fslot[e][f].
// Per-domain clock in device memory, advanced once per time step by the
// post-step kernel, so that replayed CUDA graphs see the current time.
struct DomainClock
{
  double time; // time at the start of the current step
  int nsamp;   // receiver samples recorded
  int pad;
};

// Ricker point force of a domain (src_elem < 0: none).  Per node of the
// source element, src_w = phi_n(x_s) / (w_n J): the point force projected on
// the Lagrange basis through the lumped LGL mass.
struct PointSource
{
  int elem;
  const double *__restrict__ w; // [Np]
  double force[3];              // force vector (amplitude and direction)
  double f0, t0;                // peak frequency, time of the peak
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
  const int2 *__restrict__ fdesc; // [K][NF]
  // upwind flux constants {Zp+, 1/(Zp- + Zp+), Zs+, 1/(Zs- + Zs+)}:
  const double4 *__restrict__ fcE; // [K][NF] conforming / whole-face glue
  const int *__restrict__ fslot;   // [K][NF] mortar slot of a fine face
  double *mbuf; // [slots][NJ][Nfp] projected coarse-side jumps per piece
  const int *__restrict__ elist; // elements of this launch (NULL: all)
  const double *__restrict__ ops; // Dr | interp[3] | proj[3] | w
  int *err;
  double dt; // time step of this domain (batches step domains with their own)
  PointSource src;
  const DomainClock *clock;
};

struct StageParams
{
  double A, B, dt;
  double C;        // stage time t + C dt
  int first_stage; // A == 0: dq is not read
  int flux;        // 0 upwind, 1 central
  // one element per CTA: the CTA of work item i prefetches into L2 the
  // element of item i + ahead (half a wave of resident CTAs later), so that
  // its loads find L2 (0: no prefetch)
  int ahead;
};

// Ricker wavelet (1 - 2 a) exp(-a), a = (pi f0 (t - t0))^2
__host__ __device__ inline double ricker(double t, double f0, double t0)
{
  const double pi = 3.14159265358979323846;
  const double x = pi * f0 * (t - t0);
  const double a = x * x;
  return (1.0 - 2.0 * a) * exp(-a);
}

// The 1-D operators travel in the kernel's parameter space so that their
// entries, indexed by unrolled loop counters, are constant-bank operands of
// the FMAs.  All column-major, A(i,m) = A[i + (N+1) m].
// CT is the arithmetic type of the right-hand side (double: plain form,
// float: precision form); the L2 projection always stays in double.
template <int N, typename CT = double> struct DiffOp
{
  CT D[(N + 1) * (N + 1)];      // LGL differentiation
  CT Ib[(N + 1) * (N + 1)];     // interpolation to the bottom half
  double Pb[(N + 1) * (N + 1)]; // L2 projection from the bottom half
  double iwend;                 // 1 / w_0, the lumped-mass face weight
};
// The top-half operators are the reflections of the bottom-half ones,
// I_top(m,i) = I_bot(N-m, N-i) and P_top(i,m) = P_bot(N-i, N-m), because the
// LGL nodes are symmetric (r_{N-i} = -r_i); the host checks this on the glue
// grid's operators before using it.

// MODE_STAGE_NC: an LSRK stage over elements without coarse-side faces
// (the first launch level), compiled without the coarse-face pass
enum
{
  MODE_STAGE = 0,
  MODE_RHS = 1,
  MODE_STAGE_NC = 2
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
  // trace fields the flux needs on a face normal to axis a: the velocity
  // and row a of the stress (traction = sg * row a)
  static constexpr int NTF = 2 * DIM;
  static constexpr int ROWS = DIM == 3 ? Nq : 1; // rows of a face
  // one thread per node, or per face node where those are fewer (3D N=7:
  // 384 face nodes, 512 nodes in two passes, so that two CTAs fit an SM)
  static constexpr int work =
      (DIM == 3 && N == 7) ? NF * Nfp : (Np > NF * Nfp ? Np : NF * Nfp);
  static constexpr int NT = ((work + 31) / 32) * 32 > 1024
                                ? 1024
                                : ((work + 31) / 32) * 32;
  // CTAs per SM the register allocation is sized for (about 96 registers,
  // at most 16 CTAs of the smallest shapes), measured where it matters
  // (G DOF-updates/s, same box):
  //   3D N=5: five CTAs of 224 threads at 56 registers in the plain form,
  //     which then reads dq from L2 for room in shared memory (121.8-123.6
  //     vs 120.0-120.5 with four CTAs at 72 registers and dq staged); four
  //     in the precision form (126.3 vs 113.6 with five);
  //   3D N=3: ten CTAs of 96 threads at 64 registers in the plain form
  //     (109.1-109.4 vs 105.1-105.3 with seven; 105.6 with twelve), twelve
  //     in the precision form, which then reads dq from L2 (115.4 vs 104.3
  //     with seven, 109.2 with ten);
  //   3D N=7: two CTAs of 384 threads (three: 92.2 vs 102.3, spills).
  static constexpr int MINB_RAW = 65536 / (NT * 96);
  static constexpr int MINB =
      (DIM == 3 && N == 7)   ? 2
      : (DIM == 3 && N == 5) ? 5
      : (DIM == 3 && N == 3) ? 10
                             : (MINB_RAW < 1 ? 1 : (MINB_RAW > 16 ? 16 : MINB_RAW));
  static constexpr int MINB_NARROW = (DIM == 3 && N == 5)   ? 4
                                     : (DIM == 3 && N == 3) ? 12
                                                            : MINB;
  // dq read from global memory (L2) in the update instead of staged in
  // shared memory: at 3D N=7 (two CTAs of 103 KB with dq staged leave the
  // L1 cache about 22 KB for the neighbour-trace gathers; 105.6 vs 102.4 G
  // DOF-updates/s in the plain form), and in the precision form at N=5
  static constexpr bool DQ_L2 = DIM == 3 && N == 7;
  static constexpr bool DQ_L2_NARROW = DIM == 3 && N == 5;
  static constexpr bool TMA = (Np % 2) == 0; // 16-byte aligned element rows
  // shared memory regions in doubles (all even, so 16-byte aligned)
  static constexpr int SM_QS = NFLD * Np + (NFLD * Np) % 2; // q
  static constexpr int SM_DQ = SM_QS; // dq, then A dq + dt rhs in place
  // per face: the neighbour's NTF trace fields, then in place the NJ flux
  // jumps of each face node (NJ == NTF)
  static constexpr int SM_PT = NF * NTF * Nfp + (NF * NTF * Nfp) % 2;
  // coarse-side jumps of the fine faces, projected in place; an element has
  // at most DIM faces on the fine side of a hanging face (those on its
  // parent's boundary)
  static constexpr int SM_MJ = DIM * NJ * Nfp + (DIM * NJ * Nfp) % 2;
  // differentiation matrix (Nq*Nq entries, one double slot per entry): the
  // volume pass reads its rows per node, at thread-dependent rows
  static constexpr int SM_IP = Nq * Nq + (Nq % 2);
  // precision form only: FP32 copy of q minus the element's first node,
  // after the mbarriers
  static constexpr int SM_QF = (NFLD * Np + 3) / 4 * 2;
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

// bulk prefetch of a 16-byte aligned global range into L2 (no completion)
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src),
               "r"(bytes)
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

// Order this CTA's earlier generic-proxy shared-memory accesses (made visible
// by a preceding __syncthreads) before subsequent async-proxy (TMA) writes.
__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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

// ------------------------------------------------------------- physics

// Jump terms J = (T* - T-, v* - v-) at one face point from the trace jumps
// dq = q+ - q- of the point's trace slots (velocity, then row ax of the
// stress: see trace_field), formed in FP64 by the caller so that the
// precision form rounds the jump, not the traces.  n = e_axis * sg is the
// minus side's outward unit normal, so the traction jump is sg * [row ax].
// Upwind: exact Riemann solution of the normal (P, impedance Zp) and
// tangential (S, impedance Zs) problems; T - Z v travels out of the minus
// side, T + Z v out of the plus side:
//   v*_n - v-_n = (Zp+ [v_n] + [T_n]) / (Zp- + Zp+),  T*_n - T-_n = Zp- (..)
//   v*_t - v-_t = (Zs+ [v_t] + [T_t]) / (Zs- + Zs+),  T*_t - T-_t = Zs- (..)
// Central: half the jumps.  fc = {Zp+, 1/(Zp- + Zp+), Zs+, 1/(Zs- + Zs+)},
// computed once per face.
template <int DIM, typename CT>
__device__ __forceinline__ void flux_jumps(const CT *dq, int ax, CT sg,
                                           CT Zpm, CT Zsm, const double *fc,
                                           int flux, CT *J)
{
  const bool x = ax == 0, y = ax == 1;
  CT dv[3], dT[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    dv[a] = a < DIM ? dq[a] : CT(0);
    dT[a] = a < DIM ? sg * dq[DIM + a] : CT(0);
  }
  if (flux == 1)
  {
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      J[a] = CT(0.5) * dT[a];
      J[3 + a] = CT(0.5) * dv[a];
    }
    return;
  }
  const CT f0 = CT(fc[0]), f1 = CT(fc[1]), f2 = CT(fc[2]), f3 = CT(fc[3]);
  // normal parts
  const CT dvn = sg * (x ? dv[0] : (y ? dv[1] : dv[2]));
  const CT dTn = sg * (x ? dT[0] : (y ? dT[1] : dT[2]));
  const CT un = (f0 * dvn + dTn) * f1;
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    const CT na = a == ax ? sg : CT(0);
    const CT ut = (f2 * (dv[a] - dvn * na) + (dT[a] - dTn * na)) * f3;
    J[a] = Zpm * un * na + Zsm * ut;
    J[3 + a] = un * na + ut;
  }
}

// slot in the 6-component jump vector of stored component c
template <int DIM> __device__ __forceinline__ constexpr int jslot(int c)
{
  return c < DIM ? c : 3 + (c - DIM);
}

// out = A v with A the bottom-half mortar operator PROJ ? Pb : Ib of the
// parameter bank, or its top-half reflection when top != 0:
//   (A_top v)[m] = (A_bot reverse(v))[N - m].
// T is the arithmetic type: CT for interpolations, double for projections.
template <int N, bool PROJ, typename T, typename CT>
__device__ __forceinline__ void apply_half(const DiffOp<N, CT> &op, int top,
                                           const T *v, T *out)
{
  constexpr int Nq = N + 1;
  T vr[Nq], o[Nq];
#pragma unroll
  for (int i = 0; i < Nq; ++i)
    vr[i] = top ? v[N - i] : v[i];
#pragma unroll
  for (int m = 0; m < Nq; ++m)
  {
    T s = 0;
#pragma unroll
    for (int i = 0; i < Nq; ++i)
      s += (PROJ ? T(op.Pb[m + Nq * i]) : T(op.Ib[m + Nq * i])) * vr[i];
    o[m] = s;
  }
#pragma unroll
  for (int m = 0; m < Nq; ++m)
    out[m] = top ? o[N - m] : o[m];
}

// Position of face node idx = m0 + Nq m1 (m0 along face axis 0) in the
// g-th Nfp-array of a face region (trace slots and flux jumps: g = f NTF +
// slot; mortar jumps: g = fine rank NJ + slot).  In 3D at N = 7 the rows
// and columns are XOR-swizzled by g: a thread per row (or column) in the
// mortar line passes puts the lines of two consecutive arrays in a
// half-warp, whose 8-byte accesses then fall on 16 distinct bank pairs,
// where rows of 8 doubles would put them on 2 (rows) or 8 (columns); a
// thread per face node (16 consecutive nodes: two whole rows of one array)
// stays conflict-free.  The other orders keep the plain layout: at N = 5
// every row offset 6 m1 and array offset 36 g is even in bank pairs, which
// no permutation within a row fixes, and at N = 3 the analogous swizzle
// (rows and columns XOR g mod 4) removed the conflicts but ran 2-3 %
// slower.
template <int DIM, int N>
__host__ __device__ __forceinline__ int fpos(int g, int idx)
{
  if constexpr (DIM == 3 && N == 7)
  {
    const int m0 = idx & 7, m1 = idx >> 3, p = g & 1;
    return 8 * (m1 ^ p) + (m0 ^ ((m1 >> 1) | (p << 2)));
  }
  else
    return idx;
}

// Position of value i of line `line` of face array g: row m1 = line (ROWS)
// or column m0 = line
template <int DIM, int N, bool ROWS>
__host__ __device__ __forceinline__ int line_pos(int g, int line, int i)
{
  return fpos<DIM, N>(g, ROWS ? i + (N + 1) * line : line + (N + 1) * i);
}

// In-place 1-D mortar operator pass on one line of face array g (x: the
// array; ROWS: the row m1 = line, along face axis 0, else the column m0 =
// line, along axis 1), computed in T and stored back in double.  One thread
// owns one line.  An interpolation in a type narrower than double is applied
// to the line minus its first value, which is added back in double
// (interpolation reproduces constants), so that the rounding is relative to
// the variation along the line rather than to the values.
template <int DIM, int N, bool ROWS, bool PROJ, typename T, typename CT>
__device__ __forceinline__ void line_apply(const DiffOp<N, CT> &op, int top,
                                           double *x, int g, int line)
{
  constexpr int Nq = N + 1;
  constexpr bool OFFSET = !PROJ && sizeof(T) < sizeof(double);
  const double ref = OFFSET ? x[line_pos<DIM, N, ROWS>(g, line, 0)] : 0.0;
  T v[Nq];
#pragma unroll
  for (int i = 0; i < Nq; ++i)
  {
    const double xi = x[line_pos<DIM, N, ROWS>(g, line, i)];
    v[i] = OFFSET ? T(xi - ref) : T(xi);
  }
  apply_half<N, PROJ, T, CT>(op, top, v, v);
#pragma unroll
  for (int m = 0; m < Nq; ++m)
    x[line_pos<DIM, N, ROWS>(g, line, m)] = OFFSET ? ref + double(v[m]) : double(v[m]);
}

// Field of trace slot c on a face normal to axis ax: slots [0, DIM) are the
// velocity, slots [DIM, 2 DIM) row ax of the stress (bfam field order).
template <int DIM>
__device__ __forceinline__ int trace_field(int ax, int c)
{
  if (c < DIM)
    return c;
  const int k = c - DIM;
  if (DIM == 3)
  {
    if (ax == 0)
      return k == 0 ? 3 : (k == 1 ? 6 : 7); // sxx sxy sxz
    if (ax == 1)
      return k == 0 ? 6 : (k == 1 ? 4 : 8); // sxy syy syz
    return k == 0 ? 7 : (k == 1 ? 8 : 5);   // sxz syz szz
  }
  if (ax == 0)
    return k == 0 ? 2 : 4; // sxx sxy
  return k == 0 ? 4 : 3;   // sxy syy
}

// 16-byte asynchronous copy global -> shared (both 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)),
               "l"(src)
               : "memory");
}


} // namespace bfam_b200
