// Volume term and face lift of the elastic DG operator, per node.  CT is the
// arithmetic type (double: plain form, float: precision form); the state in
// shared memory is always double.
#pragma once

#include <type_traits>

#include "dg_common.cuh"

namespace bfam_b200
{

// Derivative along x at one node: sum_m Dl[m] x[m] over a contiguous line of
// the tile, read with vector loads (2 doubles, or 4 or 2 floats) where Nq
// allows.  Every volume pass calls this (and line_d2) so that the sums run
// in the same order and round alike.
template <int N, typename CT>
__device__ __forceinline__ CT line_dx(const CT *x, const CT *Dl)
{
  constexpr int Nq = N + 1;
  CT acc = 0;
  constexpr bool F4 = sizeof(CT) == 4 && Nq % 4 == 0;
  if constexpr (F4)
  {
#pragma unroll
    for (int m = 0; m < Nq; m += 4)
    {
      const float4 v = *reinterpret_cast<const float4 *>(x + m);
      acc += Dl[m] * v.x;
      acc += Dl[m + 1] * v.y;
      acc += Dl[m + 2] * v.z;
      acc += Dl[m + 3] * v.w;
    }
  }
  else if constexpr (Nq % 2 == 0)
  {
    using V2 =
        typename std::conditional<sizeof(CT) == 4, float2, double2>::type;
#pragma unroll
    for (int m = 0; m < Nq; m += 2)
    {
      const V2 v = *reinterpret_cast<const V2 *>(x + m);
      acc += Dl[m] * v.x;
      acc += Dl[m + 1] * v.y;
    }
  }
  else
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      acc += Dl[m] * x[m];
  }
  return acc;
}

// Derivatives at two nodes of one strided line (along y or z): oa =
// sum_m Da[m] x[STRIDE m], ob = sum_m Db[m] x[STRIDE m] (each value loaded
// once).  With Db = Da only oa is formed.
template <int N, int STRIDE, bool TWO, typename CT>
__device__ __forceinline__ void line_d2(const CT *x, const CT *Da,
                                        const CT *Db, CT &oa, CT &ob)
{
  constexpr int Nq = N + 1;
  oa = 0;
  ob = 0;
#pragma unroll
  for (int m = 0; m < Nq; ++m)
  {
    const CT v = x[STRIDE * m];
    oa += Da[m] * v;
    if constexpr (TWO)
      ob += Db[m] * v;
  }
}

// s times the volume right-hand side at node (i, j, k):
//   rho dv/dt = div S,  dS/dt = lambda div(v) I + mu (grad v + grad v^T)
// with the derivative along each axis the 1-D LGL differentiation matrix
// applied along that axis -- the BFAM_KRON_IXIXA / IXAXI / AXIXI
// contractions of src/bfam.c:3519-3624 evaluated at one node.  qs is the
// element's state tile in CT, sD the column-major D(i,m) = sD[i + Nq m], both
// in shared memory.
template <int DIM, int N, typename CT>
__device__ __forceinline__ void volume_node(const CT *qs, const CT *sD,
                                            const ElemData &me, double s, int i,
                                            int j, int k, CT *rv)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np, NFLD = S::NFLD;
  const CT lam = CT(me.lam), mu = CT(me.mu), irho = CT(me.irho);
  const CT l2m = lam + CT(2) * mu;
#pragma unroll
  for (int c = 0; c < NFLD; ++c)
    rv[c] = CT(0);

  // derivative of field c along axis ax at this node
  auto deriv = [&](int c, int ax, const CT *Dl) {
    if (ax == 0)
      return line_dx<N, CT>(qs + c * Np + Nq * (j + Nq * k), Dl);
    CT acc, unused;
    if (ax == 1)
      line_d2<N, Nq, false, CT>(qs + c * Np + i + Nq * Nq * k, Dl, Dl, acc,
                                unused);
    else
      line_d2<N, Nq * Nq, false, CT>(qs + c * Np + i + Nq * j, Dl, Dl, acc,
                                     unused);
    return acc;
  };

  CT Dl[Nq];
  // x
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[i + Nq * m];
    const CT r = CT(s * me.rx);
    const CT dvx = r * deriv(0, 0, Dl), dvy = r * deriv(1, 0, Dl);
    if (DIM == 3)
    {
      const CT dvz = r * deriv(2, 0, Dl);
      rv[3] += l2m * dvx;
      rv[4] += lam * dvx;
      rv[5] += lam * dvx;
      rv[6] += mu * dvy;
      rv[7] += mu * dvz;
      rv[0] += irho * r * deriv(3, 0, Dl); // sxx
      rv[1] += irho * r * deriv(6, 0, Dl); // sxy
      rv[2] += irho * r * deriv(7, 0, Dl); // sxz
    }
    else
    {
      rv[2] += l2m * dvx;
      rv[3] += lam * dvx;
      rv[4] += mu * dvy;
      rv[0] += irho * r * deriv(2, 0, Dl); // sxx
      rv[1] += irho * r * deriv(4, 0, Dl); // sxy
    }
  }
  // y
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[j + Nq * m];
    const CT r = CT(s * me.ry);
    const CT dvx = r * deriv(0, 1, Dl), dvy = r * deriv(1, 1, Dl);
    if (DIM == 3)
    {
      const CT dvz = r * deriv(2, 1, Dl);
      rv[6] += mu * dvx;
      rv[3] += lam * dvy;
      rv[4] += l2m * dvy;
      rv[5] += lam * dvy;
      rv[8] += mu * dvz;
      rv[0] += irho * r * deriv(6, 1, Dl); // sxy
      rv[1] += irho * r * deriv(4, 1, Dl); // syy
      rv[2] += irho * r * deriv(8, 1, Dl); // syz
    }
    else
    {
      rv[4] += mu * dvx;
      rv[2] += lam * dvy;
      rv[3] += l2m * dvy;
      rv[0] += irho * r * deriv(4, 1, Dl); // sxy
      rv[1] += irho * r * deriv(3, 1, Dl); // syy
    }
  }
  // z
  if (DIM == 3)
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[k + Nq * m];
    const CT r = CT(s * me.rz);
    const CT dvx = r * deriv(0, 2, Dl), dvy = r * deriv(1, 2, Dl),
             dvz = r * deriv(2, 2, Dl);
    rv[7] += mu * dvx;
    rv[8] += mu * dvy;
    rv[3] += lam * dvz;
    rv[4] += lam * dvz;
    rv[5] += l2m * dvz;
    rv[0] += irho * r * deriv(7, 2, Dl); // sxz
    rv[1] += irho * r * deriv(8, 2, Dl); // syz
    rv[2] += irho * r * deriv(5, 2, Dl); // szz
  }
}

// Node-group volume passes (3D).  A thread owns QJ * QK nodes
//   g = a + QJ b:  (i, a ? N-j : j, b ? N-k : k),  a < QJ, b < QK,
// with 0 <= j < Nq/2 when QJ = 2 and 0 <= k < Nq/2 when QK = 2 (Nq even).
// A line along y through (i, ., k') then gives the derivatives at j and
// N-j, a line along z through (i, j', .) those at k and N-k, so a thread
// reads fewer lines than its nodes would one by one (QJ = 1, QK = 2: 5
// lines per differentiated field for 2 nodes instead of 6) and the row of
// D along an unpaired axis once.  Each output gets exactly volume_node's
// terms in volume_node's order (x, then y, then z) through the same
// line_dx / line_d2, so the passes give the same bits as volume_node.
// Three groups of three outputs (normal stress, shear stress, velocity)
// keep 3 QJ QK accumulators live at a time.

// the thread's node g's coordinates along y and z
template <int N, int QJ>
__device__ __forceinline__ void group_node(int g, int j, int k, int &jj,
                                           int &kk)
{
  jj = (g % QJ) ? N - j : j;
  kk = (g / QJ) ? N - k : k;
}

// The lines along y (AX = 1: one per k') or z (AX = 2: one per j') the
// thread reads, each giving the derivative at one node or, where the axis
// is paired, at the node pair g0(h), g1(h).
template <int N, int QJ, int QK, int AX> struct GroupAxis
{
  static constexpr int Nq = N + 1;
  static constexpr bool TWO = AX == 1 ? QJ == 2 : QK == 2;
  static constexpr int NLINE = AX == 1 ? QK : QJ;
  static constexpr int STR = AX == 1 ? Nq : Nq * Nq;
  static constexpr int NU = TWO ? 2 : 1;
  __device__ __forceinline__ static int off(int h, int i, int j, int k)
  {
    return AX == 1 ? i + Nq * Nq * (h ? N - k : k) : i + Nq * (h ? N - j : j);
  }
  __device__ __forceinline__ static int node(int h, int u)
  {
    return AX == 1 ? QJ * h + u : h + QJ * u;
  }
  // rows of D: Da at the thread's own coordinate, Db at its mirror
  template <typename CT>
  __device__ __forceinline__ static void rows(const CT *sD, int j, int k,
                                              CT *Da, CT *Db)
  {
    const int jk = AX == 1 ? j : k;
#pragma unroll
    for (int m = 0; m < Nq; ++m)
    {
      Da[m] = sD[jk + Nq * m];
      Db[m] = TWO ? sD[N - jk + Nq * m] : CT(0);
    }
  }
};

// normal-stress rates (fields 3..5: sxx syy szz) at the thread's nodes
template <int N, int QJ, int QK, typename CT>
__device__ __forceinline__ void group_normal(const CT *qs, const CT *sD,
                                             const ElemData &me, double s,
                                             int i, int j, int k,
                                             CT rs[QJ * QK][3])
{
  constexpr int Nq = N + 1, Np = Nq * Nq * Nq, G = QJ * QK;
  const CT lam = CT(me.lam), mu = CT(me.mu);
  const CT l2m = lam + CT(2) * mu;
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      rs[g][c] = CT(0);
  {
    CT Dl[Nq];
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[i + Nq * m];
    const CT r = CT(s * me.rx);
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      int jj, kk;
      group_node<N, QJ>(g, j, k, jj, kk);
      const CT dvx = r * line_dx<N, CT>(qs + Nq * (jj + Nq * kk), Dl);
      rs[g][0] += l2m * dvx;
      rs[g][1] += lam * dvx;
      rs[g][2] += lam * dvx;
    }
  }
  {
    using A = GroupAxis<N, QJ, QK, 1>;
    CT Da[Nq], Db[Nq];
    A::rows(sD, j, k, Da, Db);
    const CT r = CT(s * me.ry);
#pragma unroll
    for (int h = 0; h < A::NLINE; ++h)
    {
      CT d[2];
      line_d2<N, A::STR, A::TWO, CT>(qs + Np + A::off(h, i, j, k), Da, Db,
                                     d[0], d[1]);
#pragma unroll
      for (int u = 0; u < A::NU; ++u)
      {
        CT *o = rs[A::node(h, u)];
        const CT dvy = r * d[u];
        o[0] += lam * dvy;
        o[1] += l2m * dvy;
        o[2] += lam * dvy;
      }
    }
  }
  {
    using A = GroupAxis<N, QJ, QK, 2>;
    CT Da[Nq], Db[Nq];
    A::rows(sD, j, k, Da, Db);
    const CT r = CT(s * me.rz);
#pragma unroll
    for (int h = 0; h < A::NLINE; ++h)
    {
      CT d[2];
      line_d2<N, A::STR, A::TWO, CT>(qs + 2 * Np + A::off(h, i, j, k), Da,
                                     Db, d[0], d[1]);
#pragma unroll
      for (int u = 0; u < A::NU; ++u)
      {
        CT *o = rs[A::node(h, u)];
        const CT dvz = r * d[u];
        o[0] += lam * dvz;
        o[1] += lam * dvz;
        o[2] += l2m * dvz;
      }
    }
  }
}

// shear-stress rates (fields 6..8: sxy sxz syz) at the thread's nodes
template <int N, int QJ, int QK, typename CT>
__device__ __forceinline__ void group_shear(const CT *qs, const CT *sD,
                                            const ElemData &me, double s,
                                            int i, int j, int k,
                                            CT rs[QJ * QK][3])
{
  constexpr int Nq = N + 1, Np = Nq * Nq * Nq, G = QJ * QK;
  const CT mu = CT(me.mu);
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      rs[g][c] = CT(0);
  {
    CT Dl[Nq];
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[i + Nq * m];
    const CT r = CT(s * me.rx);
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      int jj, kk;
      group_node<N, QJ>(g, j, k, jj, kk);
      const CT *x = qs + Nq * (jj + Nq * kk);
      const CT dvy = r * line_dx<N, CT>(x + Np, Dl),
               dvz = r * line_dx<N, CT>(x + 2 * Np, Dl);
      rs[g][0] += mu * dvy;
      rs[g][1] += mu * dvz;
    }
  }
  {
    // along y: vx -> sxy, vz -> syz
    using A = GroupAxis<N, QJ, QK, 1>;
    CT Da[Nq], Db[Nq];
    A::rows(sD, j, k, Da, Db);
    const CT r = CT(s * me.ry);
#pragma unroll
    for (int h = 0; h < A::NLINE; ++h)
    {
      const CT *x = qs + A::off(h, i, j, k);
      CT dx[2], dz[2];
      line_d2<N, A::STR, A::TWO, CT>(x, Da, Db, dx[0], dx[1]);
      line_d2<N, A::STR, A::TWO, CT>(x + 2 * Np, Da, Db, dz[0], dz[1]);
#pragma unroll
      for (int u = 0; u < A::NU; ++u)
      {
        CT *o = rs[A::node(h, u)];
        const CT dvx = r * dx[u], dvz = r * dz[u];
        o[0] += mu * dvx;
        o[2] += mu * dvz;
      }
    }
  }
  {
    // along z: vx -> sxz, vy -> syz
    using A = GroupAxis<N, QJ, QK, 2>;
    CT Da[Nq], Db[Nq];
    A::rows(sD, j, k, Da, Db);
    const CT r = CT(s * me.rz);
#pragma unroll
    for (int h = 0; h < A::NLINE; ++h)
    {
      const CT *x = qs + A::off(h, i, j, k);
      CT dx[2], dy[2];
      line_d2<N, A::STR, A::TWO, CT>(x, Da, Db, dx[0], dx[1]);
      line_d2<N, A::STR, A::TWO, CT>(x + Np, Da, Db, dy[0], dy[1]);
#pragma unroll
      for (int u = 0; u < A::NU; ++u)
      {
        CT *o = rs[A::node(h, u)];
        const CT dvx = r * dx[u], dvy = r * dy[u];
        o[1] += mu * dvx;
        o[2] += mu * dvy;
      }
    }
  }
}

// velocity rates along y (AX = 1: sxy syy syz) or z (AX = 2: sxz syz szz)
template <int N, int QJ, int QK, int AX, typename CT>
__device__ __forceinline__ void group_velocity_axis(const CT *qs,
                                                    const CT *sD, CT irho,
                                                    CT r, int i, int j, int k,
                                                    CT rv[QJ * QK][3])
{
  constexpr int Nq = N + 1, Np = Nq * Nq * Nq;
  constexpr int F0 = AX == 1 ? 6 : 7, F1 = AX == 1 ? 4 : 8,
                F2 = AX == 1 ? 8 : 5;
  using A = GroupAxis<N, QJ, QK, AX>;
  CT Da[Nq], Db[Nq];
  A::rows(sD, j, k, Da, Db);
#pragma unroll
  for (int h = 0; h < A::NLINE; ++h)
  {
    const CT *x = qs + A::off(h, i, j, k);
    CT d0[2], d1[2], d2[2];
    line_d2<N, A::STR, A::TWO, CT>(x + F0 * Np, Da, Db, d0[0], d0[1]);
    line_d2<N, A::STR, A::TWO, CT>(x + F1 * Np, Da, Db, d1[0], d1[1]);
    line_d2<N, A::STR, A::TWO, CT>(x + F2 * Np, Da, Db, d2[0], d2[1]);
#pragma unroll
    for (int u = 0; u < A::NU; ++u)
    {
      CT *o = rv[A::node(h, u)];
      o[0] += irho * r * d0[u];
      o[1] += irho * r * d1[u];
      o[2] += irho * r * d2[u];
    }
  }
}

// velocity rates (fields 0..2) at the thread's nodes
template <int N, int QJ, int QK, typename CT>
__device__ __forceinline__ void group_velocity(const CT *qs, const CT *sD,
                                               const ElemData &me, double s,
                                               int i, int j, int k,
                                               CT rv[QJ * QK][3])
{
  constexpr int Nq = N + 1, Np = Nq * Nq * Nq, G = QJ * QK;
  const CT irho = CT(me.irho);
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      rv[g][c] = CT(0);
  {
    CT Dl[Nq];
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = sD[i + Nq * m];
    const CT r = CT(s * me.rx);
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      int jj, kk;
      group_node<N, QJ>(g, j, k, jj, kk);
      const CT *x = qs + Nq * (jj + Nq * kk);
      rv[g][0] += irho * r * line_dx<N, CT>(x + 3 * Np, Dl); // sxx
      rv[g][1] += irho * r * line_dx<N, CT>(x + 6 * Np, Dl); // sxy
      rv[g][2] += irho * r * line_dx<N, CT>(x + 7 * Np, Dl); // sxz
    }
  }
  group_velocity_axis<N, QJ, QK, 1, CT>(qs, sD, irho, CT(s * me.ry), i, j, k,
                                        rv);
  group_velocity_axis<N, QJ, QK, 2, CT>(qs, sD, irho, CT(s * me.rz), i, j, k,
                                        rv);
}

// Lifted face contribution of one face point: jump terms J = (T* - T-,
// v* - v-) times the lift factor L = s (2/h_ax) / w_0 of the lumped LGL mass,
// mapped onto the fields (outward normal n = sg e_ax):
//   v += L / rho (T* - T-),
//   S += L (lambda (dv.n) I + mu (dv n^T + n dv^T)).
template <int DIM, typename CT>
__device__ __forceinline__ void lift_face(const CT *J, int ax, CT sg, CT L,
                                          const ElemData &me, CT *out)
{
  const bool x = ax == 0, y = ax == 1, z = ax == 2;
  const CT dv0 = J[3], dv1 = J[4], dv2 = J[5];
  const CT dvn = sg * (x ? dv0 : (y ? dv1 : dv2));
  const CT Li = L * CT(me.irho), ll = L * CT(me.lam) * dvn,
           lm = L * CT(me.mu) * sg;
  const CT two = CT(2), zero = CT(0);
  if (DIM == 3)
  {
    out[0] = Li * J[0];
    out[1] = Li * J[1];
    out[2] = Li * J[2];
    out[3] = ll + (x ? two * lm * dv0 : zero);
    out[4] = ll + (y ? two * lm * dv1 : zero);
    out[5] = ll + (z ? two * lm * dv2 : zero);
    out[6] = lm * ((y ? dv0 : zero) + (x ? dv1 : zero));
    out[7] = lm * ((z ? dv0 : zero) + (x ? dv2 : zero));
    out[8] = lm * ((z ? dv1 : zero) + (y ? dv2 : zero));
  }
  else
  {
    out[0] = Li * J[0];
    out[1] = Li * J[1];
    out[2] = ll + (x ? two * lm * dv0 : zero);
    out[3] = ll + (y ? two * lm * dv1 : zero);
    out[4] = lm * ((y ? dv0 : zero) + (x ? dv1 : zero));
  }
}

} // namespace bfam_b200
