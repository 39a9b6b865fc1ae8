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
// allows.
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

// Derivative along y or z at one node: sum_m Dl[m] x[STRIDE m] over a
// strided line of the tile.
template <int N, int STRIDE, typename CT>
__device__ __forceinline__ CT line_ds(const CT *x, const CT *Dl)
{
  constexpr int Nq = N + 1;
  CT acc = 0;
#pragma unroll
  for (int m = 0; m < Nq; ++m)
    acc += Dl[m] * x[STRIDE * m];
  return acc;
}

// Axes whose row of the differentiation matrix a node reads from the
// kernel's parameter space (constant cache) rather than from its shared
// memory copy (bit 0: x, 1: y, 2: z).  Shared 8-byte loads cost two L1
// wavefronts per warp however few distinct rows a warp reads, and the L1
// data pipe is the busiest unit of the stage kernel; constant-cache reads
// cost nothing there but serialise over the distinct rows of a warp.  A
// warp's nodes share k at N = 5 (but for the last warp) and N = 7, and span
// two k at N = 3.  Measured per shape (G DOF-updates/s against shared
// rows): z alone +0.6 % (FP64) and +1 % (FP32) at N = 7, where all three
// axes (eight distinct i) lost 3 and 9 %; all three axes +0.8 % at N = 3
// (four distinct rows) in both forms and +0.6 % at N = 5 in FP64, where
// FP32 lost 3.5 % with them and gains 0.4 % with z alone.  Other shapes
// keep the shared copy.
template <int DIM, int N, typename CT> constexpr int dparam_axes()
{
  if (DIM != 3)
    return 0;
  return N == 3 ? 7 : N == 5 ? (sizeof(CT) == 8 ? 7 : 4) : N == 7 ? 4 : 0;
}

// s times the volume right-hand side at node (i, j, k):
//   rho dv/dt = div S,  dS/dt = lambda div(v) I + mu (grad v + grad v^T)
// with the derivative along each axis the 1-D LGL differentiation matrix
// applied along that axis -- the BFAM_KRON_IXIXA / IXAXI / AXIXI
// contractions of src/bfam.c:3519-3624 evaluated at one node.  qs is the
// element's state tile in CT, sD the column-major D(i,m) = sD[i + Nq m], both
// in shared memory, dop the same operators in the kernel's parameter space.
template <int DIM, int N, typename CT>
__device__ __forceinline__ void volume_node(const CT *qs, const CT *sD,
                                            const DiffOp<N, CT> &dop,
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
    if (ax == 1)
      return line_ds<N, Nq, CT>(qs + c * Np + i + Nq * Nq * k, Dl);
    return line_ds<N, Nq * Nq, CT>(qs + c * Np + i + Nq * j, Dl);
  };

  constexpr int PA = dparam_axes<DIM, N, CT>();
  CT Dl[Nq];
  // x
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
      Dl[m] = (PA & 1) ? dop.D[i + Nq * m] : sD[i + Nq * m];
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
      Dl[m] = (PA & 2) ? dop.D[j + Nq * m] : sD[j + Nq * m];
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
      Dl[m] = (PA & 4) ? dop.D[k + Nq * m] : sD[k + Nq * m];
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
