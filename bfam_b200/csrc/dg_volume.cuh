// Volume term and face lift of the elastic DG operator, per node.  CT is the
// arithmetic type (double: plain form, float: precision form); the state in
// shared memory is always double.
#pragma once

#include <type_traits>

#include "dg_common.cuh"

namespace bfam_b200
{

// NQ consecutive CT values from / to shared memory, in 16-byte pieces where
// the alignment allows (every line and row of an element tile starts on a
// 16-byte boundary when NQ is even).
template <int NQ, typename CT>
__device__ __forceinline__ void ld_line(const CT *p, CT *v)
{
  if constexpr (sizeof(CT) == 8 && NQ % 2 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 2)
    {
      const double2 x = *reinterpret_cast<const double2 *>(p + m);
      v[m] = x.x;
      v[m + 1] = x.y;
    }
  }
  else if constexpr (sizeof(CT) == 4 && NQ % 4 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 4)
    {
      const float4 x = *reinterpret_cast<const float4 *>(p + m);
      v[m] = x.x;
      v[m + 1] = x.y;
      v[m + 2] = x.z;
      v[m + 3] = x.w;
    }
  }
  else if constexpr (sizeof(CT) == 4 && NQ % 2 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 2)
    {
      const float2 x = *reinterpret_cast<const float2 *>(p + m);
      v[m] = x.x;
      v[m + 1] = x.y;
    }
  }
  else
  {
#pragma unroll
    for (int m = 0; m < NQ; ++m)
      v[m] = p[m];
  }
}

template <int NQ, typename CT>
__device__ __forceinline__ void st_line(CT *p, const CT *v)
{
  if constexpr (sizeof(CT) == 8 && NQ % 2 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 2)
      *reinterpret_cast<double2 *>(p + m) = make_double2(v[m], v[m + 1]);
  }
  else if constexpr (sizeof(CT) == 4 && NQ % 4 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 4)
      *reinterpret_cast<float4 *>(p + m) =
          make_float4(v[m], v[m + 1], v[m + 2], v[m + 3]);
  }
  else if constexpr (sizeof(CT) == 4 && NQ % 2 == 0)
  {
#pragma unroll
    for (int m = 0; m < NQ; m += 2)
      *reinterpret_cast<float2 *>(p + m) = make_float2(v[m], v[m + 1]);
  }
  else
  {
#pragma unroll
    for (int m = 0; m < NQ; ++m)
      p[m] = v[m];
  }
}

// Volume right-hand side, s times
//   rho dv/dt = div S,  dS/dt = lambda div(v) I + mu (grad v + grad v^T),
// by lines: work item (g, l) takes x-line l of the element (nodes
// i + Nq l, i = 0..N; l = j + Nq k) and derivative group g, three
// derivatives of the tensor-product LGL operator, one along each axis
// (2D: two), each evaluated at all Nq nodes of the line -- the
// BFAM_KRON_IXIXA / IXAXI / AXIXI contractions of src/bfam.c:3519-3624
// restricted to the line:
//   along x: the line itself, D(i, m) from the parameter bank (constant
//            operands), so every value is read once;
//   along y: rows m of the line's k-plane, D(j, m) from shared memory;
//   along z: rows (j, m), D(k, m).
// The 18 derivatives of the 3D operator (2D: 8) split into 6 (2D: 4)
// groups of one per axis, so that every item does the same work:
//   3D  g0 (sxx,sxy,sxz) -> vx   g1 (sxy,syy,syz) -> vy  g2 (sxz,syz,szz) -> vz
//       g3 (vx,vy,vz) -> sxx syy szz   g4 (vy,vx,vy) -> sxy, half of syz
//       g5 (vz,vz,vx) -> sxz, the other half of syz
//   2D  g0 (sxx,sxy) -> vx  g1 (sxy,syy) -> vy  g2 (vx,vy) -> sxx syy
//       g3 (vy,vx) -> sxy
// The results go to the right-hand-side tile rhs[field][node] (CT), g4's
// half of syz to part[node] (3D), both in shared memory.  qv is the
// element's state tile in CT, sD the column-major D(i, m) = sD[i + Nq m].
template <int DIM, int N, typename CT>
__device__ __forceinline__ void volume_lines(const CT *qv, const CT *sD,
                                             const DiffOp<N, CT> &dop,
                                             const ElemData &me, double s,
                                             int g, int l, CT *rhs, CT *part)
{
  using S = Shape<DIM, N>;
  constexpr int Nq = S::Nq, Np = S::Np;
  const int j = l % Nq, k = DIM == 3 ? l / Nq : 0;
  int fx, fy, fz = 0;
  if constexpr (DIM == 3)
  {
    switch (g)
    {
    case 0: fx = 3; fy = 6; fz = 7; break;
    case 1: fx = 6; fy = 4; fz = 8; break;
    case 2: fx = 7; fy = 8; fz = 5; break;
    case 3: fx = 0; fy = 1; fz = 2; break;
    case 4: fx = 1; fy = 0; fz = 1; break;
    default: fx = 2; fy = 2; fz = 0; break;
    }
  }
  else
  {
    switch (g)
    {
    case 0: fx = 2; fy = 4; break;
    case 1: fx = 4; fy = 3; break;
    case 2: fx = 0; fy = 1; break;
    default: fx = 1; fy = 0; break;
    }
  }
  CT A[Nq], B[Nq], C[Nq];
  {
    CT x[Nq];
    ld_line<Nq, CT>(qv + fx * Np + Nq * l, x);
#pragma unroll
    for (int i = 0; i < Nq; ++i)
    {
      CT a = 0;
#pragma unroll
      for (int m = 0; m < Nq; ++m)
        a += dop.D[i + Nq * m] * x[m];
      A[i] = a;
    }
  }
#pragma unroll
  for (int i = 0; i < Nq; ++i)
    B[i] = C[i] = CT(0);
#pragma unroll
  for (int m = 0; m < Nq; ++m)
  {
    CT r[Nq];
    const CT dm = sD[j + Nq * m];
    ld_line<Nq, CT>(qv + fy * Np + Nq * m + Nq * Nq * k, r);
#pragma unroll
    for (int i = 0; i < Nq; ++i)
      B[i] += dm * r[i];
  }
  if constexpr (DIM == 3)
  {
#pragma unroll
    for (int m = 0; m < Nq; ++m)
    {
      CT r[Nq];
      const CT dm = sD[k + Nq * m];
      ld_line<Nq, CT>(qv + fz * Np + Nq * j + Nq * Nq * m, r);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        C[i] += dm * r[i];
    }
  }
  const CT sx = CT(s * me.rx), sy = CT(s * me.ry), sz = CT(s * me.rz);
#pragma unroll
  for (int i = 0; i < Nq; ++i)
  {
    A[i] *= sx;
    B[i] *= sy;
    C[i] *= sz;
  }
  const CT irho = CT(me.irho), lam = CT(me.lam), mu = CT(me.mu);
  const CT l2m = lam + CT(2) * mu;
  CT o[Nq];
  CT *line = rhs + Nq * l;
  if constexpr (DIM == 3)
  {
    if (g < 3)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = irho * (A[i] + B[i] + C[i]);
      st_line<Nq, CT>(line + g * Np, o);
    }
    else if (g == 3)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = l2m * A[i] + lam * (B[i] + C[i]);
      st_line<Nq, CT>(line + 3 * Np, o);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = l2m * B[i] + lam * (A[i] + C[i]);
      st_line<Nq, CT>(line + 4 * Np, o);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = l2m * C[i] + lam * (A[i] + B[i]);
      st_line<Nq, CT>(line + 5 * Np, o);
    }
    else if (g == 4)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = mu * (A[i] + B[i]);
      st_line<Nq, CT>(line + 6 * Np, o);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = mu * C[i];
      st_line<Nq, CT>(part + Nq * l, o);
    }
    else
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = mu * (A[i] + C[i]);
      st_line<Nq, CT>(line + 7 * Np, o);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = mu * B[i];
      st_line<Nq, CT>(line + 8 * Np, o);
    }
  }
  else
  {
    if (g < 2)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = irho * (A[i] + B[i]);
      st_line<Nq, CT>(line + g * Np, o);
    }
    else if (g == 2)
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = l2m * A[i] + lam * B[i];
      st_line<Nq, CT>(line + 2 * Np, o);
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = lam * A[i] + l2m * B[i];
      st_line<Nq, CT>(line + 3 * Np, o);
    }
    else
    {
#pragma unroll
      for (int i = 0; i < Nq; ++i)
        o[i] = mu * (A[i] + B[i]);
      st_line<Nq, CT>(line + 4 * Np, o);
    }
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
