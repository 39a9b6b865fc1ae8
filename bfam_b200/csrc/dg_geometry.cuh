// Element boxes from p4est quadrant data, on the device.
#pragma once

#include "dg_common.cuh"

namespace bfam_b200
{

// Element e (one thread each): tree t = quads[5 e], level l = quads[5 e + 1],
// integer corner quads[5 e + 2 ..]; x0 = tree_x0 + tree_h * (x / root_len),
// h = tree_h * 2^-l (exact: a power-of-two scaling), and the element's
// metric 2 / h into its ElemData (axes beyond dim: h = 0, metric 2).
__global__ void __launch_bounds__(256)
    dg_geometry_kernel(int32_t K, int dim, const int32_t *__restrict__ quads,
                       const double *__restrict__ tree_x0,
                       const double *__restrict__ tree_h, double inv_root,
                       ElemData *__restrict__ ed, double *__restrict__ x0,
                       double *__restrict__ h)
{
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K)
    return;
  const int32_t *q = quads + 5 * (size_t)e;
  const int32_t t = q[0];
  const double scale = ldexp(1.0, -q[1]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    const bool on = a < dim;
    const double th = on ? tree_h[3 * (size_t)t + a] : 1.0;
    const double ha = th * scale;
    x0[3 * (size_t)e + a] =
        on ? tree_x0[3 * (size_t)t + a] + th * (q[2 + a] * inv_root) : 0.0;
    h[3 * (size_t)e + a] = on ? ha : 0.0;
    (&ed[e].rx)[a] = 2.0 / (on ? ha : 1.0);
  }
}

} // namespace bfam_b200
