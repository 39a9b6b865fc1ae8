// Host-side check of the shared-memory face-array layout of the stage
// kernel (fpos / line_pos in dg_common.cuh): every array's positions form a
// permutation of its Nfp slots, and at 3D N=7 the access patterns of the
// mortar line passes (a thread per row or column, a half-warp over the
// lines of two consecutive arrays) and of the face-node passes (a thread
// per face node, 16 consecutive nodes per half-warp) fall on 16 distinct
// 8-byte bank pairs per half-warp.  Prints one line per failed check and
// exits non-zero if any failed.
#include <cstdio>
#include <set>

#include "dg_common.cuh"

using namespace bfam_b200;

static int fails = 0;

static void expect(bool ok, const char *what, int N, int g, int a, int b)
{
  if (!ok)
  {
    ++fails;
    std::printf("FAIL %s N=%d g=%d %d %d\n", what, N, g, a, b);
  }
}

// bank pair of slot p of array g (8-byte words, 16 pairs of 4-byte banks)
template <int N> static int pair_of(int g, int p)
{
  constexpr int Nfp = (N + 1) * (N + 1);
  return (g * Nfp + p) % 16;
}

template <int N> static void permutation(int narrays)
{
  constexpr int Nfp = (N + 1) * (N + 1);
  for (int g = 0; g < narrays; ++g)
  {
    std::set<int> seen;
    for (int idx = 0; idx < Nfp; ++idx)
    {
      const int p = fpos<3, N>(g, idx);
      expect(p >= 0 && p < Nfp, "position out of range", N, g, idx, p);
      seen.insert(p);
    }
    expect((int)seen.size() == Nfp, "positions not a permutation", N, g,
           (int)seen.size(), Nfp);
  }
}

// lines of arrays g and g+1, value i of every line in one instruction
template <int N, bool ROWS> static void line_pass(int narrays, const char *what)
{
  constexpr int Nq = N + 1;
  for (int g = 0; g + 1 < narrays; ++g)
    for (int i = 0; i < Nq; ++i)
    {
      std::set<int> pairs;
      for (int a = 0; a < 2; ++a)
        for (int line = 0; line < Nq; ++line)
          pairs.insert(pair_of<N>(g + a, line_pos<3, N, ROWS>(g + a, line, i)));
      expect((int)pairs.size() == 16, what, N, g, i, (int)pairs.size());
    }
}

// 16 consecutive face nodes of array g in one half-warp
template <int N> static void node_pass(int narrays)
{
  constexpr int Nfp = (N + 1) * (N + 1);
  for (int g = 0; g < narrays; ++g)
    for (int h = 0; h < Nfp; h += 16)
    {
      std::set<int> pairs;
      for (int pn = h; pn < h + 16; ++pn)
        pairs.insert(pair_of<N>(g, fpos<3, N>(g, pn)));
      expect((int)pairs.size() == 16, "face-node pass conflicts", N, g, h,
             (int)pairs.size());
    }
}

int main()
{
  // 6 faces x 9 trace slots, and 3 fine ranks x 6 jump slots
  permutation<1>(54);
  permutation<3>(54);
  permutation<5>(54);
  permutation<7>(54);
  line_pass<7, true>(54, "row pass conflicts");
  line_pass<7, false>(54, "column pass conflicts");
  node_pass<7>(54);
  if (fails == 0)
    std::printf("face layout: all checks passed\n");
  return fails == 0 ? 0 : 1;
}
