// gauge_common.cuh -- device-side field access and lattice geometry shared by
// the kernel translation units.
//
// Memory layout in HBM: a color-matrix field with multiplicity m over V sites
// is stored structure-of-arrays, element (site, mu, k) of the 3x3 matrix at
// Cx<R>[(mu * 9 + k) * V + site], sites in the reference's order (x fastest,
// coordinate.h:182-188).  A warp touches 32 consecutive sites per component,
// so every load and store is a fully coalesced 512-byte (FP64) or 256-byte
// (FP32) transaction.  Neighbour links come through L1/L2; the lattice is
// periodic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "su3.cuh"

namespace qgb
{

// ------------------------------------------------------------------------
// field access

__device__ __forceinline__ Cx<double> ldg_cx(const Cx<double>* p)
{
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return cx<double>(v.x, v.y);
}
__device__ __forceinline__ Cx<float> ldg_cx(const Cx<float>* p)
{
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return cx<float>(v.x, v.y);
}

template <typename R>
struct CField {
  const Cx<R>* __restrict__ p;
  long V;
  __device__ __forceinline__ M3<R> ld(long site, int mu) const
  {
    M3<R> r;
    const Cx<R>* q = p + (long)mu * 9 * V + site;
#pragma unroll
    for (int k = 0; k < 9; ++k) r.e[k] = ldg_cx(q + (long)k * V);
    return r;
  }
};

template <typename R>
struct WField {
  Cx<R>* __restrict__ p;
  long V;
  __device__ __forceinline__ M3<R> ld(long site, int mu) const
  {
    M3<R> r;
    const Cx<R>* q = p + (long)mu * 9 * V + site;
#pragma unroll
    for (int k = 0; k < 9; ++k) r.e[k] = q[(long)k * V];
    return r;
  }
  __device__ __forceinline__ void st(long site, int mu, const M3<R>& r) const
  {
    Cx<R>* q = p + (long)mu * 9 * V + site;
#pragma unroll
    for (int k = 0; k < 9; ++k) q[(long)k * V] = r.e[k];
  }
};

__device__ __forceinline__ int wrap(int v, int L)
{
  if (v < 0) v += L;
  if (v < 0) v += L;
  if (v >= L) v -= L;
  if (v >= L) v -= L;
  return v;
}

struct Coord {
  int c[4];
};

__device__ __forceinline__ Coord coord_of(const Geo& g, long s)
{
  Coord x;
  x.c[0] = (int)(s % g.d[0]);
  s /= g.d[0];
  x.c[1] = (int)(s % g.d[1]);
  s /= g.d[1];
  x.c[2] = (int)(s % g.d[2]);
  x.c[3] = (int)(s / g.d[2]);
  return x;
}

// site index of x + a e_MU + b e_NU
template <int MU, int NU>
__device__ __forceinline__ long site_at(const Geo& g, const Coord& x, int a, int b)
{
  int y[4] = {x.c[0], x.c[1], x.c[2], x.c[3]};
  y[MU] = wrap(y[MU] + a, g.d[MU]);
  if (b != 0) y[NU] = wrap(y[NU] + b, g.d[NU]);
  return g.off + (long)y[0] + (long)g.d[0] * ((long)y[1] + (long)g.d[1] * ((long)y[2] + (long)g.d[2] * (long)y[3]));
}

// Same with run-time directions mu != nu (no local-memory arrays: each
// coordinate picks its offset with selects).
__device__ __forceinline__ long site_rt(const Geo& g, const Coord& x, int mu, int a, int nu, int b)
{
  long idx = 0;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    const int off = (k == mu ? a : 0) + (k == nu ? b : 0);
    const int y = wrap(x.c[k] + off, g.d[k]);
    idx = (k == 3) ? (long)y : idx * (long)g.d[k] + y;
  }
  return g.off + idx;
}

// Chain of global site sg: the largest i with offs[i] <= sg (offs ascending, offs[0] = 0).
__device__ __forceinline__ int chain_of(const long* __restrict__ offs, int n, long sg)
{
  int lo = 0, hi = n;  // invariant: offs[lo] <= sg < offs[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(offs + mid) <= sg) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ Geo chain_geo(const ChainInfo& c)
{
  Geo g;
  g.d[0] = c.d[0];
  g.d[1] = c.d[1];
  g.d[2] = c.d[2];
  g.d[3] = c.d[3];
  g.V = c.V;
  g.off = c.off;
  return g;
}

}  // namespace qgb
