// gauge_common.cuh -- device-side field access and lattice geometry shared by
// the kernel translation units.
//
// Memory layout in HBM: the sites of a field are cut into blocks of 32
// consecutive sites (the reference's order, x fastest, coordinate.h:182-188),
// and entry k of component m of site s (k < K: the 9 complex entries of a
// color matrix, K = 9; or one real, K = 1) is stored at
//     ((m * nblk + s / 32) * K + k) * 32 + s % 32,     nblk = ceil(V / 32).
// A warp touching 32 consecutive sites reads one fully coalesced 512-byte
// (FP64) or 256-byte (FP32) segment per matrix entry, as in a plain
// structure-of-arrays layout, but the 9 entries of one link are a fixed 32
// elements apart, so a link costs one address computation and 9 loads with
// immediate offsets instead of 9 address computations.  A real field is plain
// structure-of-arrays with the site count padded to a multiple of 32.  Padding
// sites are zero and no kernel writes them.  Neighbour links come through L1 /
// L2; the lattice is periodic.
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

// offset (in Cx<R> for K = 9, in reals for K = 1) of entry k of component m of site s
template <int K>
__host__ __device__ __forceinline__ long lay_index(long V, int m, int k, long s)
{
  return ((m * site_blocks(V) + (s >> 5)) * K + k) * 32 + (s & 31);
}

template <typename R>
struct CField {
  const Cx<R>* __restrict__ p;
  long V;
  __device__ __forceinline__ M3<R> ld(long site, int mu) const
  {
    M3<R> r;
    const Cx<R>* q = p + lay_index<9>(V, mu, 0, site);
#pragma unroll
    for (int k = 0; k < 9; ++k) r.e[k] = ldg_cx(q + 32 * k);
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
    const Cx<R>* q = p + lay_index<9>(V, mu, 0, site);
#pragma unroll
    for (int k = 0; k < 9; ++k) r.e[k] = q[32 * k];
    return r;
  }
  __device__ __forceinline__ void st(long site, int mu, const M3<R>& r) const
  {
    Cx<R>* q = p + lay_index<9>(V, mu, 0, site);
#pragma unroll
    for (int k = 0; k < 9; ++k) q[32 * k] = r.e[k];
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

// Link loads by 32-bit link and site indices (kernels that compute neighbour
// sites as the thread's own site plus per-direction offsets; valid while
// 36 * padded_sites(V) < 2^31):
// site(x + a mu + b nu) = site(x) + D_mu(a) + D_nu(b) for mu != nu, with
// D_k(a) = nb_delta(x_k, a, L_k, stride_k).
template <typename R>
struct LinkLd {
  const Cx<R>* __restrict__ p;
  int nblk;  // 32-site blocks of the field
  __device__ __forceinline__ M3<R> operator()(int link, int site) const
  {
    const Cx<R>* q = p + (((link * nblk + (site >> 5)) * 9) * 32 + (site & 31));
    M3<R> r;
#pragma unroll
    for (int k = 0; k < 9; ++k) r.e[k] = ldg_cx(q + 32 * k);
    return r;
  }
};

// Site of linear work index w (chunks of bs consecutive sites) in the
// traversal order of g: the owned box of a domain (box_site); linear when
// g.zs == 0; otherwise chunk c = w / bs
// is (xy chunk, z in slab, t, slab) from fastest to slowest, which needs
// X Y % bs == 0 and Z % g.zs == 0 (set_slab_order).
__host__ __device__ __forceinline__ long site_of_work(const Geo& g, long w, int bs)
{
  if (has_box(g)) return box_site(g, w);
  if (g.zs == 0) return w;
  const long xy = (long)g.d[0] * g.d[1];
  const long per_plane = xy / bs;
  long c = w / bs;
  const long lane = w - c * bs;
  const long cxy = c % per_plane;
  c /= per_plane;
  const long zz = c % g.zs;
  c /= g.zs;
  const long t = c % g.d[3];
  const long zb = c / g.d[3];
  return cxy * bs + lane + xy * ((zb * g.zs + zz) + (long)g.d[2] * t);
}

// z-slab order for site kernels with blocks of bs sites and links of
// link_bytes (144 FP64, 72 FP32): slabs of 16 z-planes when a time slice of
// the links exceeds 12 MB (then the +-2 slices a force reads no longer stay
// in L2 under a linear sweep) and the lattice allows it; linear otherwise.
__host__ __device__ __forceinline__ void set_slab_order(Geo& g, int bs, int link_bytes)
{
  const long xy = (long)g.d[0] * g.d[1];
  const long slice_bytes = xy * g.d[2] * 4 * link_bytes;
  g.zs = (g.off == 0 && g.r1 < 0 && !has_box(g) && xy % bs == 0 && g.d[2] % 16 == 0 && g.d[2] > 16 && slice_bytes > (12L << 20))
             ? 16
             : 0;
}

__device__ __forceinline__ int sel4(const int (&v)[4], int k)
{
  return k == 0 ? v[0] : k == 1 ? v[1] : k == 2 ? v[2] : v[3];
}

__device__ __forceinline__ int nb_delta(int xk, int a, int L, int stride) { return (wrap(xk + a, L) - xk) * stride; }

}  // namespace qgb
