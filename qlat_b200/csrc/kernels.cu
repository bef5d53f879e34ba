// kernels.cu -- CUDA kernels of the pure-gauge hot path for sm_100a.
//
// Memory layout in HBM (gauge_common.cuh): sites in the reference's order (x
// fastest, coordinate.h:182-188) cut into blocks of 32; entry k of the 3x3
// matrix of component mu at site s is Cx<R>[((mu * nblk + s / 32) * 9 + k) *
// 32 + s % 32].  A warp touching 32 consecutive sites reads one fully coalesced
// 512-byte (FP64) or 256-byte (FP32) segment per matrix entry.  Neighbour
// links come through L1/L2; the lattice is periodic.
//
// Kernels use one thread per link (site, mu) for link-local work and force
// evaluation, and one thread per site for the site reductions.  Reductions
// accumulate in FP64 whatever the storage precision, then reduce in a fixed
// order (warp shuffles, block, then one block over the partials), so results
// are deterministic run to run.
#include <cuda_runtime.h>
#include <type_traits>
#include <stdint.h>
#include <string.h>

#include "gauge_common.cuh"
#include "kernels.h"
#include "rng.cuh"
#include "su3.cuh"

namespace qgb
{

ShaConst qgb_sha_host;

// ------------------------------------------------------------------------
// constants

static void sha_const_compute(ShaConst& c)
{
  int primes[64];
  int n = 0;
  for (int v = 2; n < 64; ++v) {
    bool p = true;
    for (int d = 2; d * d <= v; ++d)
      if (v % d == 0) {
        p = false;
        break;
      }
    if (p) primes[n++] = v;
  }
  // first 32 fractional bits of cube roots (k) and square roots (h0) of primes
  for (int i = 0; i < 64; ++i) {
    const unsigned __int128 target = ((unsigned __int128)primes[i]) << 96;
    uint64_t lo = 0, hi = (uint64_t)1 << 36;
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) / 2;
      if ((unsigned __int128)mid * mid * mid <= target) lo = mid; else hi = mid;
    }
    c.k[i] = (uint32_t)lo;
  }
  for (int i = 0; i < 8; ++i) {
    const unsigned __int128 target = ((unsigned __int128)primes[i]) << 64;
    uint64_t lo = 0, hi = (uint64_t)1 << 36;
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) / 2;
      if ((unsigned __int128)mid * mid <= target) lo = mid; else hi = mid;
    }
    c.h0[i] = (uint32_t)lo;
  }
}

struct HostConstInit {
  HostConstInit() { sha_const_compute(qgb_sha_host); }
};
static HostConstInit host_const_init;

void init_constants()
{
  cudaMemcpyToSymbol(qgb_sha_dev, &qgb_sha_host, sizeof(ShaConst));
  cudaMemcpyToSymbol(qgb_logtab_dev, qgb_logtab_host, sizeof(qgb_logtab_host));
}

// ------------------------------------------------------------------------
// gf_evolve: U = unitarize(exp(eps P) U) (hmc.cpp:311-328, matrix-hmc.h:179-188)

template <typename R>
__global__ void __launch_bounds__(256) k_evolve(Geo g, Cx<R>* U, const Cx<R>* P, double eps, int unit, int taylor)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int mu = blockIdx.y;
  const WField<R> Uf{U, g.V};
  const CField<R> Pf{P, g.V};
  const M3<R> a = scale(R(eps), Pf.ld(s, mu));
  const M3<R> e = taylor ? exp_taylor(a, 20) : exp_ch(a);
  M3<R> un = mul(e, Uf.ld(s, mu));
  if (unit) unitarize(un);
  Uf.st(s, mu, un);
}

template <typename R>
cudaError_t launch_evolve(const Geo& g, void* U, const void* P, double eps, int unitarize, int taylor,
                          cudaStream_t st)
{
  const int bs = 256;
  dim3 grid((unsigned)((g.V + bs - 1) / bs), 4);
  k_evolve<R><<<grid, bs, 0, st>>>(g, (Cx<R>*)U, (const Cx<R>*)P, eps, unitarize, taylor);
  return cudaGetLastError();
}

template <typename R, typename C>
__global__ void k_unitarize(long V, int m, Cx<R>* U)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const WField<R> Uf{U, V};
  for (int mu = 0; mu < m; ++mu) {
    M3<R> u = Uf.ld(s, mu);
    unitarize_as<C, R>(u);
    Uf.st(s, mu, u);
  }
}

template <typename R, typename C>
cudaError_t launch_unitarize(const Geo& g, int m, void* U, cudaStream_t st)
{
  const int bs = 256;
  k_unitarize<R, C><<<(unsigned)((g.V + bs - 1) / bs), bs, 0, st>>>(g.V, m, (Cx<R>*)U);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// deterministic reductions

static const int RED_BS = 256;

int reduce_blocks(const Geo& g) { return (int)((g.V + RED_BS - 1) / RED_BS); }

// Reduce NV values across the block in a fixed order; thread 0 writes
// partials[k * gridDim.x + blockIdx.x].
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* partials)
{
  __shared__ double sm[NV][RED_BS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sm[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int i = 0; i < RED_BS / 32; ++i) t += sm[k][i];
      partials[(long)k * gridDim.x + blockIdx.x] = t;
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(RED_BS) k_gm_hamilton(Geo g, const Cx<R>* P, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (s < g.V && in_reduce(g, s)) {
    const CField<R> Pf{P, g.V};
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) v[0] += neg_half_tr_square(Pf.ld(s, mu));
  }
  block_reduce_store<1>(v, partials);
}

template <typename R>
cudaError_t launch_gm_hamilton(const Geo& g, const void* P, double* partials, cudaStream_t st)
{
  k_gm_hamilton<R><<<reduce_blocks(g), RED_BS, 0, st>>>(g, (const Cx<R>*)P, partials);
  return cudaGetLastError();
}

// Threads cover the padded sites too (reduce_blocks(g) blocks of RED_BS span
// padded_sites(V), RED_BS being a multiple of 32), so Q's padding is written
// (with the zeros of P's).  The sum uses the FP64 one of the two matrices, so
// it equals k_gm_hamilton<double> on the FP64 field bit for bit.
template <typename RI, typename RO>
__global__ void __launch_bounds__(RED_BS) k_gm_hamilton_convert(Geo g, const Cx<RI>* P, Cx<RO>* Q, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (s < padded_sites(g.V)) {
    const CField<RI> Pf{P, g.V};
    const WField<RO> Qf{Q, g.V};
    const bool sum = s < g.V && in_reduce(g, s);
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
      const M3<RI> p = Pf.ld(s, mu);
      M3<RO> q;
      M3<double> d;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        q.e[k] = cx<RO>((RO)p.e[k].re, (RO)p.e[k].im);
        d.e[k] = sizeof(RI) == 8 ? cx<double>((double)p.e[k].re, (double)p.e[k].im)
                                 : cx<double>((double)q.e[k].re, (double)q.e[k].im);
      }
      Qf.st(s, mu, q);
      if (sum) v[0] += neg_half_tr_square(d);
    }
  }
  block_reduce_store<1>(v, partials);
}

template <typename RI, typename RO>
cudaError_t launch_gm_hamilton_convert(const Geo& g, const void* P, void* Q, double* partials, cudaStream_t st)
{
  k_gm_hamilton_convert<RI, RO><<<reduce_blocks(g), RED_BS, 0, st>>>(g, (const Cx<RI>*)P, (Cx<RO>*)Q, partials);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_unitarize_to_f64(long V, const Cx<float>* P, Cx<double>* Q)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= padded_sites(V)) return;
  const CField<float> Pf{P, V};
  const WField<double> Qf{Q, V};
#pragma unroll 1
  for (int mu = 0; mu < 4; ++mu) {
    const M3<float> p = Pf.ld(s, mu);
    M3<double> u;
#pragma unroll
    for (int k = 0; k < 9; ++k) u.e[k] = cx<double>((double)p.e[k].re, (double)p.e[k].im);
    if (s < V) unitarize_as<double, double>(u);
    Qf.st(s, mu, u);
  }
}

cudaError_t launch_unitarize_to_f64(const Geo& g, const void* P, void* Q, cudaStream_t st)
{
  const int bs = 256;
  k_unitarize_to_f64<<<(unsigned)((padded_sites(g.V) + bs - 1) / bs), bs, 0, st>>>(g.V, (const Cx<float>*)P,
                                                                                  (Cx<double>*)Q);
  return cudaGetLastError();
}

// Sums over the 6 planes mu < nu at x of (Re tr plaq - 3) and, with RECT, of
// (Re tr rect - 3) for both rectangle orientations (hmc.cpp:9-25,203-252):
// plaq = A B^+ with A = U_mu(x) U_nu(x+mu), B = U_nu(x) U_mu(x+nu);
// rect (mu, mu, nu, -mu, -mu, -nu) = A B^+ with A = U_mu(x) U_mu(x+mu) U_nu(x+2mu),
// B = U_nu(x) U_mu(x+nu) U_mu(x+mu+nu).
template <typename R, bool RECT>
__global__ void __launch_bounds__(RED_BS) k_action(Geo g, const Cx<R>* Up, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (s < g.V && in_reduce(g, s)) {
    const CField<R> U{Up, g.V};
    const Coord x = coord_of(g, s);
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2);
      const int nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
      {
        const M3<R> A = mul(U.ld(s, mu), U.ld(site_rt(g, x, mu, 1, nu, 0), nu));
        const M3<R> B = mul(U.ld(s, nu), U.ld(site_rt(g, x, mu, 0, nu, 1), mu));
        v[0] += (double)re_tr_mul_adj(A, B) - 3.0;
      }
      if (RECT) {
#pragma unroll 1
        for (int o = 0; o < 2; ++o) {
          const int a = o == 0 ? mu : nu, b = o == 0 ? nu : mu;  // long side along a
          M3<R> A = mul(U.ld(s, a), U.ld(site_rt(g, x, a, 1, b, 0), a));
          A = mul(A, U.ld(site_rt(g, x, a, 2, b, 0), b));
          M3<R> B = mul(U.ld(s, b), U.ld(site_rt(g, x, a, 0, b, 1), a));
          B = mul(B, U.ld(site_rt(g, x, a, 1, b, 1), a));
          v[1] += (double)re_tr_mul_adj(A, B) - 3.0;
        }
      }
    }
  }
  block_reduce_store<2>(v, partials);
}

// The same sums with each loop walked as one running product (two 3x3
// matrices live instead of four; at most 128 registers, two blocks per SM),
// neighbours as the site plus per-direction offsets (LinkLd):
// plaq = Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+),
// rect = Re tr(U_a(x) U_a(x+a) U_b(x+2a) U_a(x+a+b)^+ U_a(x+b)^+ U_b(x)^+)
// over the 12 ordered pairs (a, b), i.e. both orientations of every plane.
// In FP32 the double link U_a(x) U_a(x+a) is formed once for the three
// rectangles whose long side runs along a (52 instead of 60 products per
// site); in FP64 the extra live matrix costs more than the products it saves
// (24^3 x 64 on B200: FP64 0.56 ms with the double link recomputed against
// 0.59 ms shared, FP32 0.31 ms shared against 0.34 ms; 0.79 / 0.53 ms for
// k_action).
// With copy != nullptr each thread also writes its site's links, converted to
// FP32, into copy (padded sites included, with zeros).
template <typename R, bool RECT>
__global__ void __launch_bounds__(RED_BS, 2) k_action_loops(Geo g, const Cx<R>* Up, double* partials,
                                                            Cx<float>* copy)
{
  constexpr bool SHARE = sizeof(R) == 4;
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (copy != nullptr && s < padded_sites(g.V)) {
    const CField<R> Uf{Up, g.V};
    const WField<float> Cf{copy, g.V};
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
      const M3<R> u = Uf.ld(s, mu);
      M3<float> c;
#pragma unroll
      for (int k = 0; k < 9; ++k) c.e[k] = cx<float>((float)u.e[k].re, (float)u.e[k].im);
      Cf.st(s, mu, c);
    }
  }
  double v[2] = {0.0, 0.0};
  if (s < g.V && in_reduce(g, s)) {
    const LinkLd<R> L{Up, (int)site_blocks(g.V)};
    const Coord x = coord_of(g, s);
    const int si = (int)s;
    const int st[4] = {1, g.d[0], g.d[0] * g.d[1], g.d[0] * g.d[1] * g.d[2]};
    int d1[4], d2[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      d1[k] = nb_delta(x.c[k], 1, g.d[k], st[k]);
      d2[k] = nb_delta(x.c[k], 2, g.d[k], st[k]);
    }
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2);
      const int nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
      M3<R> M = mul(L(mu, si), L(nu, si + sel4(d1, mu)));
      M = mul_adj(M, L(mu, si + sel4(d1, nu)));
      v[0] += (double)re_tr_mul_adj(M, L(nu, si)) - 3.0;
    }
    if (RECT) {
#pragma unroll 1
      for (int a = 0; a < 4; ++a) {
        const int a1 = sel4(d1, a), a2 = sel4(d2, a);
        M3<R> D;
        if constexpr (SHARE) D = mul(L(a, si), L(a, si + a1));
#pragma unroll 1
        for (int i = 1; i < 4; ++i) {
          const int b = (a + i) & 3;
          const int b1 = sel4(d1, b);
          M3<R> M;
          if constexpr (SHARE) {
            M = mul(D, L(b, si + a2));
          } else {
            M = mul(L(a, si), L(a, si + a1));
            M = mul(M, L(b, si + a2));
          }
          M = mul_adj(M, L(a, si + a1 + b1));
          M = mul_adj(M, L(a, si + b1));
          v[1] += (double)re_tr_mul_adj(M, L(b, si)) - 3.0;
        }
      }
    }
  }
  block_reduce_store<2>(v, partials);
}

// The same sums with the two corners of each plane (a, b) shared by its
// plaquette and its two rectangles (FP64; one thread per site, up to 255
// registers):
//   Pa = U_a(x) U_b(x+a), Pb = U_b(x) U_a(x+b):   plaq = Re tr(Pa Pb^+)
//   rect, long side a = Re tr([U_a(x) U_a(x+a) U_b(x+2a)] [Pb U_a(x+a+b)]^+)
//   rect, long side b = Re tr([U_b(x) U_b(x+b) U_a(x+2b)] [Pa U_b(x+a+b)]^+)
// 8 products, 3 traces and 10 link loads per plane instead of 10, 3 and 16:
// the loops of hmc.cpp:203-252, grouped differently.  The plaquette-only sum
// (gf_avg_plaq, Wilson actions) fits 128 registers and runs two blocks per SM.
template <typename R, bool RECT>
__global__ void __launch_bounds__(RED_BS, RECT ? 1 : 2) k_action_corners(Geo g, const Cx<R>* Up, double* partials,
                                                              Cx<float>* copy)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (copy != nullptr && s < padded_sites(g.V)) {
    const CField<R> Uf{Up, g.V};
    const WField<float> Cf{copy, g.V};
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
      const M3<R> u = Uf.ld(s, mu);
      M3<float> c;
#pragma unroll
      for (int k = 0; k < 9; ++k) c.e[k] = cx<float>((float)u.e[k].re, (float)u.e[k].im);
      Cf.st(s, mu, c);
    }
  }
  double v[2] = {0.0, 0.0};
  if (s < g.V && in_reduce(g, s)) {
    const LinkLd<R> L{Up, (int)site_blocks(g.V)};
    const Coord x = coord_of(g, s);
    const int si = (int)s;
    const int st[4] = {1, g.d[0], g.d[0] * g.d[1], g.d[0] * g.d[1] * g.d[2]};
    int d1[4], d2[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      d1[k] = nb_delta(x.c[k], 1, g.d[k], st[k]);
      d2[k] = nb_delta(x.c[k], 2, g.d[k], st[k]);
    }
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const int a = p < 3 ? 0 : (p < 5 ? 1 : 2);
      const int b = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
      const int a1 = sel4(d1, a), b1 = sel4(d1, b);
      const M3<R> ua = L(a, si), ub = L(b, si);
      const M3<R> Pa = mul(ua, L(b, si + a1));
      const M3<R> Pb = mul(ub, L(a, si + b1));
      v[0] += (double)re_tr_mul_adj(Pa, Pb) - 3.0;
      if (RECT) {
        {
          const M3<R> A = mul(mul(ua, L(a, si + a1)), L(b, si + sel4(d2, a)));
          v[1] += (double)re_tr_mul_adj(A, mul(Pb, L(a, si + a1 + b1))) - 3.0;
        }
        {
          const M3<R> A = mul(mul(ub, L(b, si + b1)), L(a, si + sel4(d2, b)));
          v[1] += (double)re_tr_mul_adj(A, mul(Pa, L(b, si + a1 + b1))) - 3.0;
        }
      }
    }
  }
  block_reduce_store<2>(v, partials);
}

template <typename R>
cudaError_t launch_action(const Geo& g, const void* U, int rect, double* partials, cudaStream_t st, void* copy_f32)
{
  const Cx<R>* u = (const Cx<R>*)U;
  Cx<float>* c = (Cx<float>*)copy_f32;
  if (sizeof(R) == 8 && padded_sites(g.V) * 36 < 2147483647L) {
    if (rect) k_action_corners<R, true><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials, c);
    else k_action_corners<R, false><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials, c);
  } else if (padded_sites(g.V) * 36 < 2147483647L) {
    if (rect) k_action_loops<R, true><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials, c);
    else k_action_loops<R, false><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials, c);
  } else {  // 32-bit link offsets would overflow
    if (rect) k_action<R, true><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials);
    else k_action<R, false><<<reduce_blocks(g), RED_BS, 0, st>>>(g, u, partials);
    if (c != nullptr) return launch_convert<R, float>(padded_sites(g.V) * 4 * 18, U, c, st);
  }
  return cudaGetLastError();
}

// Clover leaf sum C_mu_nu(x) (the 4 leaves of qcd-acc.h:135-150, without the 1/4).
template <typename R>
__device__ __forceinline__ M3<R> clover_sum(const CField<R>& U, const Geo& g, const Coord& x, long s, int mu, int nu)
{
  // leaf 1: (mu, nu, -mu, -nu) = U_mu(x) U_nu(x+mu) [U_nu(x) U_mu(x+nu)]^+
  M3<R> C = mul_adj(mul(U.ld(s, mu), U.ld(site_rt(g, x, mu, 1, nu, 0), nu)),
                    mul(U.ld(s, nu), U.ld(site_rt(g, x, mu, 0, nu, 1), mu)));
  // leaf 2: (-mu, -nu, mu, nu) = [U_nu(x-mu-nu) U_mu(x-mu)]^+ U_mu(x-mu-nu) U_nu(x-nu)
  {
    const M3<R> a = mul(U.ld(site_rt(g, x, mu, -1, nu, -1), nu), U.ld(site_rt(g, x, mu, -1, nu, 0), mu));
    const M3<R> b = mul(U.ld(site_rt(g, x, mu, -1, nu, -1), mu), U.ld(site_rt(g, x, mu, 0, nu, -1), nu));
    C = add_adj_mul(C, a, b);
  }
  // leaf 3: (nu, -mu, -nu, mu) = U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
  {
    const M3<R> a = mul_adj(U.ld(s, nu), U.ld(site_rt(g, x, mu, -1, nu, 1), mu));
    const M3<R> b = adj_mul(U.ld(site_rt(g, x, mu, -1, nu, 0), nu), U.ld(site_rt(g, x, mu, -1, nu, 0), mu));
    C = add_mul(C, a, b);
  }
  // leaf 4: (-nu, mu, nu, -mu) = U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+
  {
    const M3<R> a = adj_mul(U.ld(site_rt(g, x, mu, 0, nu, -1), nu), U.ld(site_rt(g, x, mu, 0, nu, -1), mu));
    const M3<R> b = mul_adj(U.ld(site_rt(g, x, mu, 1, nu, -1), nu), U.ld(s, mu));
    C = add_mul(C, a, b);
  }
  return C;
}

// (C - C^+)/8 = the anti-Hermitian part of the leaf average C/4.
template <typename R>
__device__ __forceinline__ M3<R> leaf_antiherm(const M3<R>& C)
{
  M3<R> ah;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      ah.e[3 * r + c] = cx<R>(R(0.125) * (C.e[3 * r + c].re - C.e[3 * c + r].re),
                             R(0.125) * (C.e[3 * r + c].im + C.e[3 * c + r].im));
  return ah;
}

// -tr(G^2) with G = TA(C/4) = Fa - i Im(tr Fa)/3 (matrix-hmc.h:202-213)
template <typename R>
__device__ __forceinline__ double energy_of(const M3<R>& Fa)
{
  M3<R> G = Fa;
  const R t = (G.e[0].im + G.e[4].im + G.e[8].im) / R(3);
  G.e[0].im -= t;
  G.e[4].im -= t;
  G.e[8].im -= t;
  return -(double)re_tr_mul(G, G);
}

// Energy density E(x) = sum_{mu<nu} -tr(G_mu_nu^2), G = TA(C/4)
// (wilson-flow.cpp:99-129) and the clover topological charge density
// -1/(4 pi^2) [-tr(F02 F13) + tr(F03 F12) + tr(F23 F01)], F = (C/4 - C^+/4)/2
// (qcd.cpp:64-79), sharing the leaves; planes are visited in the pairs the
// charge needs so that only two plane matrices are live at a time.
template <typename R>
__global__ void __launch_bounds__(RED_BS) k_clover(Geo g, const Cx<R>* Up, R* ef, R* qf, double* partials)
{
  const long s = site_of_work(g, (long)blockIdx.x * blockDim.x + threadIdx.x, RED_BS);
  double v[2] = {0.0, 0.0};
  if (s < g.V && in_reduce(g, s)) {
    const CField<R> U{Up, g.V};
    const Coord x = coord_of(g, s);
    double e = 0.0, q = 0.0;
    // plane pairs (02,13) -, (03,12) +, (23,01) +
#pragma unroll 1
    for (int p = 0; p < 3; ++p) {
      const int m1 = p == 2 ? 2 : 0, n1 = p == 0 ? 2 : (p == 1 ? 3 : 3);
      const int m2 = p == 2 ? 0 : 1, n2 = p == 0 ? 3 : (p == 1 ? 2 : 1);
      const M3<R> Fa = leaf_antiherm(clover_sum<R>(U, g, x, s, m1, n1));
      const M3<R> Fb = leaf_antiherm(clover_sum<R>(U, g, x, s, m2, n2));
      e += energy_of(Fa) + energy_of(Fb);
      const double t = (double)re_tr_mul(Fa, Fb);
      q += p == 0 ? -t : t;
    }
    q *= -1.0 / (4.0 * 3.141592653589793 * 3.141592653589793);
    v[0] = e;
    v[1] = q;
    if (ef) ef[s] = (R)e;
    if (qf) qf[s] = (R)q;
  }
  block_reduce_store<2>(v, partials);
}

template <typename R>
cudaError_t launch_clover(const Geo& g, const void* U, void* e_field, void* q_field, double* partials,
                          cudaStream_t st)
{
  // the grid covers every site of the field: a domain's owned-box traversal does not apply here
  if (has_box(g)) return cudaErrorInvalidValue;
  Geo gk = g;  // z slabs on large lattices (the leaves reach one slice either way)
  set_slab_order(gk, RED_BS, (int)(18 * sizeof(R)));
  k_clover<R><<<reduce_blocks(g), RED_BS, 0, st>>>(gk, (const Cx<R>*)U, (R*)e_field, (R*)q_field, partials);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// 5-loop improved topological charge (qcd.cpp:425-489, hep-lat/9701012)

// Site index of x + the offsets (o0, o1, o2, o3), periodic.
__device__ __forceinline__ long site_of4(const Geo& g, int y0, int y1, int y2, int y3)
{
  return (long)y0 + (long)g.d[0] * ((long)y1 + (long)g.d[1] * ((long)y2 + (long)g.d[2] * (long)y3));
}

// Sum of the four m x n leaves at x in the (mu, nu) plane (qcd.cpp:11-31,
// without its 1/4): each a Wilson line of qcd-acc.h:23-41 walked link by link
// -- forward steps multiply by U_dir(y), backward steps by U_dir(y - dir)^+.
template <typename R>
__device__ M3<R> leaf_sum_mn(const CField<R>& U, const Geo& g, const Coord& x, int mu, int m, int nu, int n)
{
  M3<R> acc = m3_zero<R>();
#pragma unroll 1
  for (int l = 0; l < 4; ++l) {
    // leaves (mu m, nu n, -mu m, -nu n), (-mu m, -nu n, mu m, nu n),
    //        (nu n, -mu m, -nu n, mu m), (-nu n, mu m, nu n, -mu m)
    const int first = l < 2 ? mu : nu, second = l < 2 ? nu : mu;
    const int cf = l < 2 ? m : n, cs = l < 2 ? n : m;
    const int sf = (l == 0 || l == 2) ? 1 : -1;  // sign of the first leg
    const int ss = (l == 0 || l == 3) ? 1 : -1;  // sign of the second leg
    int y0 = x.c[0], y1 = x.c[1], y2 = x.c[2], y3 = x.c[3];
    M3<R> w = m3_unit<R>();
    bool first_link = true;
#pragma unroll 1
    for (int leg = 0; leg < 4; ++leg) {
      const int dir = (leg & 1) ? second : first;
      const int cnt = (leg & 1) ? cs : cf;
      const int sgn = ((leg & 1) ? ss : sf) * (leg < 2 ? 1 : -1);
#pragma unroll 1
      for (int r = 0; r < cnt; ++r) {
        if (sgn < 0) {
          y0 = dir == 0 ? wrap(y0 - 1, g.d[0]) : y0;
          y1 = dir == 1 ? wrap(y1 - 1, g.d[1]) : y1;
          y2 = dir == 2 ? wrap(y2 - 1, g.d[2]) : y2;
          y3 = dir == 3 ? wrap(y3 - 1, g.d[3]) : y3;
        }
        const M3<R> u = U.ld(site_of4(g, y0, y1, y2, y3), dir);
        if (first_link) w = sgn > 0 ? u : adj(u);  // 1 * u is u exactly
        else w = sgn > 0 ? mul(w, u) : mul_adj(w, u);
        first_link = false;
        if (sgn > 0) {
          y0 = dir == 0 ? wrap(y0 + 1, g.d[0]) : y0;
          y1 = dir == 1 ? wrap(y1 + 1, g.d[1]) : y1;
          y2 = dir == 2 ? wrap(y2 + 1, g.d[2]) : y2;
          y3 = dir == 3 ? wrap(y3 + 1, g.d[3]) : y3;
        }
      }
    }
    add_to(acc, w);
  }
  return acc;
}

// F = (C - C^+)/2 of the (averaged) m x n leaf C of plane p (qcd.cpp:536-568)
template <typename R>
__device__ M3<R> leaf_f_mn(const CField<R>& U, const Geo& g, const Coord& x, int p, int m, int n)
{
  const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2);
  const int nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
  M3<R> c = scale(R(0.25), leaf_sum_mn(U, g, x, mu, m, nu, n));
  if (m != n) {
    add_to(c, scale(R(0.25), leaf_sum_mn(U, g, x, mu, n, nu, m)));
    c = scale(R(0.5), c);
  }
  M3<R> f;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      f.e[3 * i + j] = cx<R>(R(0.5) * (c.e[3 * i + j].re - c.e[3 * j + i].re),
                             R(0.5) * (c.e[3 * i + j].im + c.e[3 * j + i].im));
  return f;
}

// Per site the five terms c_k / (m n)^2 * q_{m x n} (terms field, multiplicity
// 5, optional), their per-site sum (total field, optional), and the block
// partial sums of the five terms.
template <typename R>
__global__ void __launch_bounds__(RED_BS) k_topology_5li(Geo g, const Cx<R>* Up, R* terms, R* total, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (s < g.V) {
    const CField<R> U{Up, g.V};
    const Coord x = coord_of(g, s);
    const double c5 = 1.0 / 20.0;
    const double coef[5] = {(19.0 - 55.0 * c5) / 9.0, (1.0 - 64.0 * c5) / 9.0 / 16.0,
                            (-64.0 + 640.0 * c5) / 45.0 / 4.0, (1.0 / 5.0 - 2.0 * c5) / 9.0, c5 / 81.0};
    const double fac = -1.0 / (4.0 * 3.141592653589793 * 3.141592653589793);
    double tot = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const int m = k == 1 ? 2 : (k == 4 ? 3 : 1);
      const int n = k == 0 ? 1 : (k == 1 ? 2 : (k == 2 ? 2 : 3));
      double q = 0.0;
      // qcd.cpp:64-79: -tr(F02 F13) + tr(F03 F12) + tr(F23 F01)
#pragma unroll 1
      for (int pr = 0; pr < 3; ++pr) {
        const int pa = pr == 0 ? 1 : (pr == 1 ? 2 : 5), pb = pr == 0 ? 4 : (pr == 1 ? 3 : 0);
        const M3<R> fa = leaf_f_mn(U, g, x, pa, m, n);
        const M3<R> fb = leaf_f_mn(U, g, x, pb, m, n);
        const double t = (double)re_tr_mul(fa, fb);
        q += pr == 0 ? -t : t;
      }
      v[k] = coef[k] * (fac * q);
      tot += v[k];
    }
    if (terms) {
#pragma unroll
      for (int k = 0; k < 5; ++k) terms[lay_index<1>(g.V, k, 0, s)] = (R)v[k];
    }
    if (total) total[s] = (R)tot;
  }
  block_reduce_store<5>(v, partials);
}

template <typename R>
cudaError_t launch_topology_5li(const Geo& g, const void* U, void* terms, void* total, double* partials,
                                cudaStream_t st)
{
  k_topology_5li<R><<<reduce_blocks(g), RED_BS, 0, st>>>(g, (const Cx<R>*)U, (R*)terms, (R*)total, partials);
  return cudaGetLastError();
}

template <typename R>
__global__ void __launch_bounds__(RED_BS) k_qnorm(long n, const R* x, double* partials)
{
  double v[1] = {0.0};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double t = (double)x[i];
    v[0] += t * t;
  }
  block_reduce_store<1>(v, partials);
}

template <typename R>
cudaError_t launch_qnorm(long n_reals, const void* x, double* partials, int blocks, cudaStream_t st)
{
  k_qnorm<R><<<blocks, RED_BS, 0, st>>>(n_reals, (const R*)x, partials);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(1024) k_finalize(const double* partials, int nv, int blocks, double* results,
                                                   int slot)
{
  __shared__ double sm[32];
  for (int k = 0; k < nv; ++k) {
    double t = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) t += partials[(long)k * blocks + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sm[i];
      results[slot + k] = r;
    }
    __syncthreads();
  }
}

cudaError_t launch_finalize(const double* partials, int n_values, int blocks, double* results, int slot,
                            cudaStream_t st)
{
  k_finalize<<<1, 1024, 0, st>>>(partials, n_values, blocks, results, slot);
  return cudaGetLastError();
}

__global__ void k_combine(double* r, int out, int a, int b, int c) { r[out] = r[a] + r[b] - r[c]; }

cudaError_t launch_combine(double* results, int out, int a, int b, int c, cudaStream_t st)
{
  k_combine<<<1, 1, 0, st>>>(results, out, a, b, c);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// per-site random fields (qcd-utils.cpp:47-92)

struct RngArg {
  uint32_t v[24];
};

// One link's momentum from its 8 Gaussians (make_g_rand_anti_hermitian_matrix,
// matrix-hmc.h:125-142), stored in the field's precision.
template <typename R>
__device__ __forceinline__ void momentum_store(const WField<R>& Pf, long s, int mu, const double* b, double inv_sqrt3)
{
  const M3<double> m = x_make_anti_hermitian(b, inv_sqrt3);
  M3<R> mr;
#pragma unroll
  for (int k = 0; k < 9; ++k) mr.e[k] = cx<R>((R)m.e[k].re, (R)m.e[k].im);
  Pf.st(s, mu, mr);
}

// set_g_rand_anti_hermitian_matrix_field: per site RngState(rs, gindex),
// 4 x make_g_rand_anti_hermitian_matrix (matrix-hmc.h:125-142).
template <typename R>
__global__ void __launch_bounds__(128) k_rand_momentum(Geo g, RngArg ra, double s_sigma, double inv_sqrt3,
                                                       Cx<R>* P, int* ambiguous)
{
  // every lane of the warp stays to the end (warp-wide refills); lanes past
  // the last site draw nothing, and so do the halo sites of a domain, whose
  // momenta no force or sum reads (they are set to zero)
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool inside = s < g.V;
  const bool active = inside && (!has_box(g) || in_box(g, s));
  Rng base, rs;
  rng_import(base, ra.v);
  if (active) rng_split_long(rs, base, (int64_t)rng_index(g, s));
  int amb = 0;
  const WField<R> Pf{P, g.V};
  if (inside && !active) {
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) Pf.st(s, mu, m3_zero<R>());
  }
  // the 8 Gaussians of a link wait in shared memory (the draw index is a
  // run-time value; a per-thread array would live in local memory)
  __shared__ double sb[8 * 128];
  rng_gaussians_converged<32>(rs, s_sigma, active, &amb, [&](int i, double v) {
    sb[(i & 7) * 128 + threadIdx.x] = v;
    if ((i & 7) == 7) {
      double b[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) b[k] = sb[k * 128 + threadIdx.x];
      momentum_store(Pf, s, i >> 3, b, inv_sqrt3);
    }
  });
  if (amb) atomicAdd(ambiguous, 1);
}

template <typename R>
cudaError_t launch_rand_momentum(const Geo& g, void* P, const uint32_t* rs24, double sigma, int* ambiguous,
                                 cudaStream_t st)
{
  RngArg ra;
  memcpy(ra.v, rs24, sizeof(ra.v));
  const double s_sigma = sigma / sqrt(2.0);
  const double inv_sqrt3 = 1.0 / sqrt(3.0);
  const int bs = 128;
  k_rand_momentum<R><<<(unsigned)((g.V + bs - 1) / bs), bs, 0, st>>>(g, ra, s_sigma, inv_sqrt3, (Cx<R>*)P,
                                                                     ambiguous);
  return cudaGetLastError();
}

// The four links of one site of a hot start (below): per link n_step factors,
// each unitarize(exp_taylor20(X)) with X made from 8 Gaussians, multiplied in
// order.  The Gaussians come from rng_gaussians_converged, 8 per factor, so a
// warp's SHA-256 refills run together; the values are those of 8 successive
// g_rand_gen calls.  Called by all 32 lanes of a warp.
template <typename R>
__device__ __forceinline__ void hot_start_links(Rng& rs, bool active, double s_sigma, double inv_sqrt3, int n_step,
                                                const WField<R>& Uf, long s, int* amb)
{
  __shared__ double sb[8 * 128];  // the 8 Gaussians of a factor (run-time draw index)
  const int nk = n_step > 1 ? n_step : 1;  // the reference always draws at least one factor
  for (int mu = 0; mu < 4; ++mu) {
    M3<double> v;
    for (int k = 0; k < nk; ++k) {
      rng_gaussians_converged<8>(rs, s_sigma, active, amb,
                                 [&](int i, double x) { sb[i * 128 + threadIdx.x] = x; });
      double b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) b[i] = active ? sb[i * 128 + threadIdx.x] : 0.0;
      M3<double> e = x_exp_taylor20(x_make_anti_hermitian(b, inv_sqrt3));
      x_unitarize(e);
      v = (k == 0) ? e : xm_mul(v, e);
    }
    if (active) {
      M3<R> vr;
#pragma unroll
      for (int k = 0; k < 9; ++k) vr.e[k] = cx<R>((R)v.e[k].re, (R)v.e[k].im);
      Uf.st(s, mu, vr);
    }
  }
}

// set_g_rand_color_matrix_field: per link n_step products of
// unitarize(exp_taylor20(X)) with X from make_g_rand_anti_hermitian_matrix.
template <typename R>
__global__ void __launch_bounds__(128) k_hot_start(Geo g, RngArg ra, double s_sigma, double inv_sqrt3, int n_step,
                                                   Cx<R>* U, int* ambiguous)
{
  // every lane of the warp stays to the end (warp-wide refills); lanes past
  // the last site draw nothing and store nothing
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s < g.V;
  Rng base, rs;
  rng_import(base, ra.v);
  if (active) rng_split_long(rs, base, (int64_t)rng_index(g, s));
  int amb = 0;
  hot_start_links<R>(rs, active, s_sigma, inv_sqrt3, n_step, WField<R>{U, g.V}, s, &amb);
  if (amb) atomicAdd(ambiguous, 1);
}

template <typename R>
cudaError_t launch_hot_start(const Geo& g, void* U, const uint32_t* rs24, double sigma, int n_step, int* ambiguous,
                             cudaStream_t st)
{
  RngArg ra;
  memcpy(ra.v, rs24, sizeof(ra.v));
  const double s_sigma = sigma / sqrt(2.0);
  const double inv_sqrt3 = 1.0 / sqrt(3.0);
  const int bs = 128;
  k_hot_start<R><<<(unsigned)((g.V + bs - 1) / bs), bs, 0, st>>>(g, ra, s_sigma, inv_sqrt3, n_step, (Cx<R>*)U,
                                                                 ambiguous);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// batches of independent chains (all chains in one launch)

// Per-site random momenta of every chain: chain c uses RngState rs24[24 c ..]
// split by the site's index within its chain.
template <typename R>
__global__ void __launch_bounds__(128) k_rand_momentum_batch(long Vtot, int nchain, const long* __restrict__ offs,
                                                             const uint32_t* __restrict__ rs24, double s_sigma,
                                                             double inv_sqrt3, Cx<R>* P, int* ambiguous)
{
  const long sg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = sg < Vtot;
  Rng rs;
  if (active) {
    const int c = chain_of(offs, nchain, sg);
    Rng base;
    rng_import(base, rs24 + 24 * c);
    rng_split_long(rs, base, (int64_t)(sg - offs[c]));
  }
  int amb = 0;
  const WField<R> Pf{P, Vtot};
  double b[8];
  rng_gaussians_converged<32>(rs, s_sigma, active, &amb, [&](int i, double v) {
    b[i & 7] = v;
    if ((i & 7) == 7) momentum_store(Pf, sg, i >> 3, b, inv_sqrt3);
  });
  if (amb) atomicAdd(ambiguous, 1);
}

template <typename R>
__global__ void __launch_bounds__(128) k_hot_start_batch(long Vtot, int nchain, const long* __restrict__ offs,
                                                         const uint32_t* __restrict__ rs24, double s_sigma,
                                                         double inv_sqrt3, int n_step, Cx<R>* U, int* ambiguous)
{
  const long sg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = sg < Vtot;
  Rng rs;
  if (active) {
    const int c = chain_of(offs, nchain, sg);
    Rng base;
    rng_import(base, rs24 + 24 * c);
    rng_split_long(rs, base, (int64_t)(sg - offs[c]));
  }
  int amb = 0;
  hot_start_links<R>(rs, active, s_sigma, inv_sqrt3, n_step, WField<R>{U, Vtot}, sg, &amb);
  if (amb) atomicAdd(ambiguous, 1);
}

// Site values for the per-chain Hamiltonians: what = 0: sum_mu -tr(P^2)/2 from
// P into vals[sg]; what = 1: plaquette sum (vals[sg]) and, if rect, rectangle
// sum (vals[Vtot + sg]) from U.
template <typename R>
__global__ void __launch_bounds__(128) k_site_values_batch(long Vtot, int nchain, const long* __restrict__ offs,
                                                           const ChainInfo* __restrict__ chains, int what, int rect,
                                                           const Cx<R>* F, double* vals)
{
  const long sg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (sg >= Vtot) return;
  const CField<R> Ff{F, Vtot};
  if (what == 0) {
    double v = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) v += neg_half_tr_square(Ff.ld(sg, mu));
    vals[sg] = v;
    return;
  }
  const int c = chain_of(offs, nchain, sg);
  const Geo g = chain_geo(chains[c]);
  const Coord x = coord_of(g, sg - g.off);
  double sp = 0.0, sr = 0.0;
#pragma unroll 1
  for (int p = 0; p < 6; ++p) {
    const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
    const M3<R> A = mul(Ff.ld(sg, mu), Ff.ld(site_rt(g, x, mu, 1, nu, 0), nu));
    const M3<R> B = mul(Ff.ld(sg, nu), Ff.ld(site_rt(g, x, mu, 0, nu, 1), mu));
    sp += (double)re_tr_mul_adj(A, B) - 3.0;
    if (rect) {
#pragma unroll 1
      for (int o = 0; o < 2; ++o) {
        const int a = o == 0 ? mu : nu, b = o == 0 ? nu : mu;
        M3<R> A2 = mul(Ff.ld(sg, a), Ff.ld(site_rt(g, x, a, 1, b, 0), a));
        A2 = mul(A2, Ff.ld(site_rt(g, x, a, 2, b, 0), b));
        M3<R> B2 = mul(Ff.ld(sg, b), Ff.ld(site_rt(g, x, a, 0, b, 1), a));
        B2 = mul(B2, Ff.ld(site_rt(g, x, a, 1, b, 1), a));
        sr += (double)re_tr_mul_adj(A2, B2) - 3.0;
      }
    }
  }
  vals[sg] = sp;
  if (rect) vals[Vtot + sg] = sr;
}

// out[c] = sum of vals over chain c's sites, one block per chain, fixed order.
__global__ void __launch_bounds__(256) k_segment_sum(int nchain, const long* __restrict__ offs,
                                                     const double* __restrict__ vals, double* out)
{
  const int c = blockIdx.x;
  const long a = offs[c], b = offs[c + 1];
  double t = 0.0;
  for (long i = a + threadIdx.x; i < b; i += blockDim.x) t += vals[i];
  __shared__ double sm[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int i = 0; i < 8; ++i) r += sm[i];
    out[c] = r;
  }
}

// dst = src on the sites of chains whose flag is set (4 links per site).
template <typename R>
__global__ void k_accept_batch(long Vtot, int nchain, const long* __restrict__ offs, const int* __restrict__ flags,
                               Cx<R>* dst, const Cx<R>* src)
{
  const long sg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (sg >= Vtot) return;
  const int c = chain_of(offs, nchain, sg);
  if (!flags[c]) return;
  const CField<R> S{src, Vtot};
  const WField<R> D{dst, Vtot};
  for (int mu = 0; mu < 4; ++mu) D.st(sg, mu, S.ld(sg, mu));
}

template <typename R>
cudaError_t launch_rand_momentum_batch(long Vtot, int nchain, const long* offs, const uint32_t* rs24, double sigma,
                                       void* P, int* ambiguous, cudaStream_t st)
{
  k_rand_momentum_batch<R><<<(unsigned)((Vtot + 127) / 128), 128, 0, st>>>(Vtot, nchain, offs, rs24, sigma / sqrt(2.0),
                                                                          1.0 / sqrt(3.0), (Cx<R>*)P, ambiguous);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_hot_start_batch(long Vtot, int nchain, const long* offs, const uint32_t* rs24, double sigma,
                                   int n_step, void* U, int* ambiguous, cudaStream_t st)
{
  k_hot_start_batch<R><<<(unsigned)((Vtot + 127) / 128), 128, 0, st>>>(Vtot, nchain, offs, rs24, sigma / sqrt(2.0),
                                                                      1.0 / sqrt(3.0), n_step, (Cx<R>*)U, ambiguous);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_site_values_batch(long Vtot, int nchain, const long* offs, const ChainInfo* chains, int what,
                                     int rect, const void* F, double* vals, cudaStream_t st)
{
  k_site_values_batch<R><<<(unsigned)((Vtot + 127) / 128), 128, 0, st>>>(Vtot, nchain, offs, chains, what, rect,
                                                                        (const Cx<R>*)F, vals);
  return cudaGetLastError();
}

cudaError_t launch_segment_sum(int nchain, const long* offs, const double* vals, double* out, cudaStream_t st)
{
  k_segment_sum<<<nchain, 256, 0, st>>>(nchain, offs, vals, out);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_accept_batch(long Vtot, int nchain, const long* offs, const int* flags, void* dst, const void* src,
                                cudaStream_t st)
{
  k_accept_batch<R><<<(unsigned)((Vtot + 127) / 128), 128, 0, st>>>(Vtot, nchain, offs, flags, (Cx<R>*)dst,
                                                                    (const Cx<R>*)src);
  return cudaGetLastError();
}

template cudaError_t launch_rand_momentum_batch<double>(long, int, const long*, const uint32_t*, double, void*, int*,
                                                        cudaStream_t);
template cudaError_t launch_hot_start_batch<double>(long, int, const long*, const uint32_t*, double, int, void*, int*,
                                                    cudaStream_t);
template cudaError_t launch_site_values_batch<double>(long, int, const long*, const ChainInfo*, int, int, const void*,
                                                      double*, cudaStream_t);
template cudaError_t launch_site_values_batch<float>(long, int, const long*, const ChainInfo*, int, int, const void*,
                                                     double*, cudaStream_t);
template cudaError_t launch_accept_batch<double>(long, int, const long*, const int*, void*, const void*, cudaStream_t);

// ------------------------------------------------------------------------
// elementwise field operations

template <typename R>
__global__ void k_set_unit(long V, int m, Cx<R>* U)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const WField<R> Uf{U, V};
  for (int mu = 0; mu < m; ++mu) Uf.st(s, mu, m3_unit<R>());
}

template <typename R>
cudaError_t launch_set_unit(const Geo& g, int m, void* U, cudaStream_t st)
{
  k_set_unit<R><<<(unsigned)((g.V + 255) / 256), 256, 0, st>>>(g.V, m, (Cx<R>*)U);
  return cudaGetLastError();
}

template <typename R>
__global__ void k_axpby(long n, R* y, R a, const R* x, R b)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const R xv = x ? x[i] : R(0);
    y[i] = (b == R(0)) ? a * xv : fma(a, xv, b * y[i]);
  }
}

template <typename R>
cudaError_t launch_axpby(long n, void* y, double a, const void* x, double b, cudaStream_t st)
{
  const long blocks = (n + 255) / 256;
  k_axpby<R><<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, st>>>(n, (R*)y, (R)a, (const R*)x, (R)b);
  return cudaGetLastError();
}

// reference image [site][m][k] (doubles) <-> device layout (gauge_common.cuh).
// Sites [off, off + n) of a field of Vf sites; the image holds those n sites.
// One thread per (component, site), sites fastest, so the device-side accesses
// of a warp are coalesced.
template <typename R>
__global__ void k_aos_to_store(long Vf, long off, long n, int m, int k_per, const double* __restrict__ aos,
                               R* __restrict__ store)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * m) return;
  const int mm = (int)(i / n);
  const long s = i % n;
  const double* src = aos + (s * m + mm) * k_per;
  if (k_per == 1) {
    store[lay_index<1>(Vf, mm, 0, off + s)] = (R)src[0];
  } else {
    Cx<R>* dst = (Cx<R>*)store + lay_index<9>(Vf, mm, 0, off + s);
#pragma unroll
    for (int c = 0; c < 9; ++c) dst[32 * c] = cx<R>((R)src[2 * c], (R)src[2 * c + 1]);
  }
}

template <typename R>
__global__ void k_store_to_aos(long Vf, long off, long n, int m, int k_per, const R* __restrict__ store,
                               double* __restrict__ aos)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * m) return;
  const int mm = (int)(i / n);
  const long s = i % n;
  double* dst = aos + (s * m + mm) * k_per;
  if (k_per == 1) {
    dst[0] = (double)store[lay_index<1>(Vf, mm, 0, off + s)];
  } else {
    const Cx<R>* src = (const Cx<R>*)store + lay_index<9>(Vf, mm, 0, off + s);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const Cx<R> v = src[32 * c];
      dst[2 * c] = (double)v.re;
      dst[2 * c + 1] = (double)v.im;
    }
  }
}

template <typename R>
cudaError_t launch_aos_to_store(long Vf, long off, long n, int m, int k_per, const double* aos, void* store,
                                cudaStream_t st)
{
  const long t = n * m;
  k_aos_to_store<R><<<(unsigned)((t + 255) / 256), 256, 0, st>>>(Vf, off, n, m, k_per, aos, (R*)store);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_store_to_aos(long Vf, long off, long n, int m, int k_per, const void* store, double* aos,
                                cudaStream_t st)
{
  const long t = n * m;
  k_store_to_aos<R><<<(unsigned)((t + 255) / 256), 256, 0, st>>>(Vf, off, n, m, k_per, (const R*)store, aos);
  return cudaGetLastError();
}

template <typename RI, typename RO>
__global__ void k_convert(long n, const RI* in, RO* out)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (RO)in[i];
}

// four elements per thread: 16- or 32-byte loads and stores (n % 4 == 0, 16-byte aligned buffers)
template <typename RI, typename RO>
__global__ void k_convert4(long n4, const RI* __restrict__ in, RO* __restrict__ out)
{
  using I2 = typename std::conditional<sizeof(RI) == 8, double2, float2>::type;
  using O2 = typename std::conditional<sizeof(RO) == 8, double2, float2>::type;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    const I2 a = reinterpret_cast<const I2*>(in)[2 * i], b = reinterpret_cast<const I2*>(in)[2 * i + 1];
    O2 c, d;
    c.x = (decltype(c.x))a.x;
    c.y = (decltype(c.y))a.y;
    d.x = (decltype(d.x))b.x;
    d.y = (decltype(d.y))b.y;
    reinterpret_cast<O2*>(out)[2 * i] = c;
    reinterpret_cast<O2*>(out)[2 * i + 1] = d;
  }
}

template <typename RI, typename RO>
cudaError_t launch_convert(long n, const void* in, void* out, cudaStream_t st)
{
  const bool vec = n % 4 == 0 && ((uintptr_t)in % 16) == 0 && ((uintptr_t)out % 16) == 0;
  const long work = vec ? n / 4 : n;
  const long blocks = (work + 255) / 256;
  const unsigned grid = (unsigned)(blocks < 148 * 16 ? blocks : 148 * 16);
  if (vec) k_convert4<RI, RO><<<grid, 256, 0, st>>>(work, (const RI*)in, (RO*)out);
  else k_convert<RI, RO><<<grid, 256, 0, st>>>(n, (const RI*)in, (RO*)out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// explicit instantiations

#define QGB_INST(R)                                                                                          \
  template cudaError_t launch_evolve<R>(const Geo&, void*, const void*, double, int, int, cudaStream_t);    \
  template cudaError_t launch_gm_hamilton<R>(const Geo&, const void*, double*, cudaStream_t);              \
  template cudaError_t launch_action<R>(const Geo&, const void*, int, double*, cudaStream_t, void*);       \
  template cudaError_t launch_clover<R>(const Geo&, const void*, void*, void*, double*, cudaStream_t);     \
  template cudaError_t launch_topology_5li<R>(const Geo&, const void*, void*, void*, double*, cudaStream_t); \
  template cudaError_t launch_qnorm<R>(long, const void*, double*, int, cudaStream_t);                    \
  template cudaError_t launch_rand_momentum<R>(const Geo&, void*, const uint32_t*, double, int*, cudaStream_t); \
  template cudaError_t launch_hot_start<R>(const Geo&, void*, const uint32_t*, double, int, int*, cudaStream_t); \
  template cudaError_t launch_set_unit<R>(const Geo&, int, void*, cudaStream_t);                          \
  template cudaError_t launch_axpby<R>(long, void*, double, const void*, double, cudaStream_t);           \
  template cudaError_t launch_aos_to_store<R>(long, long, long, int, int, const double*, void*, cudaStream_t); \
  template cudaError_t launch_store_to_aos<R>(long, long, long, int, int, const void*, double*, cudaStream_t);

QGB_INST(double)
QGB_INST(float)
template cudaError_t launch_unitarize<double, double>(const Geo&, int, void*, cudaStream_t);
template cudaError_t launch_unitarize<float, float>(const Geo&, int, void*, cudaStream_t);
template cudaError_t launch_unitarize<float, double>(const Geo&, int, void*, cudaStream_t);
template cudaError_t launch_gm_hamilton_convert<double, float>(const Geo&, const void*, void*, double*, cudaStream_t);
template cudaError_t launch_gm_hamilton_convert<float, double>(const Geo&, const void*, void*, double*, cudaStream_t);
template cudaError_t launch_convert<double, float>(long, const void*, void*, cudaStream_t);
template cudaError_t launch_convert<float, double>(long, const void*, void*, cudaStream_t);
template cudaError_t launch_convert<double, double>(long, const void*, void*, cudaStream_t);
template cudaError_t launch_convert<float, float>(long, const void*, void*, cudaStream_t);

}  // namespace qgb

namespace qgb
{
// ------------------------------------------------------------------------
// host RngState API

void rng_host_seed(uint32_t out[24], const char* seed)
{
  Rng r;
  memset(&r, 0, sizeof(r));
  memcpy(r.hash, qgb_sha_host.h0, 32);
  r.type = RNG_NO_TYPE;
  if (!seed) {  // RngState(): reset(rs) only
    rng_export(out, r);
    return;
  }
  Rng o;
  rng_split_bytes(o, r, (const uint8_t*)seed, (int)strlen(seed));
  rng_export(out, o);
}

bool rng_host_split(uint32_t out[24], const uint32_t rs[24], const char* sindex)
{
  Rng r, o;
  rng_import(r, rs);
  if (!rng_split_bytes(o, r, (const uint8_t*)sindex, (int)strlen(sindex))) return false;
  rng_export(out, o);
  return true;
}

uint64_t rng_host_rand_gen(uint32_t rs[24])
{
  Rng r;
  rng_import(r, rs);
  const uint64_t v = rng_rand_gen(r);
  rng_export(rs, r);
  return v;
}

double rng_host_u_rand_gen(uint32_t rs[24], double upper, double lower)
{
  Rng r;
  rng_import(r, rs);
  const double v = rng_u_rand_gen(r, upper, lower);
  rng_export(rs, r);
  return v;
}

double rng_host_g_rand_gen(uint32_t rs[24], double center, double sigma)
{
  Rng r;
  rng_import(r, rs);
  const double v = rng_g_rand_gen<false>(r, center, sigma, nullptr);
  rng_export(rs, r);
  return v;
}
// ------------------------------------------------------------------------
// box pack / unpack (halo exchange of a domain-decomposed field)

template <typename E>
__global__ void k_box_copy(Geo g, int K, int lo0, int lo1, int lo2, int lo3, int n0, int n1, int n2, long nbox,
                           E* field, E* buf, bool unpack)
{
  const long w = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nbox) return;
  const int c = blockIdx.y;  // component * K + entry
  const int m = c / K, k = c - m * K;
  long r = w;
  const long x0 = r % n0 + lo0;
  r /= n0;
  const long x1 = r % n1 + lo1;
  r /= n1;
  const long x2 = r % n2 + lo2;
  const long x3 = r / n2 + lo3;
  const long s = x0 + (long)g.d[0] * (x1 + (long)g.d[1] * (x2 + (long)g.d[2] * x3));
  const long fi = ((m * site_blocks(g.V) + (s >> 5)) * K + k) * 32 + (s & 31);
  const long bi = (long)c * nbox + w;
  if (unpack) field[fi] = buf[bi];
  else buf[bi] = field[fi];
}

template <typename E>
cudaError_t launch_box_copy(const Geo& g, int m, int K, const int lo[4], const int n[4], void* field, void* buf,
                            bool unpack, cudaStream_t st)
{
  const long nbox = (long)n[0] * n[1] * n[2] * n[3];
  if (nbox == 0) return cudaSuccess;
  dim3 grid((unsigned)((nbox + 255) / 256), (unsigned)(m * K));
  k_box_copy<E><<<grid, 256, 0, st>>>(g, K, lo[0], lo[1], lo[2], lo[3], n[0], n[1], n[2], nbox, (E*)field, (E*)buf,
                                      unpack);
  return cudaGetLastError();
}

template cudaError_t launch_box_copy<double2>(const Geo&, int, int, const int*, const int*, void*, void*, bool,
                                              cudaStream_t);
template cudaError_t launch_box_copy<float2>(const Geo&, int, int, const int*, const int*, void*, void*, bool,
                                             cudaStream_t);
template cudaError_t launch_box_copy<double>(const Geo&, int, int, const int*, const int*, void*, void*, bool,
                                             cudaStream_t);
template cudaError_t launch_box_copy<float>(const Geo&, int, int, const int*, const int*, void*, void*, bool,
                                            cudaStream_t);

}  // namespace qgb
