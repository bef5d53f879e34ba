// force_impl.cuh -- the gauge force kernel and its fused consumers.
// Included once per precision (force_f64.cu, force_f32.cu) so the two
// instantiations compile in parallel.
#pragma once

#include "gauge_common.cuh"

namespace qgb
{

// ------------------------------------------------------------------------
// staples
//
// Sum over the 6 signed directions e = +-nu (nu != mu) of the plaquette
// staple and, for c1 != 0, the three rectangle shapes of hmc.cpp:27-46
// (paths in the reference's signed-direction encoding):
//   plaq  (nu, mu, -nu)            = B Hb
//   rect1 (nu, nu, mu, -nu, -nu)   = C1 Hb
//   rect2 (nu, mu, mu, -nu, -mu)   = B U_mu(x+e+mu) hop_back(x+e+2mu) U_mu(x+mu)^+
//   rect3 (-mu, nu, mu, mu, -nu)   = C3 Hb
// with A = hop(x) (the link from x to x+e), B = A U_mu(x+e), Hb =
// hop_back(x+e+mu) (the link from x+e+mu to x+mu), C1 = A hop(x+e) U_mu(x+2e)
// hop_back(x+2e+mu), C3 = U_mu(x-mu)^+ hop(x-mu) U_mu(x-mu+e) U_mu(x+e).
// The common right factor Hb is applied once to (1-8c1) B + c1 (C1 + C3):
// 11 matrix products per signed direction instead of the 14 of walking the
// four paths separately.  The sum equals the reference's
// gf_all_staple_no_comm (hmc.cpp:48-62) up to the order of the
// floating-point additions.
//
// The chains are evaluated one after another with the loops kept rolled, so
// at most five 3x3 matrices are live (accumulator, B or T, chain product,
// loaded link, product being formed): ~180 registers in FP64, ~90 in FP32.

// hop(y) for the signed direction: sgn = +1: U_nu(y); sgn = -1: U_nu(y - nu)^+.
// `where` is the site of the stored link (y or y - nu); the caller picks
// mul / adj_mul / mul_adj accordingly.

template <typename R, bool RECT>
__device__ __forceinline__ M3<R> staple_sum_rt(const CField<R>& U, const Geo& g, const Coord& x, int mu, R cp, R cr)
{
  M3<R> S = m3_zero<R>();
#pragma unroll 1
  for (int k = 0; k < 6; ++k) {
    const int nu = (mu + 1 + (k >> 1)) & 3;  // the three directions != mu
    const int s = (k & 1) ? -1 : 1;          // sign of e
    // B = A U_mu(x+e)
    M3<R> B;
    if (s > 0) B = mul(U.ld(site_rt(g, x, mu, 0, nu, 0), nu), U.ld(site_rt(g, x, mu, 0, nu, 1), mu));
    else B = adj_mul(U.ld(site_rt(g, x, mu, 0, nu, -1), nu), U.ld(site_rt(g, x, mu, 0, nu, -1), mu));
    if (!RECT) {
      // S += B Hb
      if (s > 0) S = add_mul_adj(S, B, U.ld(site_rt(g, x, mu, 1, nu, 0), nu));
      else S = add_mul(S, B, U.ld(site_rt(g, x, mu, 1, nu, -1), nu));
      continue;
    }
    // rect2: S += c1 B U_mu(x+e+mu) hop_back(x+e+2mu) U_mu(x+mu)^+
    {
      M3<R> C = mul(B, U.ld(site_rt(g, x, mu, 1, nu, s), mu));
      if (s > 0) C = mul_adj(C, U.ld(site_rt(g, x, mu, 2, nu, 0), nu));
      else C = mul(C, U.ld(site_rt(g, x, mu, 2, nu, -1), nu));
      C = mul_adj(C, U.ld(site_rt(g, x, mu, 1, nu, 0), mu));
      axpy(S, cr, C);
    }
    M3<R> T = scale(cp, B);
    // rect1: C1 = A hop(x+e) U_mu(x+2e) hop_back(x+2e+mu)
    {
      M3<R> C;
      if (s > 0) {
        C = mul(U.ld(site_rt(g, x, mu, 0, nu, 0), nu), U.ld(site_rt(g, x, mu, 0, nu, 1), nu));
        C = mul(C, U.ld(site_rt(g, x, mu, 0, nu, 2), mu));
        C = mul_adj(C, U.ld(site_rt(g, x, mu, 1, nu, 1), nu));
      } else {
        // A hop(x-nu) = [U_nu(x-2nu) U_nu(x-nu)]^+
        C = mul(U.ld(site_rt(g, x, mu, 0, nu, -2), nu), U.ld(site_rt(g, x, mu, 0, nu, -1), nu));
        C = adj_mul(C, U.ld(site_rt(g, x, mu, 0, nu, -2), mu));
        C = mul(C, U.ld(site_rt(g, x, mu, 1, nu, -2), nu));
      }
      axpy(T, cr, C);
    }
    // rect3: C3 = U_mu(x-mu)^+ hop(x-mu) U_mu(x-mu+e) U_mu(x+e)
    {
      M3<R> C;
      if (s > 0) {
        C = adj_mul(U.ld(site_rt(g, x, mu, -1, nu, 0), mu), U.ld(site_rt(g, x, mu, -1, nu, 0), nu));
      } else {
        // U_mu(x-mu)^+ U_nu(x-mu-nu)^+ = [U_nu(x-mu-nu) U_mu(x-mu)]^+
        C = mul(U.ld(site_rt(g, x, mu, -1, nu, -1), nu), U.ld(site_rt(g, x, mu, -1, nu, 0), mu));
        C = adj(C);
      }
      C = mul(C, U.ld(site_rt(g, x, mu, -1, nu, s), mu));
      C = mul(C, U.ld(site_rt(g, x, mu, 0, nu, s), mu));
      axpy(T, cr, C);
    }
    // S += T Hb
    if (s > 0) S = add_mul_adj(S, T, U.ld(site_rt(g, x, mu, 1, nu, 0), nu));
    else S = add_mul(S, T, U.ld(site_rt(g, x, mu, 1, nu, -1), nu));
  }
  if (!RECT) S = scale(cp, S);
  return S;
}

// ------------------------------------------------------------------------
// force: F = TA(-beta/3 U_mu(x) S^+) (hmc.cpp:64-75) and its fused consumers

template <typename R, int MODE, bool RECT>
__global__ void __launch_bounds__(128) k_force(Geo g, ForceArgs a)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int mu = blockIdx.y;
  const CField<R> U{(const Cx<R>*)a.U, g.V};
  const Coord x = coord_of(g, s);
  const R cp = R(1.0 - 8.0 * a.c1), cr = R(a.c1);
  const M3<R> S = staple_sum_rt<R, RECT>(U, g, x, mu, cp, cr);
  const M3<R> u = U.ld(s, mu);
  M3<R> F = traceless_antiherm(mul_adj(u, S));
  F = scale(R(-a.beta / 3.0), F);
  if (MODE == FORCE_SET) {
    WField<R>{(Cx<R>*)a.out, g.V}.st(s, mu, F);
  } else if (MODE == FORCE_UPDATE) {
    const WField<R> P{(Cx<R>*)a.out, g.V};
    M3<R> p = P.ld(s, mu);
    axpy(p, R(a.dt), F);
    P.st(s, mu, p);
  } else {
    M3<R> Z = F;
    if (MODE == FORCE_FLOW) {
      Z = scale(R(a.a), F);
      if (a.zp != nullptr && a.b != 0.0) axpy(Z, R(a.b), CField<R>{(const Cx<R>*)a.zp, g.V}.ld(s, mu));
      if (a.z != nullptr) WField<R>{(Cx<R>*)a.z, g.V}.st(s, mu, Z);
    }
    M3<R> un = mul(exp_ch(scale(R(a.dt), Z)), u);
    if (a.unitarize) unitarize(un);
    WField<R>{(Cx<R>*)a.out, g.V}.st(s, mu, un);
  }
}

template <typename R>
cudaError_t launch_force(const Geo& g, ForceMode mode, const ForceArgs& a, cudaStream_t st)
{
  const int bs = 128;
  dim3 grid((unsigned)((g.V + bs - 1) / bs), 4);
  const bool rect = a.c1 != 0.0;
#define QGB_LAUNCH(M)                                       \
  if (rect) k_force<R, M, true><<<grid, bs, 0, st>>>(g, a); \
  else k_force<R, M, false><<<grid, bs, 0, st>>>(g, a);
  switch (mode) {
    case FORCE_SET: QGB_LAUNCH(FORCE_SET) break;
    case FORCE_UPDATE: QGB_LAUNCH(FORCE_UPDATE) break;
    case FORCE_EVOLVE: QGB_LAUNCH(FORCE_EVOLVE) break;
    case FORCE_FLOW: QGB_LAUNCH(FORCE_FLOW) break;
  }
#undef QGB_LAUNCH
  return cudaGetLastError();
}

}  // namespace qgb
