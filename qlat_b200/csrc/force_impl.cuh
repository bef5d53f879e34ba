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

// Positions are x + a mu + b e with e = s nu (s = +1 or -1).  The link from
// such a point along +e ("hop") is U_nu(y) for s = +1 and U_nu(y - nu)^+ for
// s = -1; the link along -e ("back") is U_nu(y - nu)^+ for s = +1 and U_nu(y)
// for s = -1.  Both signs therefore run the same code: only the stored site
// and a warp-uniform conjugate-transpose differ, which keeps the loop body
// small enough for the instruction cache.

template <typename R>
struct SignedDir {
  const CField<R>& U;
  const Geo& g;
  const Coord& x;
  int mu, nu, s;
  __device__ __forceinline__ M3<R> umu(int a, int b) const { return U.ld(site_rt(g, x, mu, a, nu, b * s), mu); }
  __device__ __forceinline__ M3<R> hop(int a, int b) const
  {
    M3<R> m = U.ld(site_rt(g, x, mu, a, nu, b * s + (s < 0 ? -1 : 0)), nu);
    return s < 0 ? adj(m) : m;
  }
  __device__ __forceinline__ M3<R> back(int a, int b) const
  {
    M3<R> m = U.ld(site_rt(g, x, mu, a, nu, b * s + (s < 0 ? 0 : -1)), nu);
    return s < 0 ? m : adj(m);
  }
};

template <typename R, bool RECT>
__device__ __forceinline__ M3<R> staple_sum_rt(const CField<R>& U, const Geo& g, const Coord& x, int mu, R cp, R cr,
                                               int k0, int k1)
{
  M3<R> S = m3_zero<R>();
#pragma unroll 1
  for (int k = k0; k < k1; ++k) {
    const SignedDir<R> d{U, g, x, mu, (mu + 1 + (k >> 1)) & 3, (k & 1) ? -1 : 1};
    // B = hop(x) U_mu(x+e)
    const M3<R> B = mul(d.hop(0, 0), d.umu(0, 1));
    if (!RECT) {
      S = add_mul(S, B, d.back(1, 1));
      continue;
    }
    // rect2: S += c1 B U_mu(x+e+mu) back(x+e+2mu) U_mu(x+mu)^+
    {
      M3<R> C = mul(B, d.umu(1, 1));
      C = mul(C, d.back(2, 1));
      C = mul_adj(C, d.umu(1, 0));
      axpy(S, cr, C);
    }
    M3<R> T = scale(cp, B);
    // rect1: C1 = hop(x) hop(x+e) U_mu(x+2e) back(x+2e+mu)
    {
      M3<R> C = mul(d.hop(0, 0), d.hop(0, 1));
      C = mul(C, d.umu(0, 2));
      C = mul(C, d.back(1, 2));
      axpy(T, cr, C);
    }
    // rect3: C3 = U_mu(x-mu)^+ hop(x-mu) U_mu(x-mu+e) U_mu(x+e)
    {
      M3<R> C = adj_mul(d.umu(-1, 0), d.hop(-1, 0));
      C = mul(C, d.umu(-1, 1));
      C = mul(C, d.umu(0, 1));
      axpy(T, cr, C);
    }
    // S += T back(x+e+mu)
    S = add_mul(S, T, d.back(1, 1));
  }
  if (!RECT) S = scale(cp, S);
  return S;
}

// ------------------------------------------------------------------------
// staples with precomputed neighbour offsets
//
// The same sum as staple_sum_rt, evaluated with
// - neighbour sites as the thread's own site plus per-direction offsets:
//   site(x + a mu + b nu) = site(x) + D_mu(a) + D_nu(b) because mu != nu, with
//   D_k(a) = (wrap(x_k + a) - x_k) * stride_k computed once per thread for mu
//   and once per nu, instead of a 4-d wrap and index polynomial per load;
// - the sign of e = s nu as a template parameter, so the conjugate transposes
//   of the stored links fold into the products (mul_adj / adj_mul) instead of
//   being selected at run time;
// - hop(x) and U_mu(x+e), each used twice per direction, loaded once.
// Offsets are 32-bit: the launcher uses this form only when 36 V < 2^31.

// LinkLd, sel4 and nb_delta: gauge_common.cuh.

// One signed direction e = SG nu.  dn1 = D_nu(SG), dn2 = D_nu(2 SG).
// Stored links: hop(x + a mu + b e) is U_nu at D_nu(b) (SG > 0) or U_nu^+ at
// D_nu(-b-1) (SG < 0); back(x + a mu + b e) is U_nu^+ at D_nu(b-1) (SG > 0) or
// U_nu at D_nu(-b) (SG < 0).  For SG < 0 the products of two adjoints are
// formed as the adjoint of the reversed product ((H2 H)^+ = H^+ H2^+).
// Order: rect1 and rect3 (ending with U_mu(x+e)) first, then B = hop(x)
// U_mu(x+e) and rect2, so at most the accumulators S and T, hop(x), the chain
// product, a loaded link and the product being formed are live.
// TWO: carry the SU(3)-valued chains as two rows (mul2 / complete in
// su3.cuh): 924 instead of 1188 multiply-adds per direction.  Used for FP32
// only; FP64 keeps full products, identical in structure to the reference's.
template <typename R, bool RECT, int SG>
__device__ __forceinline__ void staple_dir_two_row(M3<R>& S, const LinkLd<R>& L, int s, int mu, int nu, int dmm1,
                                                   int dmp1, int dmp2, int dn1, int dn2, R cp, R cr)
{
  if (SG > 0) {
    const M3<R> H = L(nu, s);
    if (!RECT) {
      S = add_mul_adj(S, complete(mul2(H, L(mu, s + dn1))), L(nu, s + dmp1));
      return;
    }
    M3<R> T;
    {
      M32<R> C = mul2(H, L(nu, s + dn1));
      C = mul2(C, L(mu, s + dn2));
      C = mul2_adj(C, L(nu, s + dmp1 + dn1));
      T = scale(cr, complete(C));
    }
    M3<R> U01;
    {
      M32<R> C = adj_mul2(L(mu, s + dmm1), L(nu, s + dmm1));
      C = mul2(C, L(mu, s + dmm1 + dn1));
      U01 = L(mu, s + dn1);
      C = mul2(C, U01);
      axpy(T, cr, complete(C));
    }
    const M32<R> B2 = mul2(H, U01);
    axpy(T, cp, complete(B2));
    {
      M32<R> C = mul2(B2, L(mu, s + dmp1 + dn1));
      C = mul2_adj(C, L(nu, s + dmp2));
      C = mul2_adj(C, L(mu, s + dmp1));
      axpy(S, cr, complete(C));
    }
    S = add_mul_adj(S, T, L(nu, s + dmp1));
  } else {
    const M3<R> H = L(nu, s + dn1);
    if (!RECT) {
      S = add_mul(S, complete(adj_mul2(H, L(mu, s + dn1))), L(nu, s + dmp1 + dn1));
      return;
    }
    M3<R> T;
    {
      const M3<R> P = complete(mul2(L(nu, s + dn2), H));
      M32<R> C = adj_mul2(P, L(mu, s + dn2));
      C = mul2(C, L(nu, s + dmp1 + dn2));
      T = scale(cr, complete(C));
    }
    M3<R> U01;
    {
      const M3<R> P = complete(mul2(L(nu, s + dmm1 + dn1), L(mu, s + dmm1)));
      M32<R> C = adj_mul2(P, L(mu, s + dmm1 + dn1));
      U01 = L(mu, s + dn1);
      C = mul2(C, U01);
      axpy(T, cr, complete(C));
    }
    const M32<R> B2 = adj_mul2(H, U01);
    axpy(T, cp, complete(B2));
    {
      M32<R> C = mul2(B2, L(mu, s + dmp1 + dn1));
      C = mul2(C, L(nu, s + dmp2 + dn1));
      C = mul2_adj(C, L(mu, s + dmp1));
      axpy(S, cr, complete(C));
    }
    S = add_mul(S, T, L(nu, s + dmp1 + dn1));
  }
}

template <typename R, bool RECT, int SG>
__device__ __forceinline__ void staple_dir_fast(M3<R>& S, const LinkLd<R>& L, int s, int mu, int nu, int dmm1,
                                                int dmp1, int dmp2, int dn1, int dn2, R cp, R cr)
{
  if (SG > 0) {
    const M3<R> H = L(nu, s);  // hop(x)
    if (!RECT) {
      S = add_mul_adj(S, mul(H, L(mu, s + dn1)), L(nu, s + dmp1));
      return;
    }
    M3<R> T;
    {  // rect1: hop(x) hop(x+e) U_mu(x+2e) back(x+2e+mu)
      M3<R> C = mul(H, L(nu, s + dn1));
      C = mul(C, L(mu, s + dn2));
      C = mul_adj(C, L(nu, s + dmp1 + dn1));
      T = scale(cr, C);
    }
    M3<R> U01;
    {  // rect3: U_mu(x-mu)^+ hop(x-mu) U_mu(x-mu+e) U_mu(x+e)
      M3<R> C = adj_mul(L(mu, s + dmm1), L(nu, s + dmm1));
      C = mul(C, L(mu, s + dmm1 + dn1));
      U01 = L(mu, s + dn1);
      C = mul(C, U01);
      axpy(T, cr, C);
    }
    const M3<R> B = mul(H, U01);
    axpy(T, cp, B);
    {  // rect2: B U_mu(x+e+mu) back(x+e+2mu) U_mu(x+mu)^+
      M3<R> C = mul(B, L(mu, s + dmp1 + dn1));
      C = mul_adj(C, L(nu, s + dmp2));
      C = mul_adj(C, L(mu, s + dmp1));
      axpy(S, cr, C);
    }
    S = add_mul_adj(S, T, L(nu, s + dmp1));
  } else {
    const M3<R> H = L(nu, s + dn1);  // hop(x)^+
    if (!RECT) {
      S = add_mul(S, adj_mul(H, L(mu, s + dn1)), L(nu, s + dmp1 + dn1));
      return;
    }
    M3<R> T;
    {  // rect1: (hop(x+e)^+ hop(x)^+)^+ U_mu(x+2e) back(x+2e+mu)
      M3<R> C = mul(L(nu, s + dn2), H);
      C = adj_mul(C, L(mu, s + dn2));
      C = mul(C, L(nu, s + dmp1 + dn2));
      T = scale(cr, C);
    }
    M3<R> U01;
    {  // rect3: (hop(x-mu)^+ U_mu(x-mu))^+ U_mu(x-mu+e) U_mu(x+e)
      M3<R> C = mul(L(nu, s + dmm1 + dn1), L(mu, s + dmm1));
      C = adj_mul(C, L(mu, s + dmm1 + dn1));
      U01 = L(mu, s + dn1);
      C = mul(C, U01);
      axpy(T, cr, C);
    }
    const M3<R> B = adj_mul(H, U01);
    axpy(T, cp, B);
    {  // rect2
      M3<R> C = mul(B, L(mu, s + dmp1 + dn1));
      C = mul(C, L(nu, s + dmp2 + dn1));
      C = mul_adj(C, L(mu, s + dmp1));
      axpy(S, cr, C);
    }
    S = add_mul(S, T, L(nu, s + dmp1 + dn1));
  }
}

// ------------------------------------------------------------------------
// staples from precomputed two-link products (site map 5, FP32)
//
// A separate pass (k_corners) stores for every site x the double links
// D_a(x) = U_a(x) U_a(x+a) and the corners P_ab(x) = U_a(x) U_b(x+a).  Each
// of the paths of staple_dir_two_row then starts from one of them:
//   e = +nu:  B  = P_numu(x)
//             C1 = D_nu(x) U_mu(x+2nu) U_nu(x+mu+nu)^+
//             C3 = U_mu(x-mu)^+ P_numu(x-mu) U_mu(x+nu)
//             rect2 = B U_mu(x+nu+mu) P_munu(x+mu)^+
//             S += [(1-8c1) B + c1 (C1 + C3)] U_nu(x+mu)^+ + c1 rect2
//   e = -nu:  B' = U_nu(x-nu)^+ U_mu(x-nu)
//             C1 = D_nu(x-2nu)^+ P_munu(x-2nu)
//             C3 = P_numu(x-mu-nu)^+ D_mu(x-mu-nu)
//             rect2 = B' P_munu(x-nu+mu) U_mu(x+mu)^+
//             S += [(1-8c1) B' + c1 (C1 + C3)] U_nu(x+mu-nu) + c1 rect2
// 7 and 6 matrix products per signed direction instead of 11 (the plaquette
// force: 1 instead of 2); the 16 products per site of the pass are shared by
// the links that read them.  The paths are those of hmc.cpp:27-62, only
// grouped differently.
template <typename R, bool RECT, int SG>
__device__ __forceinline__ void staple_dir_corner(M3<R>& S, const LinkLd<R>& L, const LinkLd<R>& Cn, int s, int mu,
                                                  int nu, int dmm1, int dmp1, int dn1, int dn2, R cp, R cr)
{
  const int pnm = corner_id(nu, mu), pmn = corner_id(mu, nu);
  if (SG > 0) {
    const M3<R> B = Cn(pnm, s);
    if (!RECT) {
      S = add_mul_adj(S, B, L(nu, s + dmp1));
      return;
    }
    M3<R> T = scale(cp, B);
    {
      M32<R> C = mul2(Cn(nu, s), L(mu, s + dn2));
      C = mul2_adj(C, L(nu, s + dmp1 + dn1));
      axpy(T, cr, complete(C));
    }
    {
      M32<R> C = adj_mul2(L(mu, s + dmm1), Cn(pnm, s + dmm1));
      C = mul2(C, L(mu, s + dn1));
      axpy(T, cr, complete(C));
    }
    {
      M32<R> C = mul2(B, L(mu, s + dmp1 + dn1));
      C = mul2_adj(C, Cn(pmn, s + dmp1));
      axpy(S, cr, complete(C));
    }
    S = add_mul_adj(S, T, L(nu, s + dmp1));
  } else {
    const M3<R> H = L(nu, s + dn1);
    if (!RECT) {
      S = add_adj_mul(S, H, Cn(pmn, s + dn1));
      return;
    }
    const M32<R> B2 = adj_mul2(H, L(mu, s + dn1));
    M3<R> T = scale(cp, complete(B2));
    {
      const M32<R> C = adj_mul2(Cn(nu, s + dn2), Cn(pmn, s + dn2));
      axpy(T, cr, complete(C));
    }
    {
      const M32<R> C = adj_mul2(Cn(pnm, s + dmm1 + dn1), Cn(mu, s + dmm1 + dn1));
      axpy(T, cr, complete(C));
    }
    {
      M32<R> C = mul2(B2, Cn(pmn, s + dmp1 + dn1));
      C = mul2_adj(C, L(mu, s + dmp1));
      axpy(S, cr, complete(C));
    }
    S = add_mul(S, T, L(nu, s + dmp1 + dn1));
  }
}

// The staple sum of site s (g.off == 0) from the links U and the corner field.
template <typename R, bool RECT>
__device__ __forceinline__ M3<R> staple_sum_corner(const Cx<R>* U, const Cx<R>* corners, const Geo& g, int s, int mu,
                                                   R cp, R cr)
{
  const int nblk = (int)site_blocks(g.V);
  const LinkLd<R> L{U, nblk}, Cn{corners, nblk};
  const Coord x = coord_of(g, s);
  const int st[4] = {1, g.d[0], g.d[0] * g.d[1], g.d[0] * g.d[1] * g.d[2]};
  const int xm = sel4(x.c, mu), Lm = sel4(g.d, mu), sm = sel4(st, mu);
  const int dmm1 = nb_delta(xm, -1, Lm, sm), dmp1 = nb_delta(xm, 1, Lm, sm);
  M3<R> S = m3_zero<R>();
#pragma unroll 1
  for (int i = 1; i < 4; ++i) {
    const int nu = (mu + i) & 3;
    const int xn = sel4(x.c, nu), Ln = sel4(g.d, nu), sn = sel4(st, nu);
    staple_dir_corner<R, RECT, 1>(S, L, Cn, s, mu, nu, dmm1, dmp1, nb_delta(xn, 1, Ln, sn), nb_delta(xn, 2, Ln, sn),
                                  cp, cr);
    staple_dir_corner<R, RECT, -1>(S, L, Cn, s, mu, nu, dmm1, dmp1, nb_delta(xn, -1, Ln, sn),
                                   nb_delta(xn, -2, Ln, sn), cp, cr);
  }
  if (!RECT) S = scale(cp, S);
  return S;
}

// The pass that fills the corner field: one thread per (site, a), block =
// 4 * (site block) + a, storing D_a(x) and P_ab(x) for the three b != a.
// Two-row products completed to SU(3), as the chains of site map 3.
template <typename R>
__global__ void __launch_bounds__(128) k_corners(Geo g, const Cx<R>* __restrict__ U, Cx<R>* __restrict__ C)
{
  const int s = (int)((blockIdx.x >> 2) * 128 + threadIdx.x);
  if (s >= g.V) return;
  const int a = blockIdx.x & 3;
  const int nblk = (int)site_blocks(g.V);
  const LinkLd<R> L{U, nblk};
  const Coord x = coord_of(g, s);
  const int st[4] = {1, g.d[0], g.d[0] * g.d[1], g.d[0] * g.d[1] * g.d[2]};
  const int sa = s + nb_delta(sel4(x.c, a), 1, sel4(g.d, a), sel4(st, a));
  const M3<R> ua = L(a, s);
#pragma unroll 1
  for (int b = 0; b < 4; ++b) {
    const M3<R> p = complete(mul2(ua, L(b, sa)));
    Cx<R>* q = C + (((b == a ? a : corner_id(a, b)) * nblk + (s >> 5)) * 9) * 32 + (s & 31);
#pragma unroll
    for (int k = 0; k < 9; ++k) q[32 * k] = p.e[k];
  }
}


// s: the site's index in the field U (the lattice's sites start at g.off);
// nblk: the field's 32-site blocks (default: those of the lattice alone).
template <typename R, bool RECT, bool TWO>
__device__ __forceinline__ M3<R> staple_sum_fast(const Cx<R>* U, const Geo& g, int s, int mu, R cp, R cr,
                                                 int nblk = -1)
{
  const LinkLd<R> L{U, nblk >= 0 ? nblk : (int)site_blocks(g.V)};
  const Coord x = coord_of(g, s - g.off);
  const int st[4] = {1, g.d[0], g.d[0] * g.d[1], g.d[0] * g.d[1] * g.d[2]};
  const int xm = sel4(x.c, mu), Lm = sel4(g.d, mu), sm = sel4(st, mu);
  const int dmm1 = nb_delta(xm, -1, Lm, sm), dmp1 = nb_delta(xm, 1, Lm, sm), dmp2 = nb_delta(xm, 2, Lm, sm);
  M3<R> S = m3_zero<R>();
#pragma unroll 1
  for (int i = 1; i < 4; ++i) {
    const int nu = (mu + i) & 3;
    const int xn = sel4(x.c, nu), Ln = sel4(g.d, nu), sn = sel4(st, nu);
    if constexpr (TWO) {
      staple_dir_two_row<R, RECT, 1>(S, L, s, mu, nu, dmm1, dmp1, dmp2, nb_delta(xn, 1, Ln, sn),
                                             nb_delta(xn, 2, Ln, sn), cp, cr);
      staple_dir_two_row<R, RECT, -1>(S, L, s, mu, nu, dmm1, dmp1, dmp2, nb_delta(xn, -1, Ln, sn),
                                              nb_delta(xn, -2, Ln, sn), cp, cr);
    } else {
      staple_dir_fast<R, RECT, 1>(S, L, s, mu, nu, dmm1, dmp1, dmp2, nb_delta(xn, 1, Ln, sn),
                                          nb_delta(xn, 2, Ln, sn), cp, cr);
      staple_dir_fast<R, RECT, -1>(S, L, s, mu, nu, dmm1, dmp1, dmp2, nb_delta(xn, -1, Ln, sn),
                                           nb_delta(xn, -2, Ln, sn), cp, cr);
    }
  }
  if (!RECT) S = scale(cp, S);
  return S;
}

// ------------------------------------------------------------------------
// force: F = TA(-beta/3 U_mu(x) S^+) (hmc.cpp:64-75) and its fused consumers

// F = TA(-beta/3 U_mu(x) S^+) (hmc.cpp:64-75) at global site s of a field with
// `stride` sites, then the mode's consumer: store F, P += dt F, or
// U_out = unitarize(exp(eps Z) U) with Z = F or the flow combination a F + b Z'.
template <typename R, int MODE>
__device__ __forceinline__ void force_epilogue(const ForceArgs& a, const CField<R>& U, long stride, long s, int mu,
                                               const M3<R>& S, double beta)
{
  const M3<R> u = U.ld(s, mu);
  M3<R> F = traceless_antiherm(mul_adj(u, S));
  F = scale(R(-beta / 3.0), F);
  if (MODE == FORCE_SET) {
    WField<R>{(Cx<R>*)a.out, stride}.st(s, mu, F);
  } else if (MODE == FORCE_UPDATE || MODE == FORCE_UPDATE_EVOLVE) {
    const WField<R> P{(Cx<R>*)a.out, stride};
    M3<R> p = P.ld(s, mu);
    axpy(p, R(a.dt), F);
    P.st(s, mu, p);
    if (MODE == FORCE_UPDATE_EVOLVE) {
      // the link update that follows the momentum update in the integrators
      // (k_evolve, then k_unitarize<R, double> when ev_unit == 2), on this
      // thread's own link of W (or of U, written to W: the fused leapfrog
      // step, whose next force reads W)
      const WField<R> W{(Cx<R>*)a.ev, stride};
      M3<R> wn = mul(exp_md(scale(R(a.ev_eps), p)), a.ev_from_u ? U.ld(s, mu) : W.ld(s, mu));
      if (a.ev_unit == 1) unitarize(wn);
      else if (a.ev_unit == 2) unitarize_as<double, R>(wn);
      W.st(s, mu, wn);
    }
  } else {
    M3<R> Z = F;
    if (MODE == FORCE_FLOW) {
      Z = scale(R(a.a), F);
      if (a.zp != nullptr && a.b != 0.0) axpy(Z, R(a.b), CField<R>{(const Cx<R>*)a.zp, stride}.ld(s, mu));
      if (a.z != nullptr) WField<R>{(Cx<R>*)a.z, stride}.st(s, mu, Z);
    }
    M3<R> un = mul(exp_md(scale(R(a.dt), Z)), u);
    if (a.unitarize) unitarize(un);
    WField<R>{(Cx<R>*)a.out, stride}.st(s, mu, un);
  }
}

// Launch variants for the autotuner: threads per block, minimum resident
// blocks per SM (caps registers), threads per link (SPLIT = 2 gives each link
// to a lane pair, each doing 3 of the 6 signed directions, combined by a
// shuffle), and the site mapping and staple evaluation: MAP 0 runs blocks of
// consecutive sites (block = 4 * site block + mu) and staple_sum_rt; MAP 1 gives each
// block the four links of a compact tile of BS/4 sites (4 x 2 x 2 x 2 for 128
// threads, 4 x 4 x 2 x 2 for 256), one warp-group per mu, so the four
// directions share the tile's neighbourhood in L1 (it needs the lattice
// extents to be multiples of the tile, otherwise the launcher uses MAP 0);
// MAP 2 is the linear mapping of MAP 0 with staple_sum_fast (per-thread
// neighbour offsets, sign-specialised directions; needs 36 V < 2^31 and
// SPLIT = 1, otherwise MAP 0); MAP 3 is MAP 2 with the two-row SU(3) chains
// (FP32; FP64 runs MAP 2); MAP 5 is MAP 3 with the staples formed from the
// corner field of k_corners (FP32; needs ForceArgs::corners and 144 padded
// sites < 2^31, otherwise MAP 3; FP64 runs MAP 2).
#define QGB_FORCE_VARIANTS(X) \
  X(0, 128, 1, 1, 0)          \
  X(1, 256, 1, 1, 0)          \
  X(2, 128, 1, 2, 0)          \
  X(3, 128, 1, 1, 1)          \
  X(4, 128, 1, 1, 2)          \
  X(5, 256, 1, 1, 2)          \
  X(6, 128, 3, 1, 2)          \
  X(7, 128, 1, 1, 3)          \
  X(8, 256, 1, 1, 3)          \
  X(9, 128, 3, 1, 3)          \
  X(10, 128, 4, 1, 3)         \
  X(11, 128, 5, 1, 3)         \
  X(12, 128, 6, 1, 3)         \
  X(13, 128, 8, 1, 3)         \
  X(14, 128, 4, 1, 5)         \
  X(15, 128, 3, 1, 5)         \
  X(16, 256, 2, 1, 5)
static const int N_FORCE_VARIANTS = 17;

template <int BS>
struct Tile {
  static const int tx = 4, ty = BS >= 256 ? 4 : 2, tz = 2, tt = BS >= 256 ? 2 : (BS >= 128 ? 2 : 1);
  static const int sites = tx * ty * tz * tt;
};

template <typename R, int MODE, bool RECT, int BS, int MINB, int SPLIT, int MAP>
__global__ void __launch_bounds__(BS, MINB) k_force(Geo g, ForceArgs a)
{
  const R cp = R(1.0 - 8.0 * a.c1), cr = R(a.c1);
  // linear maps: block b = 4 * (site block) + mu, so the four directions of a
  // site block run back to back and share its neighbourhood in L2 (a grid
  // that sweeps the lattice once per direction reads the link field from DRAM
  // four times when it exceeds L2)
  if constexpr (MAP >= 2) {
    const long w = (long)(blockIdx.x >> 2) * BS + threadIdx.x;
    if (w >= work_sites(g)) return;
    const long t = site_of_work(g, w, BS);
    const int mu = blockIdx.x & 3;
    M3<R> S;
    if constexpr (MAP == 5)
      S = staple_sum_corner<R, RECT>((const Cx<R>*)a.U, (const Cx<R>*)a.corners, g, (int)t, mu, cp, cr);
    else
      S = staple_sum_fast<R, RECT, MAP == 3>((const Cx<R>*)a.U, g, (int)t, mu, cp, cr);
    force_epilogue<R, MODE>(a, CField<R>{(const Cx<R>*)a.U, g.V}, g.V, t, mu, S, a.beta);
    return;
  }
  long s0;
  int h, mu;
  if (MAP == 0) {
    const long t = (long)(blockIdx.x >> 2) * BS + threadIdx.x;
    s0 = t / SPLIT;
    h = (int)(t % SPLIT);
    mu = blockIdx.x & 3;
  } else {
    // tile of Tile<BS>::sites sites; thread = mu * sites + site-in-tile
    using TL = Tile<BS>;
    const int in = threadIdx.x % TL::sites;
    mu = threadIdx.x / TL::sites;
    h = 0;
    long b = blockIdx.x;
    const int nx = g.d[0] / TL::tx, ny = g.d[1] / TL::ty, nz = g.d[2] / TL::tz;
    const int bx = (int)(b % nx);
    b /= nx;
    const int by = (int)(b % ny);
    b /= ny;
    const int bz = (int)(b % nz);
    const int bt = (int)(b / nz);
    const int x0 = bx * TL::tx + in % TL::tx;
    const int x1 = by * TL::ty + (in / TL::tx) % TL::ty;
    const int x2 = bz * TL::tz + (in / (TL::tx * TL::ty)) % TL::tz;
    const int x3 = bt * TL::tt + in / (TL::tx * TL::ty * TL::tz);
    s0 = (long)x0 + (long)g.d[0] * ((long)x1 + (long)g.d[1] * ((long)x2 + (long)g.d[2] * (long)x3));
  }
  if (SPLIT == 1 && s0 >= g.V) return;
  const bool valid = s0 < g.V;  // lane pairs stay together for the shuffle
  const long s = valid ? s0 : g.V - 1;
  const CField<R> U{(const Cx<R>*)a.U, g.V};
  const Coord x = coord_of(g, s);
  M3<R> S = staple_sum_rt<R, RECT>(U, g, x, mu, cp, cr, h * (6 / SPLIT), (h + 1) * (6 / SPLIT));
  if (SPLIT == 2) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      S.e[i].re += __shfl_xor_sync(0xffffffffu, S.e[i].re, 1);
      S.e[i].im += __shfl_xor_sync(0xffffffffu, S.e[i].im, 1);
    }
    if (!valid || h != 0) return;
  }
  force_epilogue<R, MODE>(a, U, g.V, s, mu, S, a.beta);
}

template <typename R, int BS, int MINB, int SPLIT, int MAP>
cudaError_t launch_force_v(const Geo& g, ForceMode mode, const ForceArgs& a, cudaStream_t st)
{
  if constexpr ((MAP == 3 || MAP == 5) && sizeof(R) == 8) {
    return launch_force_v<R, BS, MINB, SPLIT, 2>(g, mode, a, st);
  } else {
  // site map 5 reads the corner field that launch_corners filled from a.U
  if (MAP == 5 && !(a.corners && g.off == 0 && padded_sites(g.V) * 144 < 2147483647L))
    return launch_force_v<R, BS, MINB, SPLIT, 3>(g, mode, a, st);
  using TL = Tile<BS>;
  const bool tiled = MAP == 1 && SPLIT == 1 && g.d[0] % TL::tx == 0 && g.d[1] % TL::ty == 0 &&
                     g.d[2] % TL::tz == 0 && g.d[3] % TL::tt == 0;
  if (MAP == 1 && !tiled) return launch_force_v<R, BS, MINB, SPLIT, 0>(g, mode, a, st);
  const bool fast = MAP >= 2 && SPLIT == 1 && g.off == 0 && padded_sites(g.V) * 36 < 2147483647L;
  if (MAP >= 2 && !fast) return launch_force_v<R, BS, MINB, SPLIT, 0>(g, mode, a, st);
  // the linear maps run over the owned sites of a domain only (the others are halo copies)
  const long nw = MAP >= 2 ? work_sites(g) : g.V;
  dim3 grid = tiled ? dim3((unsigned)(g.V / TL::sites), 1) : dim3((unsigned)(4 * ((nw * SPLIT + BS - 1) / BS)), 1);
  Geo gk = g;  // the linear maps traverse large lattices in z slabs
  if (MAP >= 2) set_slab_order(gk, BS, (int)(18 * sizeof(R)));
  const bool rect = a.c1 != 0.0;
#define QGB_LAUNCH(M)                                                                                  \
  if (rect) k_force<R, M, true, BS, MINB, SPLIT, MAP><<<grid, BS, 0, st>>>(gk, a); \
  else k_force<R, M, false, BS, MINB, SPLIT, MAP><<<grid, BS, 0, st>>>(gk, a);
  switch (mode) {
    case FORCE_SET: QGB_LAUNCH(FORCE_SET) break;
    case FORCE_UPDATE: QGB_LAUNCH(FORCE_UPDATE) break;
    case FORCE_EVOLVE: QGB_LAUNCH(FORCE_EVOLVE) break;
    case FORCE_FLOW: QGB_LAUNCH(FORCE_FLOW) break;
    case FORCE_UPDATE_EVOLVE: QGB_LAUNCH(FORCE_UPDATE_EVOLVE) break;
  }
#undef QGB_LAUNCH
  return cudaGetLastError();
  }
}

// The corner field of site map 5 for the links U (g.off == 0; C holds
// N_CORNER_FIELDS color matrices per padded site).
template <typename R>
cudaError_t launch_corners(const Geo& g, const void* U, void* C, cudaStream_t st)
{
  k_corners<R><<<(unsigned)(4 * ((g.V + 127) / 128)), 128, 0, st>>>(g, (const Cx<R>*)U, (Cx<R>*)C);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_force(const Geo& g, ForceMode mode, const ForceArgs& a, int variant, cudaStream_t st)
{
  switch (variant) {
#define QGB_V(ID, BS, MINB, SPLIT, MAP) \
  case ID: return launch_force_v<R, BS, MINB, SPLIT, MAP>(g, mode, a, st);
    QGB_FORCE_VARIANTS(QGB_V)
#undef QGB_V
    default: return cudaErrorInvalidValue;
  }
}

inline int force_variant_info(int variant, int* bs, int* minb, int* split, int* map)
{
  switch (variant) {
#define QGB_V(ID, BS, MINB, SPLIT, MAP) \
  case ID: *bs = BS; *minb = MINB; *split = SPLIT; *map = MAP; return 1;
    QGB_FORCE_VARIANTS(QGB_V)
#undef QGB_V
    default: return 0;
  }
}

// Batched force: every chain of a batch in one launch, one thread per link of
// the concatenated field (Vtot sites, block = 4 * site block + mu).  Each thread finds its
// chain by binary search over the chain offsets and uses that chain's lattice,
// beta and c1.  RECT is set when any chain has c1 != 0 (Wilson chains then add
// rectangle terms with weight 0).  FAST: the staple sum of the single-lattice
// kernel's fastest form (per-direction neighbour offsets within the chain's
// lattice, two-row chains in FP32; 32-bit link offsets, so the launcher uses
// it while 36 padded sites < 2^31), with that form's register budget.
template <typename R, bool RECT>
constexpr int batch_min_blocks()
{
  return sizeof(R) == 4 ? (RECT ? 4 : 8) : (RECT ? 1 : 3);
}

// Launch shapes of the batched force for the batch autotuner
// (qgb_batch_autotune): block size and minimum resident blocks per SM
// relative to the single-lattice register budget D = batch_min_blocks:
//   0: 128 threads, D     1: 256 threads, max(1, D / 2)
//   2: 128 threads, D + 1 (fewer registers, more warps)
//   3: 64 threads, 2 D    (smaller blocks, finer tail)
static const int N_BATCH_FORCE_VARIANTS = 4;

template <typename R, bool RECT, int VAR>
constexpr int batch_bs()
{
  return VAR == 1 ? 256 : (VAR == 3 ? 64 : 128);
}

template <typename R, bool RECT, int VAR>
constexpr int batch_minb()
{
  return VAR == 0 ? batch_min_blocks<R, RECT>()
                  : VAR == 1 ? (batch_min_blocks<R, RECT>() / 2 > 0 ? batch_min_blocks<R, RECT>() / 2 : 1)
                             : VAR == 2 ? batch_min_blocks<R, RECT>() + 1 : 2 * batch_min_blocks<R, RECT>();
}

template <typename R, int MODE, bool RECT, bool FAST, int VAR>
__global__ void __launch_bounds__(batch_bs<R, RECT, VAR>(), FAST ? batch_minb<R, RECT, VAR>() : 1)
    k_force_batch(long Vtot, int nchain, const long* __restrict__ offs, const ChainInfo* __restrict__ chains,
                  ForceArgs a)
{
  constexpr int BS = batch_bs<R, RECT, VAR>();
  const long sg = (long)(blockIdx.x >> 2) * BS + threadIdx.x;  // block = 4 * (site block) + mu
  if (sg >= Vtot) return;
  const int c = chain_of(offs, nchain, sg);
  const ChainInfo ci = chains[c];
  const Geo g = chain_geo(ci);
  const int mu = blockIdx.x & 3;
  const CField<R> U{(const Cx<R>*)a.U, Vtot};
  const R cp = R(1.0 - 8.0 * ci.c1), cr = R(ci.c1);
  M3<R> S;
  if constexpr (FAST) {
    S = staple_sum_fast<R, RECT, sizeof(R) == 4>((const Cx<R>*)a.U, g, (int)sg, mu, cp, cr, (int)site_blocks(Vtot));
  } else {
    const Coord x = coord_of(g, sg - ci.off);
    S = staple_sum_rt<R, RECT>(U, g, x, mu, cp, cr, 0, 6);
  }
  force_epilogue<R, MODE>(a, U, Vtot, sg, mu, S, ci.beta);
}

template <typename R, int VAR>
cudaError_t launch_force_batch_v(long Vtot, int nchain, const long* offs, const ChainInfo* chains, bool rect,
                                 ForceMode mode, const ForceArgs& a, cudaStream_t st)
{
  const bool fast = padded_sites(Vtot) * 36 < 2147483647L;
  if (!fast && VAR != 0) return launch_force_batch_v<R, 0>(Vtot, nchain, offs, chains, rect, mode, a, st);
  constexpr int BT = batch_bs<R, true, VAR>(), BF = batch_bs<R, false, VAR>();
  const dim3 gt((unsigned)(4 * ((Vtot + BT - 1) / BT))), gf((unsigned)(4 * ((Vtot + BF - 1) / BF)));
#define QGB_LAUNCH(M)                                                                                         \
  if (fast) {                                                                                                 \
    if (rect) k_force_batch<R, M, true, true, VAR><<<gt, BT, 0, st>>>(Vtot, nchain, offs, chains, a);         \
    else k_force_batch<R, M, false, true, VAR><<<gf, BF, 0, st>>>(Vtot, nchain, offs, chains, a);             \
  } else {                                                                                                    \
    if (rect) k_force_batch<R, M, true, false, 0><<<gt, BT, 0, st>>>(Vtot, nchain, offs, chains, a);          \
    else k_force_batch<R, M, false, false, 0><<<gf, BF, 0, st>>>(Vtot, nchain, offs, chains, a);              \
  }
  switch (mode) {
    case FORCE_SET: QGB_LAUNCH(FORCE_SET) break;
    case FORCE_UPDATE: QGB_LAUNCH(FORCE_UPDATE) break;
    case FORCE_EVOLVE: QGB_LAUNCH(FORCE_EVOLVE) break;
    case FORCE_FLOW: QGB_LAUNCH(FORCE_FLOW) break;
    case FORCE_UPDATE_EVOLVE: QGB_LAUNCH(FORCE_UPDATE_EVOLVE) break;
  }
#undef QGB_LAUNCH
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_force_batch(long Vtot, int nchain, const long* offs, const ChainInfo* chains, bool rect,
                               ForceMode mode, const ForceArgs& a, cudaStream_t st, int variant)
{
  switch (variant) {
    case 0: return launch_force_batch_v<R, 0>(Vtot, nchain, offs, chains, rect, mode, a, st);
    case 1: return launch_force_batch_v<R, 1>(Vtot, nchain, offs, chains, rect, mode, a, st);
    case 2: return launch_force_batch_v<R, 2>(Vtot, nchain, offs, chains, rect, mode, a, st);
    case 3: return launch_force_batch_v<R, 3>(Vtot, nchain, offs, chains, rect, mode, a, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace qgb
