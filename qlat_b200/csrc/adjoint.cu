// adjoint.cu -- reverse-mode derivative (VJP) of the gradient flow.
//
// Conventions.  A tangent or cotangent at a gauge field is an su(3) field X
// (traceless anti-Hermitian per link) acting by left multiplication,
// U -> exp(s X) U.  In the basis T_a of matrix-hmc.h:76-106 (tr T_a T_b =
// -2 delta_ab) the pairing is <X, Y> = sum_a X^a Y^a = -tr(X Y)/2, and the
// gradient of a function L is the su(3) field sum_a (dL/domega_a) T_a.
// (Qlattice's force set_gm_force is -1/2 of the action's gradient in this
// convention, since its kinetic term is sum_a p_a^2.)
//
// One flow stage W' = exp(eps Z) W with Z = a F(W) + b Z_prev pulls a
// cotangent lambda' at W' back to
//   lambda = Ad_{exp(-eps Z)} lambda' + a DF(W)^T mu,   mu = eps dexp_{-eps Z}(lambda') [+ carry],
// with dexp_A(B) = sum_k ad_A^k B / (k+1)! and a carry b mu to the previous
// stage's Z.  The transpose of the force Jacobian on the group is
// DF^T[Y] = DF[Y] + [F, Y]: the Hessian of the action is symmetric up to the
// commutator term of non-commuting left derivatives.  DF[Y] is evaluated in
// forward mode: every link U of the staple paths carries its tangent Y U.
// The forward exponential is the order-20 polynomial; its derivative is taken
// as that of the exact exponential (the difference is below rounding for the
// flow's step sizes).
#include <cuda_runtime.h>

#include "gauge_common.cuh"
#include "kernels.h"
#include "su3.cuh"

namespace qgb
{

template <typename R>
struct Dual {
  M3<R> v, d;  // value and tangent
};

template <typename R>
__device__ __forceinline__ Dual<R> dmul(const Dual<R>& a, const Dual<R>& b)
{
  Dual<R> r;
  r.v = mul(a.v, b.v);
  r.d = add_mul(mul(a.d, b.v), a.v, b.d);
  return r;
}

// link (site, dir) with tangent Y(site, dir) U(site, dir), optionally its adjoint
// (the tangent of U^+ is (Y U)^+ = -U^+ Y).
template <typename R>
__device__ __forceinline__ Dual<R> dlink(const CField<R>& U, const CField<R>& Y, long site, int dir, bool dagger)
{
  const M3<R> u = U.ld(site, dir);
  const M3<R> y = Y.ld(site, dir);
  Dual<R> r;
  if (!dagger) {
    r.v = u;
    r.d = mul(y, u);
  } else {
    r.v = adj(u);
    r.d = scale(R(-1), mul(r.v, y));
  }
  return r;
}

// [A, B]
template <typename R>
__device__ __forceinline__ M3<R> commutator(const M3<R>& a, const M3<R>& b)
{
  M3<R> r = mul(a, b);
  const M3<R> t = mul(b, a);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    r.e[i].re -= t.e[i].re;
    r.e[i].im -= t.e[i].im;
  }
  return r;
}

// The links of the staple paths at signed direction e = s nu as dual
// matrices (positions x + a mu + b e, as SignedDir in force_impl.cuh): hop is
// the link from there along +e, back the one along -e, umu U_mu there.
template <typename R>
struct DualDir {
  const CField<R>& U;
  const CField<R>& Y;
  const Geo& g;
  const Coord& x;
  int mu, nu, s;
  __device__ __forceinline__ Dual<R> umu(int a, int b, bool dagger = false) const
  {
    return dlink(U, Y, site_rt(g, x, mu, a, nu, b * s), mu, dagger);
  }
  __device__ __forceinline__ Dual<R> hop(int a, int b) const
  {
    return dlink(U, Y, site_rt(g, x, mu, a, nu, b * s + (s < 0 ? -1 : 0)), nu, s < 0);
  }
  __device__ __forceinline__ Dual<R> back(int a, int b) const
  {
    return dlink(U, Y, site_rt(g, x, mu, a, nu, b * s + (s < 0 ? 0 : -1)), nu, s > 0);
  }
};

template <typename R>
__device__ __forceinline__ void dual_acc(M3<R>& S, M3<R>& dS, R w, const Dual<R>& P)
{
  axpy(S, w, P.v);
  axpy(dS, w, P.d);
}

// The staple sums S and dS of a thread, kept in shared memory (entry k at
// [k][threadIdx.x]) while its paths are walked: the dual matrices of a path
// then have the registers to themselves.
template <typename R>
struct SmemAcc {
  Cx<R> (*s)[128];
  Cx<R> (*ds)[128];
  __device__ __forceinline__ void zero()
  {
#pragma unroll
    for (int k = 0; k < 9; ++k) s[k][threadIdx.x] = ds[k][threadIdx.x] = cx<R>(R(0), R(0));
  }
  __device__ __forceinline__ void add(R w, const Dual<R>& P)
  {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      Cx<R> a = s[k][threadIdx.x], b = ds[k][threadIdx.x];
      a.re = fma(w, P.v.e[k].re, a.re);
      a.im = fma(w, P.v.e[k].im, a.im);
      b.re = fma(w, P.d.e[k].re, b.re);
      b.im = fma(w, P.d.e[k].im, b.im);
      s[k][threadIdx.x] = a;
      ds[k][threadIdx.x] = b;
    }
  }
  __device__ __forceinline__ M3<R> S() const
  {
    M3<R> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k] = s[k][threadIdx.x];
    return m;
  }
  __device__ __forceinline__ M3<R> dS() const
  {
    M3<R> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k] = ds[k][threadIdx.x];
    return m;
  }
};

// lambda_out = lambda_local + a (DF[Y] + [F, Y]) at every link, F the force
// of GaugeAction(beta, c1) (hmc.cpp:48-75: staples (1 - 8 c1) plaq + c1 rect,
// the paths of hmc.cpp:27-46), DF[Y] its derivative along Y, every path
// walked as a product of dual matrices.
template <typename R, bool RECT>
__global__ void __launch_bounds__(128) k_force_vjp(Geo g, const Cx<R>* Up, const Cx<R>* Yp, const Cx<R>* lam_local,
                                                   Cx<R>* lam_out, double beta, double c1, double a)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int mu = blockIdx.y;
  const CField<R> U{Up, g.V}, Y{Yp, g.V};
  const Coord x = coord_of(g, s);
  const R cp = R(1.0 - 8.0 * c1), cr = R(c1);
  __shared__ Cx<R> sh_s[9][128], sh_ds[9][128];
  SmemAcc<R> acc{sh_s, sh_ds};
  acc.zero();
#pragma unroll 1
  for (int k = 0; k < 6; ++k) {
    const DualDir<R> d{U, Y, g, x, mu, (mu + 1 + (k >> 1)) & 3, (k & 1) ? -1 : 1};
    // plaq (nu, mu, -nu) = hop(x) U_mu(x+e) back(x+e+mu)
    acc.add(cp, dmul(dmul(d.hop(0, 0), d.umu(0, 1)), d.back(1, 1)));
    if (RECT) {
      // rect1 (nu, nu, mu, -nu, -nu)
      Dual<R> C = dmul(d.hop(0, 0), d.hop(0, 1));
      C = dmul(C, d.umu(0, 2));
      C = dmul(C, d.back(1, 2));
      acc.add(cr, dmul(C, d.back(1, 1)));
      // rect2 (nu, mu, mu, -nu, -mu)
      C = dmul(d.hop(0, 0), d.umu(0, 1));
      C = dmul(C, d.umu(1, 1));
      C = dmul(C, d.back(2, 1));
      acc.add(cr, dmul(C, d.umu(1, 0, true)));
      // rect3 (-mu, nu, mu, mu, -nu)
      C = dmul(d.umu(-1, 0, true), d.hop(-1, 0));
      C = dmul(C, d.umu(-1, 1));
      C = dmul(C, d.umu(0, 1));
      acc.add(cr, dmul(C, d.back(1, 1)));
    }
  }
  const M3<R> S = acc.S(), dS = acc.dS();
  const M3<R> u = U.ld(s, mu);
  const M3<R> y = Y.ld(s, mu);
  const M3<R> du = mul(y, u);
  const R c = R(-beta / 3.0);
  const M3<R> F = scale(c, traceless_antiherm(mul_adj(u, S)));
  const M3<R> dF = scale(c, traceless_antiherm(add_mul(mul_adj(du, S), u, adj(dS))));
  M3<R> out = CField<R>{lam_local, g.V}.ld(s, mu);
  axpy(out, R(a), dF);
  axpy(out, R(a), commutator(F, y));
  WField<R>{lam_out, g.V}.st(s, mu, traceless_antiherm(out));
}

template <typename R>
__device__ __forceinline__ M3<R> add_to_copy(M3<R> a, const M3<R>& b)
{
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    a.e[i].re += b.e[i].re;
    a.e[i].im += b.e[i].im;
  }
  return a;
}

// dexp_A(B) = sum_{k>=0} ad_A^k B / (k+1)!
template <typename R>
__device__ __forceinline__ M3<R> dexp_apply(const M3<R>& A, const M3<R>& B)
{
  M3<R> out = B, term = B;
#pragma unroll 1
  for (int k = 1; k <= 16; ++k) {
    term = scale(R(1) / R(k + 1), commutator(A, term));
    add_to(out, term);
  }
  return out;
}

// Link-local part of a stage's pull-back:
//   mu_out = eps dexp_{-eps Z}(lambda) + carry * mu_carry,   lam_local = e^{-eps Z} lambda e^{eps Z}.
template <typename R>
__global__ void __launch_bounds__(128) k_flow_adj_local(long V, const Cx<R>* lam, const Cx<R>* Z, const Cx<R>* mu_carry,
                                                        double carry, double eps, Cx<R>* mu_out, Cx<R>* lam_local)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  const M3<R> l = CField<R>{lam, V}.ld(s, mu);
  const M3<R> A = scale(R(-eps), CField<R>{Z, V}.ld(s, mu));
  // Both parts from one series of nested commutators c_k = ad_A^k lambda:
  // dexp_A(lambda) = sum_k c_k / (k+1)! and e^A lambda e^-A = sum_k c_k / k!,
  // cut once |c_k| / k! (Frobenius norms, |ad_A| <= 2 |A|) falls below
  // 2^-60 |lambda| (2^-30 in FP32), under the rounding of either sum.
  R na2 = R(0), nl2 = R(0);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    na2 = fma(A.e[i].re, A.e[i].re, fma(A.e[i].im, A.e[i].im, na2));
    nl2 = fma(l.e[i].re, l.e[i].re, fma(l.e[i].im, l.e[i].im, nl2));
  }
  const R nad = R(2) * sqrt(na2);
  const R tol = (sizeof(R) == 4 ? R(9.313225746154785e-10) : R(8.673617379884035e-19)) * sqrt(nl2);
  M3<R> d = l, ad = l, c = l;
  R bound = sqrt(nl2);  // bound on |c_k| / k!
#pragma unroll 1
  for (int k = 1; k <= 30 && bound > tol; ++k) {
    c = scale(R(1) / R(k), commutator(A, c));  // c_k / k!
    ad = add_to_copy(ad, c);
    d = add_to_copy(d, scale(R(1) / R(k + 1), c));
    bound *= nad / R(k);
  }
  M3<R> m = scale(R(eps), d);
  if (mu_carry != nullptr && carry != 0.0) axpy(m, R(carry), CField<R>{mu_carry, V}.ld(s, mu));
  WField<R>{mu_out, V}.st(s, mu, traceless_antiherm(m));
  WField<R>{lam_local, V}.st(s, mu, traceless_antiherm(ad));
}

// out = dexp_{-Omega}(lambda): the gradient with respect to omega of a function
// of exp(Omega) U, given its left-trivialised gradient lambda at exp(Omega) U.
template <typename R>
__global__ void k_dexp_adjoint(long V, int m, const Cx<R>* omega, const Cx<R>* lam, Cx<R>* out)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int mu = 0; mu < m; ++mu) {
    const M3<R> A = scale(R(-1), CField<R>{omega, V}.ld(s, mu));
    WField<R>{out, V}.st(s, mu, traceless_antiherm(dexp_apply(A, CField<R>{lam, V}.ld(s, mu))));
  }
}

// fc[x, m] = sum_a T_a basis[x, 8 m + a] and back (hmc.cpp:647-697,
// matrix-hmc.h:76-123); basis is a real field with multiplicity 8 m.
template <typename R>
__global__ void k_basis_to_matrix(long V, int m, const R* basis, Cx<R>* fc)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int mu = 0; mu < m; ++mu) {
    R b[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) b[a] = basis[lay_index<1>(V, 8 * mu + a, 0, s)];
    const R s3 = R(0.57735026918962584) * b[7];
    M3<R> r;
    r.e[0] = cx<R>(R(0), b[2] + s3);
    r.e[4] = cx<R>(R(0), -b[2] + s3);
    r.e[8] = cx<R>(R(0), R(-2) * s3);
    r.e[1] = cx<R>(b[1], b[0]);
    r.e[2] = cx<R>(b[4], b[3]);
    r.e[3] = cx<R>(-b[1], b[0]);
    r.e[5] = cx<R>(b[6], b[5]);
    r.e[6] = cx<R>(-b[4], b[3]);
    r.e[7] = cx<R>(-b[6], b[5]);
    WField<R>{fc, V}.st(s, mu, r);
  }
}

template <typename R>
__global__ void k_matrix_to_basis(long V, int m, const Cx<R>* fc, R* basis)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int mu = 0; mu < m; ++mu) {
    const M3<R> x = CField<R>{fc, V}.ld(s, mu);
    R b[8];
    b[0] = x.e[1].im;
    b[1] = x.e[1].re;
    b[2] = R(0.5) * (x.e[0].im - x.e[4].im);
    b[3] = x.e[2].im;
    b[4] = x.e[2].re;
    b[5] = x.e[5].im;
    b[6] = x.e[5].re;
    b[7] = R(0.86602540378443865) * (x.e[0].im + x.e[4].im);
#pragma unroll
    for (int a = 0; a < 8; ++a) basis[lay_index<1>(V, 8 * mu + a, 0, s)] = b[a];
  }
}

template <typename R>
cudaError_t launch_force_vjp(const Geo& g, const void* U, const void* Y, const void* lam_local, void* lam_out,
                             double beta, double c1, double a, cudaStream_t st)
{
  dim3 grid((unsigned)((g.V + 127) / 128), 4);
  if (c1 != 0.0)
    k_force_vjp<R, true><<<grid, 128, 0, st>>>(g, (const Cx<R>*)U, (const Cx<R>*)Y, (const Cx<R>*)lam_local,
                                               (Cx<R>*)lam_out, beta, c1, a);
  else
    k_force_vjp<R, false><<<grid, 128, 0, st>>>(g, (const Cx<R>*)U, (const Cx<R>*)Y, (const Cx<R>*)lam_local,
                                                (Cx<R>*)lam_out, beta, 0.0, a);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_flow_adj_local(long V, const void* lam, const void* Z, const void* mu_carry, double carry, double eps,
                                  void* mu_out, void* lam_local, cudaStream_t st)
{
  dim3 grid((unsigned)((V + 127) / 128), 4);
  k_flow_adj_local<R><<<grid, 128, 0, st>>>(V, (const Cx<R>*)lam, (const Cx<R>*)Z, (const Cx<R>*)mu_carry, carry, eps,
                                            (Cx<R>*)mu_out, (Cx<R>*)lam_local);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_dexp_adjoint(long V, int m, const void* omega, const void* lam, void* out, cudaStream_t st)
{
  k_dexp_adjoint<R><<<(unsigned)((V + 127) / 128), 128, 0, st>>>(V, m, (const Cx<R>*)omega, (const Cx<R>*)lam,
                                                                 (Cx<R>*)out);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_basis_to_matrix(long V, int m, const void* basis, void* fc, cudaStream_t st)
{
  k_basis_to_matrix<R><<<(unsigned)((V + 127) / 128), 128, 0, st>>>(V, m, (const R*)basis, (Cx<R>*)fc);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_matrix_to_basis(long V, int m, const void* fc, void* basis, cudaStream_t st)
{
  k_matrix_to_basis<R><<<(unsigned)((V + 127) / 128), 128, 0, st>>>(V, m, (const Cx<R>*)fc, (R*)basis);
  return cudaGetLastError();
}

#define QGB_ADJ_INST(R)                                                                                          \
  template cudaError_t launch_force_vjp<R>(const Geo&, const void*, const void*, const void*, void*, double, double, \
                                           double, cudaStream_t);                                               \
  template cudaError_t launch_flow_adj_local<R>(long, const void*, const void*, const void*, double, double, void*, \
                                                void*, cudaStream_t);                                           \
  template cudaError_t launch_dexp_adjoint<R>(long, int, const void*, const void*, void*, cudaStream_t);        \
  template cudaError_t launch_basis_to_matrix<R>(long, int, const void*, void*, cudaStream_t);                  \
  template cudaError_t launch_matrix_to_basis<R>(long, int, const void*, void*, cudaStream_t);
QGB_ADJ_INST(double)
QGB_ADJ_INST(float)

}  // namespace qgb
