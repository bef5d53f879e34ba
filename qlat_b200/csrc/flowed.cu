// flowed.cu -- flowed HMC with masked invertible flows (the reference's
// flowed-hmc.cpp / flowed-hmc.h), FP64 on the GPU.
//
// A flow is a list of steps (mask, mu, epsilon, flow_size).  A step updates
// the links U_mu(x) of the sites x of one mask -- even/odd sites for
// flow_size 1, even/odd 2^4 blocks for flow_size 2 -- by
//   U_mu(x) <- exp(-eps TA(U_mu(x) C(x)^+)) U_mu(x)        (exp unitarized)
// with C the plaquette staple (flow_size 1) or the staple of the rectangles
// whose short edge is the link (flow_size 2).  No updated link enters another
// updated link's staple, so a step is invertible link by link (50
// fixed-point iterations) and its Jacobian is block diagonal: per flowed link
// the 8 x 8 matrix M' = 1 - eps J(X) N in the su(3) basis, J the differential
// of exp at X = -eps TA(U C^+) and N the derivative of TA(U C^+) with respect
// to the link.  The flowed-HMC action is S(flow(U)) - sum ln det M', and its
// force is propagated back through the steps (the transpose of each step's
// Jacobian) with the force of the log-determinants added at each step.
//
// Layout: one thread per site.  The staple of the flowed links goes to a
// color-matrix field of multiplicity 1; per flowed link, a per-step table
// (exp(ad X), J(-ad X), the 8 traces of the determinant force and
// (-eps) M'^-1 J(X)) feeds the per-site pass over the (link, flowed link)
// pairs of the reference's set_xl_nu_from_mask_mu_yl_m.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/qlat_b200.h"
#include "gauge_common.cuh"
#include "kernels.h"

namespace qgb
{
void set_last_error(const std::string& msg);
void* field_data(const qgb_field* f);
int library_stream(cudaStream_t* st);
}

namespace
{
using namespace qgb;

// ---- su(3) basis (matrix-hmc.h:76-124) and 8 x 8 real matrices -------------

struct A8 {
  double m[64];  // row-major: (a, b) at m[8 a + b]
};

__constant__ double c_ts[8][18];  // T_a = make_anti_hermitian_matrix(e_a)
__constant__ double c_f[8][64];   // f[c](a, b) = basis_c(T_a T_b - T_b T_a)

__host__ __device__ inline M3<double> anti_herm_from_basis(const double* b)
{
  // make_anti_hermitian_matrix (matrix-hmc.h:76-106)
  const double s3 = (1.0 / sqrt(3.0)) * b[7];
  M3<double> m;
  m.e[0] = cx<double>(0.0, b[2] + s3);
  m.e[1] = cx<double>(b[1], b[0]);
  m.e[2] = cx<double>(b[4], b[3]);
  m.e[3] = cx<double>(-b[1], b[0]);
  m.e[4] = cx<double>(0.0, -b[2] + s3);
  m.e[5] = cx<double>(b[6], b[5]);
  m.e[6] = cx<double>(-b[4], b[3]);
  m.e[7] = cx<double>(-b[6], b[5]);
  m.e[8] = cx<double>(0.0, -2.0 * s3);
  return m;
}

__host__ __device__ inline void basis_of(const M3<double>& m, double* b)
{
  // basis_projection_anti_hermitian_matrix (matrix-hmc.h:108-124)
  b[0] = m.e[1].im;
  b[1] = m.e[1].re;
  b[2] = 0.5 * (m.e[0].im - m.e[4].im);
  b[3] = m.e[2].im;
  b[4] = m.e[2].re;
  b[5] = m.e[5].im;
  b[6] = m.e[5].re;
  b[7] = sqrt(3.0) * 0.5 * (m.e[0].im + m.e[4].im);
}

__device__ inline M3<double> ts(int a)
{
  M3<double> t;
#pragma unroll
  for (int k = 0; k < 9; ++k) t.e[k] = cx<double>(c_ts[a][2 * k], c_ts[a][2 * k + 1]);
  return t;
}

__device__ inline void a8_mul(A8& r, const A8& x, const A8& y)
{
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      double s = 0.0;
      for (int k = 0; k < 8; ++k) s += x.m[8 * i + k] * y.m[8 * k + j];
      r.m[8 * i + j] = s;
    }
}

__device__ inline void a8_scale(A8& r, double s, const A8& x)
{
  for (int i = 0; i < 64; ++i) r.m[i] = s * x.m[i];
}

// make_adjoint_representation (matrix-hmc.h:294-306): sum_a (-basis_a(m)) f[a]
__device__ inline void adjoint_rep(A8& am, const M3<double>& m)
{
  double b[8];
  basis_of(m, b);
  for (int i = 0; i < 64; ++i) am.m[i] = 0.0;
  for (int a = 0; a < 8; ++a)
    for (int i = 0; i < 64; ++i) am.m[i] += (-b[a]) * c_f[a][i];
}

// make_matrix_exp (matrix-hmc.h:155-167) for 8 x 8: order-20 Horner
__device__ inline void a8_exp(A8& r, const A8& a)
{
  A8 t2 = a, t3;
  for (int j = 20; j > 1; --j) {
    for (int i = 0; i < 64; ++i) t3.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) + (1.0 / j) * t2.m[i];
    a8_mul(t2, a, t3);
  }
  for (int i = 0; i < 64; ++i) r.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) + t2.m[i];
}

// make_diff_exp_map (matrix-hmc.h:308-321): sum_k (-am)^k / (k+1)!, order 20
__device__ inline void dexp_map(A8& r, const A8& am)
{
  A8 t2, t3;
  for (int i = 0; i < 64; ++i) t2.m[i] = -am.m[i];
  for (int j = 20; j > 1; --j) {
    for (int i = 0; i < 64; ++i) t3.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) + (1.0 / (j + 1)) * t2.m[i];
    A8 nam;
    for (int i = 0; i < 64; ++i) nam.m[i] = -am.m[i];
    a8_mul(t2, nam, t3);
  }
  for (int i = 0; i < 64; ++i) r.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) + 0.5 * t2.m[i];
}

// make_diff_exp_map_diff (matrix-hmc.h:341-362): derivative of dexp_map(am)
// along f[a]
__device__ inline void dexp_map_diff(A8& r, const A8& am, int a)
{
  A8 t2, dt2, t3, dt3, tmp1, tmp2;
  for (int i = 0; i < 64; ++i) {
    t2.m[i] = -am.m[i];
    dt2.m[i] = c_f[a][i];
  }
  A8 fa;
  for (int i = 0; i < 64; ++i) fa.m[i] = c_f[a][i];
  for (int j = 20; j > 1; --j) {
    for (int i = 0; i < 64; ++i) {
      t3.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) + (1.0 / (j + 1)) * t2.m[i];
      dt3.m[i] = (1.0 / (j + 1)) * dt2.m[i];
    }
    A8 nam;
    for (int i = 0; i < 64; ++i) nam.m[i] = -am.m[i];
    a8_mul(t2, nam, t3);
    a8_mul(tmp1, fa, t3);
    a8_mul(tmp2, am, dt3);
    for (int i = 0; i < 64; ++i) dt2.m[i] = tmp1.m[i] - tmp2.m[i];
  }
  for (int i = 0; i < 64; ++i) r.m[i] = 0.5 * dt2.m[i];
}

// Determinant and inverse of an 8 x 8 matrix by Gaussian / Gauss-Jordan
// elimination with partial pivoting, on local copies.  (The reference uses an
// LU decomposition, matrix.h:275-420; the pivot order only changes rounding.)
// Kept out of line: inlined into the large per-link kernel, an in-place LU
// on the matrix struct gave a wrong determinant on this toolchain, while the
// same code in a small kernel was right.
__device__ __noinline__ double a8_det(const A8& m)
{
  double a[64];
  for (int i = 0; i < 64; ++i) a[i] = m.m[i];
  double det = 1.0;
  for (int j = 0; j < 8; ++j) {
    int p = j;
    double best = fabs(a[8 * j + j]);
    for (int i = j + 1; i < 8; ++i) {
      const double v = fabs(a[8 * i + j]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (p != j) {
      for (int k = 0; k < 8; ++k) {
        const double t = a[8 * j + k];
        a[8 * j + k] = a[8 * p + k];
        a[8 * p + k] = t;
      }
      det = -det;
    }
    const double piv = a[8 * j + j];
    det *= piv;
    if (piv == 0.0) return 0.0;
    for (int i = j + 1; i < 8; ++i) {
      const double f = a[8 * i + j] / piv;
      for (int k = j + 1; k < 8; ++k) a[8 * i + k] -= f * a[8 * j + k];
    }
  }
  return det;
}

__device__ __noinline__ void a8_inverse(A8& r, const A8& m)
{
  double a[64], x[64];
  for (int i = 0; i < 64; ++i) {
    a[i] = m.m[i];
    x[i] = (i % 9 == 0) ? 1.0 : 0.0;
  }
  for (int j = 0; j < 8; ++j) {
    int p = j;
    double best = fabs(a[8 * j + j]);
    for (int i = j + 1; i < 8; ++i) {
      const double v = fabs(a[8 * i + j]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (p != j) {
      for (int k = 0; k < 8; ++k) {
        double t = a[8 * j + k];
        a[8 * j + k] = a[8 * p + k];
        a[8 * p + k] = t;
        t = x[8 * j + k];
        x[8 * j + k] = x[8 * p + k];
        x[8 * p + k] = t;
      }
    }
    const double inv = 1.0 / a[8 * j + j];
    for (int k = 0; k < 8; ++k) {
      a[8 * j + k] *= inv;
      x[8 * j + k] *= inv;
    }
    for (int i = 0; i < 8; ++i) {
      if (i == j) continue;
      const double f = a[8 * i + j];
      if (f == 0.0) continue;
      for (int k = 0; k < 8; ++k) {
        a[8 * i + k] -= f * a[8 * j + k];
        x[8 * i + k] -= f * x[8 * j + k];
      }
    }
  }
  for (int i = 0; i < 64; ++i) r.m[i] = x[i];
}

// ---- masks and lattice walks (flowed-hmc.cpp:71-110) ----------------------

struct C4 {
  int x[4];
};

__device__ inline C4 shifted(C4 c, int dir)
{
  if (dir >= 0) c.x[dir] += 1;
  else c.x[-dir - 1] -= 1;
  return c;
}

__device__ inline bool same_coor(const C4& a, const C4& b)
{
  return a.x[0] == b.x[0] && a.x[1] == b.x[1] && a.x[2] == b.x[2] && a.x[3] == b.x[3];
}

__device__ inline int mask_of(const C4& c, int flow_size)
{
  if (flow_size == 1) return 2 - (c.x[0] + c.x[1] + c.x[2] + c.x[3] + 16 * 1024 * 1024) % 2;
  return 2 - ((c.x[0] + 1024) / 2 + (c.x[1] + 1024) / 2 + (c.x[2] + 1024) / 2 + (c.x[3] + 1024) / 2) % 2;
}

__device__ inline long site_index(const Geo& g, const C4& c)
{
  long idx = 0;
  for (int k = 3; k >= 0; --k) {
    int v = c.x[k] % g.d[k];
    if (v < 0) v += g.d[k];
    idx = idx * g.d[k] + v;
  }
  return idx;
}

__device__ inline C4 coor_of_site(const Geo& g, long s)
{
  C4 c;
  for (int k = 0; k < 4; ++k) {
    c.x[k] = (int)(s % g.d[k]);
    s /= g.d[k];
  }
  return c;
}

// gf_get_link: dir >= 0 is U_dir(x); dir < 0 is U_{-dir-1}(x - e)^+
__device__ inline M3<double> get_link(const CField<double>& U, const Geo& g, const C4& x, int dir)
{
  if (dir >= 0) return U.ld(site_index(g, x), dir);
  return adj(U.ld(site_index(g, shifted(x, dir)), -dir - 1));
}

// gf_wilson_line_no_comm (qcd-acc.h:23-41): ordered product from the unit matrix
__device__ inline M3<double> wilson_line(const CField<double>& U, const Geo& g, C4 x, const int* path, int n)
{
  M3<double> r = m3_unit<double>();
  for (int i = 0; i < n; ++i) {
    r = mul(r, get_link(U, g, x, path[i]));
    x = shifted(x, path[i]);
  }
  return r;
}

// gf_plaq_staple_no_comm (qcd-acc.h:152-165) / gf_srect_staple_no_comm (flowed-hmc.cpp:363-380)
__device__ inline M3<double> flow_staple(const CField<double>& U, const Geo& g, const C4& x, int mu, int flow_size)
{
  M3<double> acc = m3_zero<double>();
  for (int nu = -4; nu < 4; ++nu) {
    if (nu == mu || -nu - 1 == mu) continue;
    if (flow_size == 1) {
      const int p[3] = {nu, mu, -nu - 1};
      add_to(acc, wilson_line(U, g, x, p, 3));
    } else {
      const int p[5] = {nu, nu, mu, -nu - 1, -nu - 1};
      add_to(acc, wilson_line(U, g, x, p, 5));
    }
  }
  return acc;
}

__device__ inline int multiplicity_flow(bool same_mask, int flow_size)
{
  if (flow_size == 1) return same_mask ? 1 + 3 * 2 : 6 + 3 * 2;
  return same_mask ? 1 + 3 * 4 : 6 + 3 * 4;
}

__device__ inline int mod4(int v) { return ((v % 4) + 4) % 4; }

// set_xl_nu_from_mask_mu_yl_m (flowed-hmc.cpp:191-360): the m-th flowed link
// (xl, mu) whose flow depends on the link (yl, nu)
__device__ inline void pair_of(C4& xl, int& nu, int mask, int mu, const C4& yl, int m, int flow_size)
{
  const int mask_yl = mask_of(yl, flow_size);
  if (flow_size == 1) {
    if (mask == mask_yl) {
      if (m < 1) {
        nu = mu;
        xl = yl;
      } else {
        const int k = (m - 1) / 2, l = (m - 1) % 2;
        nu = mod4(mu + k + 1);
        xl = l == 0 ? yl : shifted(shifted(yl, nu), -mu - 1);
      }
    } else {
      if (m < 6) {
        nu = mu;
        const int k = m / 2, l = m % 2;
        const int dir = mod4(nu + k + 1);
        xl = l == 0 ? shifted(yl, dir) : shifted(yl, -dir - 1);
      } else {
        const int k = (m - 6) / 2, l = (m - 6) % 2;
        nu = mod4(mu + k + 1);
        xl = l == 0 ? shifted(yl, -mu - 1) : shifted(yl, nu);
      }
    }
    return;
  }
  const int nu_size = mask == mask_yl ? 1 : 6;
  if (m < nu_size) {
    nu = mu;
    if (mask == mask_yl) {
      xl = yl;
    } else {
      const int k = m / 2, l = m % 2;
      const int dir = mod4(nu + k + 1);
      xl = l == 0 ? shifted(shifted(yl, dir), dir) : shifted(shifted(yl, -dir - 1), -dir - 1);
    }
    return;
  }
  // set_xg_nu_from_mask_mu_yg_m_srect_nu_neq_mu
  const int k = (m - nu_size) / 4, l = (m - nu_size) % 4;
  nu = mod4(mu + k + 1);
  C4 x;
  int step;
  if (l == 0) {
    x = shifted(yl, -nu - 1);
    step = nu;
  } else if (l == 1) {
    x = shifted(shifted(yl, nu), nu);
    step = -nu - 1;
  } else if (l == 2) {
    x = shifted(shifted(yl, -mu - 1), -nu - 1);
    step = nu;
  } else {
    x = shifted(shifted(shifted(yl, -mu - 1), nu), nu);
    step = -nu - 1;
  }
  for (int it = 0; it < 8 && mask != mask_of(x, flow_size); ++it) x = shifted(x, step);
  xl = x;
}

// is_same_link (flowed-hmc.cpp:71-83)
__device__ inline int is_same_link(const C4& xl, int dir, const C4& yl, int nu)
{
  if (dir >= 0) return (dir == nu && same_coor(xl, yl)) ? 1 : 0;
  return (-dir - 1 == nu && same_coor(shifted(xl, dir), yl)) ? -1 : 0;
}

// d_uc_mat_plaq_site_no_comm / d_uc_mat_srect_site_no_comm
// (flowed-hmc.cpp:596-777): d TA(U C^+) / d(link (yl, nu)) = TA(uc_pre T uc_post)
__device__ inline void d_uc_mat(M3<double>& uc_pre, M3<double>& uc_post, const CField<double>& C,
                                const CField<double>& U, const Geo& g, const C4& xl, int mu, const C4& yl, int nu,
                                int flow_size)
{
  const M3<double> u = U.ld(site_index(g, xl), mu);
  if (mu == nu && same_coor(xl, yl)) {
    uc_pre = m3_unit<double>();
    uc_post = mul_adj(u, C.ld(site_index(g, xl), 0));
    return;
  }
  // the staple path from xl: (dir1, [dir1,] mu, dir3, [dir3]) with dir1 = k, dir3 = -k-1
  const int len = flow_size == 1 ? 3 : 5;
  int path[5];
  C4 pts[5];
  int n_step = 0, is_pos = 0;
  for (int k = -4; k < 4 && n_step == 0; ++k) {
    if (flow_size == 1) {
      path[0] = k;
      path[1] = mu;
      path[2] = -k - 1;
    } else {
      path[0] = k;
      path[1] = k;
      path[2] = mu;
      path[3] = -k - 1;
      path[4] = -k - 1;
    }
    pts[0] = xl;
    for (int i = 1; i < len; ++i) pts[i] = shifted(pts[i - 1], path[i - 1]);
    for (int i = 0; i < len; ++i) {
      is_pos = is_same_link(pts[i], path[i], yl, nu);
      if (is_pos != 0) {
        n_step = i + 1;
        break;
      }
    }
  }
  // pre = links before the matching one, dl = the matching link, post = after
  M3<double> pre = m3_unit<double>(), dl, post = m3_unit<double>();
  bool pre_set = false, post_set = false;
  for (int i = 0; i < len; ++i) {
    const M3<double> l = get_link(U, g, pts[i], path[i]);
    if (i + 1 < n_step) {
      pre = pre_set ? mul(pre, l) : l;
      pre_set = true;
    } else if (i + 1 == n_step) {
      dl = l;
    } else {
      post = post_set ? mul(post, l) : l;
      post_set = true;
    }
  }
  if (is_pos == 1) {
    post = mul(dl, post);
  } else {
    pre = scale(-1.0, mul(pre, dl));  // - from the dagger of the link for T^b
  }
  uc_pre = scale(-1.0, mul_adj(u, post));  // - from C^+ for T^b
  uc_post = adj(pre);
}

// n_mat from the pair's (uc_pre, uc_post): N(a, b) = basis_a(TA(uc_pre T_b uc_post))
__device__ inline void n_mat(A8& n, const M3<double>& uc_pre, const M3<double>& uc_post)
{
  for (int b = 0; b < 8; ++b) {
    const M3<double> d = traceless_antiherm(mul(mul(uc_pre, ts(b)), uc_post));
    double v[8];
    basis_of(d, v);
    for (int a = 0; a < 8; ++a) n.m[8 * a + b] = v[a];
  }
}

// ---- kernels ----------------------------------------------------------------

__global__ void k_flow_staple(Geo g, const Cx<double>* Up, Cx<double>* Cp, int mask, int mu, int flow_size)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const C4 x = coor_of_site(g, s);
  if (mask_of(x, flow_size) != mask) return;
  const CField<double> U{Up, g.V};
  WField<double>{Cp, g.V}.st(s, 0, flow_staple(U, g, x, mu, flow_size));
}

// gf_flow_plaq_mask_mu_no_comm (flowed-hmc.cpp:424-454) and its inverse
// (456-490, n_iter fixed-point iterations)
__global__ void k_flow_update(Geo g, Cx<double>* Up, const Cx<double>* Cp, int mask, int mu, int flow_size, double eps,
                              int inverse, int n_iter)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const C4 x = coor_of_site(g, s);
  if (mask_of(x, flow_size) != mask) return;
  const WField<double> U{Up, g.V};
  const M3<double> c = CField<double>{Cp, g.V}.ld(s, 0);
  const M3<double> u1 = U.ld(s, mu);
  M3<double> u0 = u1;
  if (!inverse) {
    const M3<double> z = scale(-1.0, traceless_antiherm(mul_adj(u1, c)));
    M3<double> e = exp_ch(scale(eps, z));
    unitarize(e);
    u0 = mul(e, u1);
  } else {
    for (int n = 0; n < n_iter; ++n) {
      const M3<double> xm = scale(-1.0, traceless_antiherm(mul_adj(u0, c)));
      M3<double> e = exp_ch(scale(-eps, xm));
      unitarize(e);
      u0 = mul(e, u1);
    }
  }
  U.st(s, mu, u0);
}

// Per flowed link: ln det M' (flowed-hmc.cpp:1011-1025, 1234-1255) into lnd[s]
// and, for the force, the table T[s] = exp(ad X) | J(-ad X) | e2dj[8] |
// (-eps) M'^-1 J(X) (flowed-hmc.cpp:926-955, 1117-1162).
__global__ void k_flow_link_tables(Geo g, const Cx<double>* Up, const Cx<double>* Cp, int mask, int mu, int flow_size,
                                   double eps, double* lnd, double* T)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const C4 x = coor_of_site(g, s);
  if (mask_of(x, flow_size) != mask) {
    if (lnd) lnd[s] = 0.0;
    return;
  }
  const CField<double> U{Up, g.V};
  const M3<double> u = U.ld(s, mu);
  const M3<double> c = CField<double>{Cp, g.V}.ld(s, 0);
  const M3<double> uc = mul_adj(u, c);
  A8 n0;
  for (int b = 0; b < 8; ++b) {
    double v[8];
    basis_of(traceless_antiherm(mul(mul(ts(b), u), adj(c))), v);
    for (int a = 0; a < 8; ++a) n0.m[8 * a + b] = v[a];
  }
  const M3<double> xm = scale(-eps, traceless_antiherm(uc));
  A8 adx, jx, ejx, mp;
  adjoint_rep(adx, xm);
  dexp_map(jx, adx);
  a8_scale(ejx, eps, jx);
  a8_mul(mp, ejx, n0);
  for (int i = 0; i < 64; ++i) mp.m[i] = ((i % 9 == 0) ? 1.0 : 0.0) - mp.m[i];
  if (lnd) lnd[s] = log(a8_det(mp));
  if (!T) return;
  double* t = T + s * 200;
  // exp(ad X) and J(-ad X)
  A8 tmp, nadx;
  a8_exp(tmp, adx);
  for (int i = 0; i < 64; ++i) t[i] = tmp.m[i];
  for (int i = 0; i < 64; ++i) nadx.m[i] = -adx.m[i];
  dexp_map(tmp, nadx);
  for (int i = 0; i < 64; ++i) t[64 + i] = tmp.m[i];
  // M'^-1
  A8 inv;
  a8_inverse(inv, mp);
  // e2dj[e] = tr(dJ/dX_e  eps^2 N M'^-1)
  A8 e2n, e2nmi;
  a8_scale(e2n, eps * eps, n0);
  a8_mul(e2nmi, e2n, inv);
  for (int e = 0; e < 8; ++e) {
    dexp_map_diff(tmp, adx, e);
    double tr = 0.0;
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) tr += tmp.m[8 * i + j] * e2nmi.m[8 * j + i];
    t[128 + e] = tr;
  }
  // (-eps) M'^-1 J(X)
  A8 einv;
  a8_scale(einv, -eps, inv);
  a8_mul(tmp, einv, jx);
  for (int i = 0; i < 64; ++i) t[136 + i] = tmp.m[i];
}

// One step of the force propagation (flowed-hmc.cpp:1059-1091, 1164-1232,
// 1366-1427): Fout(yl, nu) = sum over pairs of the transposed Jacobian
// applied to Fin(xl, mu), plus Fin(yl, nu) for the links the step does not
// move, plus the force of the step's log-determinants.
__global__ void k_flow_force_step(Geo g, const Cx<double>* Up, const Cx<double>* Cp, const double* T,
                                  const Cx<double>* Finp, Cx<double>* Foutp, int mask, int mu, int flow_size,
                                  double eps, int with_det)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const C4 yl = coor_of_site(g, s);
  const int mask_yl = mask_of(yl, flow_size);
  const CField<double> U{Up, g.V}, C{Cp, g.V}, Fin{Finp, g.V};
  M3<double> fprop[4], fdet[4];
  for (int nu = 0; nu < 4; ++nu) fprop[nu] = fdet[nu] = m3_zero<double>();
  const int nm = multiplicity_flow(mask == mask_yl, flow_size);
  for (int m = 0; m < nm; ++m) {
    C4 xl;
    int nu;
    pair_of(xl, nu, mask, mu, yl, m, flow_size);
    M3<double> uc_pre, uc_post;
    d_uc_mat(uc_pre, uc_post, C, U, g, xl, mu, yl, nu, flow_size);
    A8 n;
    n_mat(n, uc_pre, uc_post);
    const double* t = T + site_index(g, xl) * 200;
    // m_mat = [exp(ad X) if the same link] - (eps J(-ad X)) N
    A8 ej, mm;
    for (int i = 0; i < 64; ++i) ej.m[i] = eps * t[64 + i];
    a8_mul(mm, ej, n);
    const bool same = mu == nu && same_coor(xl, yl);
    for (int i = 0; i < 64; ++i) mm.m[i] = same ? t[i] - mm.m[i] : -mm.m[i];
    double bb[8], ba[8];
    basis_of(Fin.ld(site_index(g, xl), mu), bb);
    for (int a = 0; a < 8; ++a) ba[a] = 0.0;
    for (int b = 0; b < 8; ++b)
      for (int a = 0; a < 8; ++a) ba[a] += bb[b] * mm.m[8 * b + a];
    add_to(fprop[nu], anti_herm_from_basis(ba));
    if (with_det) {
      double fd[8];
      for (int a = 0; a < 8; ++a) {
        fd[a] = 0.0;
        for (int e = 0; e < 8; ++e) fd[a] += n.m[8 * e + a] * t[128 + e];
        const M3<double> ucm = mul(mul(uc_pre, ts(a)), uc_post);
        for (int c = 0; c < 8; ++c) {
          double dnb[8];
          basis_of(traceless_antiherm(mul(ts(c), ucm)), dnb);
          for (int b = 0; b < 8; ++b) fd[a] += t[136 + 8 * c + b] * dnb[b];
        }
      }
      add_to(fdet[nu], scale(0.5, anti_herm_from_basis(fd)));
    }
  }
  const WField<double> Fout{Foutp, g.V};
  for (int nu = 0; nu < 4; ++nu) {
    if (!(mask_yl == mask && mu == nu)) add_to(fprop[nu], Fin.ld(s, nu));
    add_to(fprop[nu], fdet[nu]);
    Fout.st(s, nu, fprop[nu]);
  }
}

__global__ void k_sum_sites(long V, const double* v, double* out)
{
  // one block: fixed-order sum of the per-site values
  __shared__ double sm[256];
  double t = 0.0;
  for (long i = threadIdx.x; i < V; i += blockDim.x) t += v[i];
  sm[threadIdx.x] = t;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

// ---- host side --------------------------------------------------------------

int ffail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

#define FL_CUDA(expr)                                                                                        \
  do {                                                                                                       \
    cudaError_t e_ = (expr);                                                                                 \
    if (e_ != cudaSuccess) return ffail(QGB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define FL_RC(expr)              \
  do {                           \
    int r_ = (expr);             \
    if (r_ != QGB_OK) return r_; \
  } while (0)

int init_constants_here()
{
  static uint64_t done = 0;  // one bit per device
  int dev = 0;
  FL_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && (done >> dev) & 1u) return QGB_OK;
  double tsh[8][18], fh[8][64];
  M3<double> t[8];
  for (int a = 0; a < 8; ++a) {
    double b[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    b[a] = 1.0;
    t[a] = anti_herm_from_basis(b);
    for (int k = 0; k < 9; ++k) {
      tsh[a][2 * k] = t[a].e[k].re;
      tsh[a][2 * k + 1] = t[a].e[k].im;
    }
  }
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) {
      M3<double> ab = mul(t[a], t[b]), ba = mul(t[b], t[a]);
      for (int k = 0; k < 9; ++k) {
        ab.e[k].re -= ba.e[k].re;
        ab.e[k].im -= ba.e[k].im;
      }
      double v[8];
      basis_of(ab, v);
      for (int c = 0; c < 8; ++c) fh[c][8 * a + b] = v[c];
    }
  FL_CUDA(cudaMemcpyToSymbol(c_ts, tsh, sizeof(tsh)));
  FL_CUDA(cudaMemcpyToSymbol(c_f, fh, sizeof(fh)));
  // the per-link 8 x 8 algebra keeps several KB of matrices per thread (a
  // setting of this process's context only)
  size_t stack = 0;
  FL_CUDA(cudaDeviceGetLimit(&stack, cudaLimitStackSize));
  if (stack < 16384) FL_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, 16384));
  if (dev < 64) done |= (uint64_t)1 << dev;
  return QGB_OK;
}

struct FlowCtx {
  Geo g;
  cudaStream_t st = nullptr;
  long V = 0;
  size_t bytes = 0;  // one gauge field
  int blocks = 0;
};

int check_steps(const Geo& g, const qgb_flow_step* steps, int n)
{
  if (n < 0 || (n > 0 && !steps)) return ffail(QGB_ERR_INVALID_ARG, "flowed: bad flow-step list");
  for (int i = 0; i < n; ++i) {
    const qgb_flow_step& f = steps[i];
    if ((f.mask != 1 && f.mask != 2) || f.mu < 0 || f.mu > 3 || (f.flow_size != 1 && f.flow_size != 2))
      return ffail(QGB_ERR_INVALID_ARG, "flowed: a flow step needs mask 1 or 2, mu 0..3, flow_size 1 or 2");
    for (int k = 0; k < 4; ++k)
      if (g.d[k] % (2 * f.flow_size) != 0)
        return ffail(QGB_ERR_BAD_GEOMETRY, "flowed: each lattice extent must be a multiple of 2 * flow_size");
  }
  return QGB_OK;
}

// One flow step (or its inverse) in place on U (device buffer), C a scratch
// color-matrix buffer of multiplicity 1.
int flow_step_dev(const FlowCtx& c, void* U, void* C, const qgb_flow_step& f, bool inverse)
{
  k_flow_staple<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)U, (Cx<double>*)C, f.mask, f.mu, f.flow_size);
  FL_CUDA(cudaGetLastError());
  k_flow_update<<<c.blocks, 128, 0, c.st>>>(c.g, (Cx<double>*)U, (const Cx<double>*)C, f.mask, f.mu, f.flow_size,
                                            f.epsilon, inverse ? 1 : 0, 50);
  FL_CUDA(cudaGetLastError());
  return QGB_OK;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  cudaError_t alloc(size_t b) { return cudaMalloc(&p, b); }
};

int setup(FlowCtx& c, const qgb_field* gf, int32_t n, const qgb_flow_step* steps)
{
  int32_t ts[4], mult = 0, kind = 0, prec = 0;
  FL_RC(qgb_field_info(gf, ts, &mult, &kind, &prec));
  if (kind != QGB_KIND_COLOR_MATRIX || mult != 4 || prec != QGB_F64)
    return ffail(QGB_ERR_MISMATCH, "flowed: the gauge field must be an FP64 color-matrix field of multiplicity 4");
  for (int k = 0; k < 4; ++k) c.g.d[k] = ts[k];
  c.g.V = (long)ts[0] * ts[1] * ts[2] * ts[3];
  c.V = c.g.V;
  c.bytes = (size_t)padded_sites(c.V) * 72 * sizeof(double);
  c.blocks = (int)((c.V + 127) / 128);
  FL_RC(qgb::library_stream(&c.st));
  FL_RC(check_steps(c.g, steps, n));
  return init_constants_here();
}

}  // namespace

extern "C" {

int qgb_flow_info_step(const uint32_t rs[24], double epsilon, double epsilon2, int32_t two_eps, qgb_flow_step* out,
                       int32_t* n_out)
{
  if (!rs || !out || !n_out) return ffail(QGB_ERR_INVALID_ARG, "qgb_flow_info_step: null argument");
  // mk_flow_info_step (flowed-hmc.cpp:21-69); random_permute (rng-state.h:85-97)
  auto permute = [](std::vector<qgb_flow_step>& v, const uint32_t* r) {
    uint32_t st[24];
    memcpy(st, r, sizeof(st));
    const long size = (long)v.size();
    for (long k = 0; k < size; ++k) {
      const long kk = (long)(qgb::rng_host_rand_gen(st) % (uint64_t)(size - k));
      std::swap(v[k], v[k + kk]);
    }
  };
  auto split = [&](const char* s, uint32_t* o) { return qgb::rng_host_split(o, rs, s); };
  std::vector<qgb_flow_step> fi;
  if (!two_eps) {
    for (int mu = 3; mu >= 0; --mu) {
      fi.push_back({2, mu, epsilon, 1});
      fi.push_back({1, mu, epsilon, 1});
    }
    permute(fi, rs);
  } else {
    std::vector<std::vector<qgb_flow_step>> g1(4), g2(4);
    for (int mu = 3; mu >= 0; --mu) {
      if (epsilon != 0.0) {
        g1[mu].push_back({2, mu, epsilon, 1});
        g1[mu].push_back({1, mu, epsilon, 1});
      }
      if (epsilon2 != 0.0) {
        g2[mu].push_back({2, mu, epsilon2, 2});
        g2[mu].push_back({1, mu, epsilon2, 2});
      }
    }
    for (int i = 0; i < 4; ++i) {
      uint32_t r1[24], r2[24];
      const std::string s1 = "fi1s-" + std::to_string(i), s2 = "fi2s-" + std::to_string(i);
      if (!split(s1.c_str(), r1) || !split(s2.c_str(), r2)) return ffail(QGB_ERR_INVALID_ARG, "qgb_flow_info_step: split");
      permute(g1[i], r1);
      permute(g2[i], r2);
      g1[i].insert(g1[i].end(), g2[i].begin(), g2[i].end());
    }
    // random_permute of the four groups with rs itself
    uint32_t st[24];
    memcpy(st, rs, sizeof(st));
    for (long k = 0; k < 4; ++k) {
      const long kk = (long)(qgb::rng_host_rand_gen(st) % (uint64_t)(4 - k));
      std::swap(g1[k], g1[k + kk]);
    }
    for (int i = 0; i < 4; ++i) fi.insert(fi.end(), g1[i].begin(), g1[i].end());
  }
  if ((int)fi.size() > 16) return ffail(QGB_ERR_INVALID_ARG, "qgb_flow_info_step: too many steps");
  for (size_t i = 0; i < fi.size(); ++i) out[i] = fi[i];
  *n_out = (int32_t)fi.size();
  return QGB_OK;
}

int qgb_gf_flow(qgb_field* gf, const qgb_field* gf0, const qgb_flow_step* steps, int32_t n)
{
  FlowCtx c;
  FL_RC(setup(c, gf0, n, steps));
  FL_RC(qgb_field_copy(gf, gf0));
  DevBuf C;
  FL_CUDA(C.alloc(c.bytes / 4));
  void* U = qgb::field_data(gf);
  for (int i = 0; i < n; ++i) FL_RC(flow_step_dev(c, U, C.p, steps[i], false));
  FL_CUDA(cudaStreamSynchronize(c.st));
  return QGB_OK;
}

int qgb_gf_flow_inv(qgb_field* gf, const qgb_field* gf1, const qgb_flow_step* steps, int32_t n)
{
  FlowCtx c;
  FL_RC(setup(c, gf1, n, steps));
  FL_RC(qgb_field_copy(gf, gf1));
  DevBuf C;
  FL_CUDA(C.alloc(c.bytes / 4));
  void* U = qgb::field_data(gf);
  for (int i = n - 1; i >= 0; --i) FL_RC(flow_step_dev(c, U, C.p, steps[i], true));
  FL_CUDA(cudaStreamSynchronize(c.st));
  return QGB_OK;
}

int qgb_gf_flow_and_ln_det_node(qgb_field* gf, const qgb_field* gf0, const qgb_flow_step* steps, int32_t n,
                                double* ln_det)
{
  FlowCtx c;
  FL_RC(setup(c, gf0, n, steps));
  if (!ln_det) return ffail(QGB_ERR_INVALID_ARG, "qgb_gf_flow_and_ln_det_node: null output");
  FL_RC(qgb_field_copy(gf, gf0));
  DevBuf C, L, S;
  FL_CUDA(C.alloc(c.bytes / 4));
  FL_CUDA(L.alloc(c.V * sizeof(double)));
  FL_CUDA(S.alloc((size_t)(n > 0 ? n : 1) * sizeof(double)));
  void* U = qgb::field_data(gf);
  for (int i = 0; i < n; ++i) {
    const qgb_flow_step& f = steps[i];
    k_flow_staple<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)U, (Cx<double>*)C.p, f.mask, f.mu,
                                              f.flow_size);
    FL_CUDA(cudaGetLastError());
    k_flow_link_tables<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)U, (const Cx<double>*)C.p, f.mask, f.mu,
                                                   f.flow_size, f.epsilon, (double*)L.p, nullptr);
    FL_CUDA(cudaGetLastError());
    k_sum_sites<<<1, 256, 0, c.st>>>(c.V, (const double*)L.p, (double*)S.p + i);
    FL_CUDA(cudaGetLastError());
    k_flow_update<<<c.blocks, 128, 0, c.st>>>(c.g, (Cx<double>*)U, (const Cx<double>*)C.p, f.mask, f.mu, f.flow_size,
                                              f.epsilon, 0, 0);
    FL_CUDA(cudaGetLastError());
  }
  std::vector<double> sums((size_t)(n > 0 ? n : 1), 0.0);
  if (n > 0) FL_CUDA(cudaMemcpyAsync(sums.data(), S.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
  FL_CUDA(cudaStreamSynchronize(c.st));
  double t = 0.0;
  for (int i = 0; i < n; ++i) t += sums[i];
  *ln_det = t;
  return QGB_OK;
}

int qgb_gf_hamilton_flowed_node(const qgb_field* gf0, double beta, double c1, const qgb_flow_step* steps, int32_t n,
                                double* flowed_action, double* ln_det)
{
  int32_t ts[4];
  FL_RC(qgb_field_info(gf0, ts, nullptr, nullptr, nullptr));
  qgb_field* gf = nullptr;
  FL_RC(qgb_field_create(&gf, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
  double ld = 0.0, act = 0.0;
  int rc = qgb_gf_flow_and_ln_det_node(gf, gf0, steps, n, &ld);
  if (rc == QGB_OK) rc = qgb_gf_hamilton_node(gf, beta, c1, &act);
  qgb_field_destroy(gf);
  if (rc != QGB_OK) return rc;
  if (flowed_action) *flowed_action = act;
  if (ln_det) *ln_det = ld;
  return QGB_OK;
}

}  // extern "C"

namespace
{
// The force on gf0 of a force F on the flowed field, propagated back through
// the steps with (with_det) or without the log-determinants' force.  F is the
// action's force on the flowed field (pre == nullptr) or the given field.
int flowed_force(qgb_field* gm_force, const qgb_field* gf0, const qgb_field* pre, double beta, double c1,
                 const qgb_flow_step* steps, int32_t n, int32_t with_det)
{
  FlowCtx c;
  FL_RC(setup(c, gf0, n, steps));
  int32_t ts[4];
  FL_RC(qgb_field_info(gf0, ts, nullptr, nullptr, nullptr));
  // gf_ext_vec: the field before each step, then the flowed field
  std::vector<DevBuf> G(n + 1);
  for (int i = 0; i <= n; ++i) FL_CUDA(G[i].alloc(c.bytes));
  DevBuf C, T, F2;
  FL_CUDA(C.alloc(c.bytes / 4));
  FL_CUDA(T.alloc((size_t)c.V * 200 * sizeof(double)));
  FL_CUDA(F2.alloc(c.bytes));
  FL_CUDA(cudaMemcpyAsync(G[0].p, qgb::field_data(gf0), c.bytes,
                          cudaMemcpyDeviceToDevice, c.st));
  for (int i = 0; i < n; ++i) {
    FL_CUDA(cudaMemcpyAsync(G[i + 1].p, G[i].p, c.bytes, cudaMemcpyDeviceToDevice, c.st));
    FL_RC(flow_step_dev(c, G[i + 1].p, C.p, steps[i], false));
  }
  if (pre) {
    FL_RC(qgb_field_copy(gm_force, pre));
  } else {
    // the force of the action on the flowed field (set_gm_force, hmc.cpp:466-490)
    qgb_field* gfl = nullptr;
    FL_RC(qgb_field_create(&gfl, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
    FL_CUDA(cudaMemcpyAsync(qgb::field_data(gfl), G[n].p, c.bytes, cudaMemcpyDeviceToDevice, c.st));
    int rc = qgb_set_gm_force(gm_force, gfl, beta, c1);
    qgb_field_destroy(gfl);
    FL_RC(rc);
  }
  void* F = qgb::field_data(gm_force);
  // back through the steps (set_gm_force_propagated_det_from_flow, flowed-hmc.cpp:1456-1477)
  for (int i = n - 1; i >= 0; --i) {
    const qgb_flow_step& f = steps[i];
    k_flow_staple<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)G[i].p, (Cx<double>*)C.p, f.mask, f.mu,
                                              f.flow_size);
    FL_CUDA(cudaGetLastError());
    k_flow_link_tables<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)G[i].p, (const Cx<double>*)C.p, f.mask,
                                                   f.mu, f.flow_size, f.epsilon, nullptr, (double*)T.p);
    FL_CUDA(cudaGetLastError());
    k_flow_force_step<<<c.blocks, 128, 0, c.st>>>(c.g, (const Cx<double>*)G[i].p, (const Cx<double>*)C.p,
                                                  (const double*)T.p, (const Cx<double>*)F, (Cx<double>*)F2.p, f.mask,
                                                  f.mu, f.flow_size, f.epsilon, with_det ? 1 : 0);
    FL_CUDA(cudaGetLastError());
    FL_CUDA(cudaMemcpyAsync(F, F2.p, c.bytes, cudaMemcpyDeviceToDevice, c.st));
  }
  FL_CUDA(cudaStreamSynchronize(c.st));
  return QGB_OK;
}
}  // namespace

extern "C" {

int qgb_set_gm_force_flowed(qgb_field* gm_force, const qgb_field* gf0, double beta, double c1,
                            const qgb_flow_step* steps, int32_t n, int32_t with_det)
{
  return flowed_force(gm_force, gf0, nullptr, beta, c1, steps, n, with_det);
}

int qgb_set_gm_force_flowed_no_det(qgb_field* gm_force, const qgb_field* gm_force_pre, const qgb_field* gf0,
                                   const qgb_flow_step* steps, int32_t n)
{
  if (!gm_force_pre) return ffail(QGB_ERR_INVALID_ARG, "qgb_set_gm_force_flowed_no_det: null force");
  return flowed_force(gm_force, gf0, gm_force_pre, 0.0, 0.0, steps, n, 0);
}

}  // extern "C"
