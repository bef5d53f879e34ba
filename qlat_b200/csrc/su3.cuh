// su3.cuh -- 3x3 complex matrix algebra for the gauge kernels (FP64 / FP32).
//
// Conventions follow Qlattice's ColorMatrix (qlat-utils mat-vec.h:115,
// matrix.h:45-260): row-major, element (i, j) at e[3*i + j].  The functions
// here are written for registers: everything is unrolled and products use
// fused multiply-adds.  Algorithms that change the order of floating-point
// operations relative to the reference are noted where they occur; all agree
// with the reference to rounding level (checked against the oracle).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#if defined(__CUDACC__)
#define QGB_HD __host__ __device__ __forceinline__
#else
#define QGB_HD inline
#endif

namespace qgb
{

template <typename R>
struct alignas(2 * sizeof(R)) Cx {
  R re, im;
};

template <typename R>
struct M3 {
  Cx<R> e[9];
};

template <typename R>
QGB_HD Cx<R> cx(R re, R im)
{
  Cx<R> c;
  c.re = re;
  c.im = im;
  return c;
}

template <typename R>
QGB_HD M3<R> m3_zero()
{
  M3<R> m;
#pragma unroll
  for (int i = 0; i < 9; ++i) m.e[i] = cx<R>(0, 0);
  return m;
}

template <typename R>
QGB_HD M3<R> m3_unit()
{
  M3<R> m = m3_zero<R>();
  m.e[0].re = m.e[4].re = m.e[8].re = R(1);
  return m;
}

// c = a * b
template <typename R>
QGB_HD M3<R> mul(const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[3 * i].re * b.e[j].re;
      R im = a.e[3 * i].re * b.e[j].im;
      re = fma(-a.e[3 * i].im, b.e[j].im, re);
      im = fma(a.e[3 * i].im, b.e[j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * k + j].re, re);
        re = fma(-a.e[3 * i + k].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * i + k].re, b.e[3 * k + j].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// c = a * b^dagger : c_ij = sum_k a_ik conj(b_jk)
template <typename R>
QGB_HD M3<R> mul_adj(const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[3 * i].re * b.e[3 * j].re;
      R im = -a.e[3 * i].re * b.e[3 * j].im;
      re = fma(a.e[3 * i].im, b.e[3 * j].im, re);
      im = fma(a.e[3 * i].im, b.e[3 * j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * j + k].re, re);
        re = fma(a.e[3 * i + k].im, b.e[3 * j + k].im, re);
        im = fma(-a.e[3 * i + k].re, b.e[3 * j + k].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * j + k].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// c = a^dagger * b : c_ij = sum_k conj(a_ki) b_kj
template <typename R>
QGB_HD M3<R> adj_mul(const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[i].re * b.e[j].re;
      R im = a.e[i].re * b.e[j].im;
      re = fma(a.e[i].im, b.e[j].im, re);
      im = fma(-a.e[i].im, b.e[j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * k + i].re, b.e[3 * k + j].re, re);
        re = fma(a.e[3 * k + i].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * k + i].re, b.e[3 * k + j].im, im);
        im = fma(-a.e[3 * k + i].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// s + a * b
template <typename R>
QGB_HD M3<R> add_mul(const M3<R>& s, const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = s.e[3 * i + j].re, im = s.e[3 * i + j].im;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * k + j].re, re);
        re = fma(-a.e[3 * i + k].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * i + k].re, b.e[3 * k + j].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// s + a * b^dagger
template <typename R>
QGB_HD M3<R> add_mul_adj(const M3<R>& s, const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = s.e[3 * i + j].re, im = s.e[3 * i + j].im;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * j + k].re, re);
        re = fma(a.e[3 * i + k].im, b.e[3 * j + k].im, re);
        im = fma(-a.e[3 * i + k].re, b.e[3 * j + k].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * j + k].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// s + a^dagger * b
template <typename R>
QGB_HD M3<R> add_adj_mul(const M3<R>& s, const M3<R>& a, const M3<R>& b)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = s.e[3 * i + j].re, im = s.e[3 * i + j].im;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        re = fma(a.e[3 * k + i].re, b.e[3 * k + j].re, re);
        re = fma(a.e[3 * k + i].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * k + i].re, b.e[3 * k + j].im, im);
        im = fma(-a.e[3 * k + i].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

template <typename R>
QGB_HD M3<R> adj(const M3<R>& a)
{
  M3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c.e[3 * i + j] = cx<R>(a.e[3 * j + i].re, -a.e[3 * j + i].im);
  return c;
}

// a += s * b
template <typename R>
QGB_HD void axpy(M3<R>& a, R s, const M3<R>& b)
{
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    a.e[i].re = fma(s, b.e[i].re, a.e[i].re);
    a.e[i].im = fma(s, b.e[i].im, a.e[i].im);
  }
}

template <typename R>
QGB_HD void add_to(M3<R>& a, const M3<R>& b)
{
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    a.e[i].re += b.e[i].re;
    a.e[i].im += b.e[i].im;
  }
}

template <typename R>
QGB_HD M3<R> scale(R s, const M3<R>& b)
{
  M3<R> a;
#pragma unroll
  for (int i = 0; i < 9; ++i) a.e[i] = cx<R>(s * b.e[i].re, s * b.e[i].im);
  return a;
}

// Re tr(a b^dagger) = sum_ij Re(a_ij conj(b_ij))
template <typename R>
QGB_HD R re_tr_mul_adj(const M3<R>& a, const M3<R>& b)
{
  R s = a.e[0].re * b.e[0].re;
  s = fma(a.e[0].im, b.e[0].im, s);
#pragma unroll
  for (int i = 1; i < 9; ++i) {
    s = fma(a.e[i].re, b.e[i].re, s);
    s = fma(a.e[i].im, b.e[i].im, s);
  }
  return s;
}

// Re tr(a b) = sum_ij Re(a_ij b_ji)
template <typename R>
QGB_HD R re_tr_mul(const M3<R>& a, const M3<R>& b)
{
  R s = R(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      s = fma(a.e[3 * i + j].re, b.e[3 * j + i].re, s);
      s = fma(-a.e[3 * i + j].im, b.e[3 * j + i].im, s);
    }
  return s;
}

template <typename R>
QGB_HD R re_tr(const M3<R>& a)
{
  return a.e[0].re + a.e[4].re + a.e[8].re;
}

// Traceless anti-Hermitian part (m - m^dagger)/2 - tr(m - m^dagger)/6
// (matrix-hmc.h:202-213).  The diagonal of (m - m^dagger)/2 is i Im(m_ii).
template <typename R>
QGB_HD M3<R> traceless_antiherm(const M3<R>& m)
{
  M3<R> r;
  const R c = (m.e[0].im + m.e[4].im + m.e[8].im) / R(3);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r.e[4 * i] = cx<R>(R(0), m.e[4 * i].im - c);
#pragma unroll
    for (int j = i + 1; j < 3; ++j) {
      const R re = R(0.5) * (m.e[3 * i + j].re - m.e[3 * j + i].re);
      const R im = R(0.5) * (m.e[3 * i + j].im + m.e[3 * j + i].im);
      r.e[3 * i + j] = cx<R>(re, im);
      r.e[3 * j + i] = cx<R>(-re, im);
    }
  }
  return r;
}

// -1/2 tr(m^2) for anti-Hermitian m in the su(3) basis with tr(T_a T_b) = -2 delta_ab:
// sum of the squared basis coefficients (matrix-hmc.h:144-152).
template <typename R>
QGB_HD double neg_half_tr_square(const M3<R>& m)
{
  const double p1 = m.e[0].im, p9 = m.e[4].im, p17 = m.e[8].im;
  const double p2 = m.e[1].re, p3 = m.e[1].im, p4 = m.e[2].re, p5 = m.e[2].im;
  const double p10 = m.e[5].re, p11 = m.e[5].im;
  return p3 * p3 + p2 * p2 + (p1 - p9) * (p1 - p9) * 0.25 + p5 * p5 + p4 * p4 + p11 * p11 + p10 * p10 +
         p17 * p17 * 0.75;
}

// ---- two-row products of SU(3) matrices -------------------------------------
// For U in SU(3) the third row is conj(row0 x row1).  Rows 0 and 1 of a
// product A B depend only on rows 0 and 1 of A, so a chain of SU(3) products
// can carry two rows (18 complex multiply-adds per product instead of 27) and
// rebuild the third row once at the end (complete: 24 FMAs).  Exact for exact
// SU(3) factors; for links that are unitary to rounding the difference from
// the full product is of that rounding size.

template <typename R>
struct M32 {
  Cx<R> e[6];  // rows 0 and 1, row-major
};

// rows 0, 1 of a b, with a given by its first two rows (the first 6 entries)
template <typename R, typename A>
QGB_HD M32<R> mul2(const A& a, const M3<R>& b)
{
  M32<R> c;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[3 * i].re * b.e[j].re;
      R im = a.e[3 * i].re * b.e[j].im;
      re = fma(-a.e[3 * i].im, b.e[j].im, re);
      im = fma(a.e[3 * i].im, b.e[j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * k + j].re, re);
        re = fma(-a.e[3 * i + k].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * i + k].re, b.e[3 * k + j].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// rows 0, 1 of a b^dagger
template <typename R, typename A>
QGB_HD M32<R> mul2_adj(const A& a, const M3<R>& b)
{
  M32<R> c;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[3 * i].re * b.e[3 * j].re;
      R im = -a.e[3 * i].re * b.e[3 * j].im;
      re = fma(a.e[3 * i].im, b.e[3 * j].im, re);
      im = fma(a.e[3 * i].im, b.e[3 * j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * i + k].re, b.e[3 * j + k].re, re);
        re = fma(a.e[3 * i + k].im, b.e[3 * j + k].im, re);
        im = fma(-a.e[3 * i + k].re, b.e[3 * j + k].im, im);
        im = fma(a.e[3 * i + k].im, b.e[3 * j + k].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// rows 0, 1 of a^dagger b (needs all of a)
template <typename R>
QGB_HD M32<R> adj_mul2(const M3<R>& a, const M3<R>& b)
{
  M32<R> c;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R re = a.e[i].re * b.e[j].re;
      R im = a.e[i].re * b.e[j].im;
      re = fma(a.e[i].im, b.e[j].im, re);
      im = fma(-a.e[i].im, b.e[j].re, im);
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        re = fma(a.e[3 * k + i].re, b.e[3 * k + j].re, re);
        re = fma(a.e[3 * k + i].im, b.e[3 * k + j].im, re);
        im = fma(a.e[3 * k + i].re, b.e[3 * k + j].im, im);
        im = fma(-a.e[3 * k + i].im, b.e[3 * k + j].re, im);
      }
      c.e[3 * i + j] = cx<R>(re, im);
    }
  }
  return c;
}

// the SU(3) matrix with rows 0, 1 of a and row 2 = conj(row0 x row1)
template <typename R>
QGB_HD M3<R> complete(const M32<R>& a)
{
  M3<R> m;
#pragma unroll
  for (int k = 0; k < 6; ++k) m.e[k] = a.e[k];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const Cx<R> u1 = a.e[(j + 1) % 3], u2 = a.e[(j + 2) % 3];
    const Cx<R> v1 = a.e[3 + (j + 1) % 3], v2 = a.e[3 + (j + 2) % 3];
    // conj(u1 v2 - u2 v1)
    R re = u1.re * v2.re;
    re = fma(-u1.im, v2.im, re);
    re = fma(-u2.re, v1.re, re);
    re = fma(u2.im, v1.im, re);
    R im = -u1.re * v2.im;
    im = fma(-u1.im, v2.re, im);
    im = fma(u2.re, v1.im, im);
    im = fma(u2.im, v1.re, im);
    m.e[6 + j] = cx<R>(re, im);
  }
  return m;
}

// Gram-Schmidt projection onto SU(3) (matrix-hmc.h:11-74): normalise row 1,
// orthogonalise and normalise row 2, row 3 = conj(row1 x row2).  The
// arithmetic type C may be wider than the storage type (FP64 arithmetic on
// FP32 links).
template <typename C, typename R>
QGB_HD void unitarize_as(M3<R>& m)
{
  C r1[6], r2[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r1[2 * k] = C(m.e[k].re);
    r1[2 * k + 1] = C(m.e[k].im);
    r2[2 * k] = C(m.e[3 + k].re);
    r2[2 * k + 1] = C(m.e[3 + k].im);
  }
  C n1 = C(0);
#pragma unroll
  for (int k = 0; k < 6; ++k) n1 = fma(r1[k], r1[k], n1);
  if (!(n1 == C(1))) {
    const C inv = C(1) / sqrt(n1);
#pragma unroll
    for (int k = 0; k < 6; ++k) r1[k] *= inv;
  }
  // c = sum_k conj(r1_k) r2_k
  C cre = C(0), cim = C(0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    cre = fma(r1[2 * k], r2[2 * k], cre);
    cre = fma(r1[2 * k + 1], r2[2 * k + 1], cre);
    cim = fma(r1[2 * k], r2[2 * k + 1], cim);
    cim = fma(-r1[2 * k + 1], r2[2 * k], cim);
  }
  if (!(cre == C(0) && cim == C(0))) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const C are = r1[2 * k], aim = r1[2 * k + 1];
      r2[2 * k] -= cre * are - cim * aim;
      r2[2 * k + 1] -= cre * aim + cim * are;
    }
  }
  C n2 = C(0);
#pragma unroll
  for (int k = 0; k < 6; ++k) n2 = fma(r2[k], r2[k], n2);
  if (!(n2 == C(1))) {
    const C inv = C(1) / sqrt(n2);
#pragma unroll
    for (int k = 0; k < 6; ++k) r2[k] *= inv;
  }
  // row 3 = conj(r1 x r2)
  const C a0r = r1[0], a0i = r1[1], a1r = r1[2], a1i = r1[3], a2r = r1[4], a2i = r1[5];
  const C b0r = r2[0], b0i = r2[1], b1r = r2[2], b1i = r2[3], b2r = r2[4], b2i = r2[5];
  const C x0r = (a1r * b2r - a1i * b2i) - (a2r * b1r - a2i * b1i);
  const C x0i = (a1r * b2i + a1i * b2r) - (a2r * b1i + a2i * b1r);
  const C x1r = (a2r * b0r - a2i * b0i) - (a0r * b2r - a0i * b2i);
  const C x1i = (a2r * b0i + a2i * b0r) - (a0r * b2i + a0i * b2r);
  const C x2r = (a0r * b1r - a0i * b1i) - (a1r * b0r - a1i * b0i);
  const C x2i = (a0r * b1i + a0i * b1r) - (a1r * b0i + a1i * b0r);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    m.e[k] = cx<R>(R(r1[2 * k]), R(r1[2 * k + 1]));
    m.e[3 + k] = cx<R>(R(r2[2 * k]), R(r2[2 * k + 1]));
  }
  m.e[6] = cx<R>(R(x0r), R(-x0i));
  m.e[7] = cx<R>(R(x1r), R(-x1i));
  m.e[8] = cx<R>(R(x2r), R(-x2i));
}

template <typename R>
QGB_HD void unitarize(M3<R>& m)
{
  unitarize_as<R, R>(m);
}

// exp(a) by the order-N Taylor series in Horner form, exactly the
// reference's make_matrix_exp (matrix-hmc.h:155-167).  Used where the
// reference's own truncation must be reproduced (the hot start).
template <typename R>
QGB_HD M3<R> exp_taylor(const M3<R>& a, int max_order = 20)
{
  M3<R> t2 = a;
  M3<R> t3;
  for (int j = max_order; j > 1; --j) {
    t3 = scale(R(1) / R(j), t2);
    t3.e[0].re += R(1);
    t3.e[4].re += R(1);
    t3.e[8].re += R(1);
    t2 = mul(a, t3);
  }
  t3 = t2;
  t3.e[0].re += R(1);
  t3.e[4].re += R(1);
  t3.e[8].re += R(1);
  return t3;
}

// Complex helpers for the Cayley-Hamilton exponential.
template <typename R>
QGB_HD Cx<R> cmul(Cx<R> a, Cx<R> b)
{
  return cx<R>(fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re));
}

#if defined(__CUDACC__)
// 1/n for the exponential's recursion (compile-time constants, so the
// correctly rounded quotients)
static __constant__ double qgb_inv_n[21] = {0.0,        1.0 / 1,  1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,
                                            1.0 / 7,    1.0 / 8,  1.0 / 9,  1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13,
                                            1.0 / 14,   1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20};
#endif

// The reference's exponential, sum_{n=0}^{20} a^n / n! (the order-20 Taylor
// polynomial that make_matrix_exp evaluates in Horner form,
// matrix-hmc.h:155-167), evaluated through the Cayley-Hamilton theorem: with
// t = tr a, s = (t^2 - tr a^2)/2, d = det a, every power a^n equals
// x_n 1 + y_n a + z_n a^2 with (x, y, z)_{n+1} = (z_n d, x_n - z_n s, y_n + z_n t),
// so the polynomial is f0 1 + f1 a + f2 a^2 with f = sum_{n<=20} (x, y, z)_n / n!.
// Cost: one matrix product (a^2) plus a 20-step scalar recursion, instead of
// the 19 matrix products of the Horner form.  It is the same polynomial, so it
// keeps the reference's truncation (which matters when |a| reaches ~3, as in
// gradient flow of rough fields with large steps) and differs from it only by
// rounding.  In FP32 the recursion stops as soon as the omitted terms are below
// FP32 resolution (the same polynomial to FP32 accuracy, fewer steps for the
// small arguments of molecular dynamics).
template <typename R>
QGB_HD M3<R> exp_ch(const M3<R>& a)
{
  const M3<R> a2 = mul(a, a);
  const Cx<R> t = cx<R>(a.e[0].re + a.e[4].re + a.e[8].re, a.e[0].im + a.e[4].im + a.e[8].im);
  const Cx<R> t2 = cx<R>(a2.e[0].re + a2.e[4].re + a2.e[8].re, a2.e[0].im + a2.e[4].im + a2.e[8].im);
  const Cx<R> tt = cmul(t, t);
  const Cx<R> s = cx<R>(R(0.5) * (tt.re - t2.re), R(0.5) * (tt.im - t2.im));
  // det a by cofactor expansion along row 0
  const Cx<R> p48 = cmul(a.e[4], a.e[8]), p57 = cmul(a.e[5], a.e[7]);
  const Cx<R> p56 = cmul(a.e[5], a.e[6]), p38 = cmul(a.e[3], a.e[8]);
  const Cx<R> p37 = cmul(a.e[3], a.e[7]), p46 = cmul(a.e[4], a.e[6]);
  const Cx<R> d0 = cmul(a.e[0], cx<R>(p48.re - p57.re, p48.im - p57.im));
  const Cx<R> d1 = cmul(a.e[1], cx<R>(p56.re - p38.re, p56.im - p38.im));
  const Cx<R> d2 = cmul(a.e[2], cx<R>(p37.re - p46.re, p37.im - p46.im));
  const Cx<R> d = cx<R>(d0.re + d1.re + d2.re, d0.im + d1.im + d2.im);
  Cx<R> x = cx<R>(R(1), R(0)), y = cx<R>(R(0), R(0)), z = cx<R>(R(0), R(0));
  Cx<R> f0 = x, f1 = y, f2 = z;
  auto step = [&](R inv) {
    const Cx<R> zd = cmul(z, d), zs = cmul(z, s), zt = cmul(z, t);
    const Cx<R> xn = cx<R>(zd.re * inv, zd.im * inv);
    const Cx<R> yn = cx<R>((x.re - zs.re) * inv, (x.im - zs.im) * inv);
    const Cx<R> zn = cx<R>((y.re + zt.re) * inv, (y.im + zt.im) * inv);
    x = xn;
    y = yn;
    z = zn;
    f0.re += x.re;
    f0.im += x.im;
    f1.re += y.re;
    f1.im += y.im;
    f2.re += z.re;
    f2.im += z.im;
  };
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(R) == 4) {
    // FP32: after step n the partial sums are the Taylor polynomial of order n.
    // Stop once the remainder, bounded with the Frobenius norm by
    // sum_{k>n} |a|^k / k! <= 2 |a|^(n+1) / (n+1)! when |a| < (n+2)/2, is below
    // 2^-27 (under FP32 resolution); large |a| still runs all 20 terms.
    R nrm2 = R(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) nrm2 = fma(a.e[i].re, a.e[i].re, fma(a.e[i].im, a.e[i].im, nrm2));
    const R nrm = sqrt(nrm2);
    R term = R(1);  // |a|^n / n!
#pragma unroll 1
    for (int n = 1; n <= 20; ++n) {
      const R inv = __frcp_rn(R(n));  // the correctly rounded 1 / n
      step(inv);
      term *= nrm * inv;
      if (R(2) * term * nrm < R(7.450580596923828e-9) * R(n + 1) && nrm < R(0.5) * R(n + 2)) break;
    }
  } else {
    // FP64: all 20 steps, 1/n from a table of the correctly rounded values
#pragma unroll 1
    for (int n = 1; n <= 20; ++n) step(R(qgb_inv_n[n]));
  }
#else
  for (int n = 1; n <= 20; ++n) step(R(1) / R(n));
#endif
  M3<R> r;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const Cx<R> p = cmul(f1, a.e[i]);
    const Cx<R> q = cmul(f2, a2.e[i]);
    r.e[i] = cx<R>(p.re + q.re, p.im + q.im);
  }
  r.e[0].re += f0.re;
  r.e[0].im += f0.im;
  r.e[4].re += f0.re;
  r.e[4].im += f0.im;
  r.e[8].re += f0.re;
  r.e[8].im += f0.im;
  return r;
}

#if defined(__CUDACC__)
// 1/n in FP32 for exp_su3's recursion (compile-time quotients: correctly rounded)
static __constant__ float qgb_inv_nf[21] = {0.0f,       1.0f / 1,  1.0f / 2,  1.0f / 3,  1.0f / 4,  1.0f / 5,
                                            1.0f / 6,   1.0f / 7,  1.0f / 8,  1.0f / 9,  1.0f / 10, 1.0f / 11,
                                            1.0f / 12,  1.0f / 13, 1.0f / 14, 1.0f / 15, 1.0f / 16, 1.0f / 17,
                                            1.0f / 18,  1.0f / 19, 1.0f / 20};
#endif

// exp(a) of an su(3) matrix (anti-hermitian, traceless): the same polynomial
// as exp_ch (the reference's order-20 Taylor polynomial), with the structure
// of su(3) used in the Cayley-Hamilton coefficients: t = tr a = 0,
// s = -tr(a^2)/2 is real, d = det a = tr(a^3)/3 is imaginary (i delta), and
// a^2 is hermitian, so
//   - a^2 needs its real diagonal and upper triangle (half a product),
//   - delta = Im tr(a^3)/3 = Im sum_ij (a^2)_ij a_ji replaces the cofactor
//     determinant,
//   - a recursion step (x, y, z) <- ((i delta z), x - s z, y) / n costs real
//     multiplies instead of complex ones,
//   - the Frobenius norm is sqrt(2 s).
// The recursion stops once the omitted Taylor terms are bounded (Frobenius
// norm, sum_{k>n} |a|^k / k! <= 2 |a|^(n+1) / (n+1)! when |a| < (n+2)/2) below
// the type's resolution: 2^-27 in FP32, 2^-56 in FP64 -- the 20-term
// polynomial to rounding, in fewer steps for small arguments (a large |a|
// still runs all 20).  The fused molecular-dynamics and flow epilogues of the
// force call it: their arguments (momenta, TA-projected forces, flow
// combinations of them) are in su(3) up to rounding, and that rounding-size
// remainder is what the specialisation drops.
template <typename R>
QGB_HD M3<R> exp_su3(const M3<R>& a)
{
  // (a^2)_ii (real) and (a^2)_ij, i < j
  R h[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    R v = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) v = fma(a.e[3 * i + k].re, a.e[3 * k + i].re, fma(-a.e[3 * i + k].im, a.e[3 * k + i].im, v));
    h[i] = v;
  }
  Cx<R> u[3];  // (0,1), (0,2), (1,2)
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int i = q == 2 ? 1 : 0, j = q == 0 ? 1 : 2;
    R re = R(0), im = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      re = fma(a.e[3 * i + k].re, a.e[3 * k + j].re, fma(-a.e[3 * i + k].im, a.e[3 * k + j].im, re));
      im = fma(a.e[3 * i + k].re, a.e[3 * k + j].im, fma(a.e[3 * i + k].im, a.e[3 * k + j].re, im));
    }
    u[q] = cx<R>(re, im);
  }
  const R s = R(-0.5) * (h[0] + h[1] + h[2]);
  // Im tr(a^3) = sum_i (a^2)_ii Im a_ii + sum_{i<j} Im[(a^2)_ij a_ji + conj((a^2)_ij) a_ij]
  R t3 = h[0] * a.e[0].im;
  t3 = fma(h[1], a.e[4].im, t3);
  t3 = fma(h[2], a.e[8].im, t3);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int i = q == 2 ? 1 : 0, j = q == 0 ? 1 : 2;
    const Cx<R> aij = a.e[3 * i + j], aji = a.e[3 * j + i];
    t3 = fma(u[q].re, aji.im + aij.im, t3);
    t3 = fma(u[q].im, aji.re - aij.re, t3);
  }
  const R delta = t3 * (R(1) / R(3));
  const R nrm = sqrt(fmax(R(2) * s, R(0)));
  const R tol = sizeof(R) == 4 ? R(7.450580596923828e-9) : R(1.3877787807814457e-17);
  // (x, y, z)_n: a^n / n! = x 1 + y a + z a^2; f = sum_n (x, y, z)_n
  Cx<R> x = cx<R>(R(1), R(0)), y = cx<R>(R(0), R(0)), z = cx<R>(R(0), R(0));
  Cx<R> f0 = x, f1 = y, f2 = z;
  R term = R(1);  // |a|^n / n!
#pragma unroll 1
  for (int n = 1; n <= 20; ++n) {
#if defined(__CUDA_ARCH__)
    const R inv = sizeof(R) == 4 ? R(qgb_inv_nf[n]) : R(qgb_inv_n[n]);
#else
    const R inv = R(1) / R(n);
#endif
    const R di = delta * inv;
    const Cx<R> xn = cx<R>(-di * z.im, di * z.re);
    const Cx<R> yn = cx<R>(fma(-s, z.re, x.re) * inv, fma(-s, z.im, x.im) * inv);
    z = cx<R>(y.re * inv, y.im * inv);
    x = xn;
    y = yn;
    f0.re += x.re;
    f0.im += x.im;
    f1.re += y.re;
    f1.im += y.im;
    f2.re += z.re;
    f2.im += z.im;
    term *= nrm * inv;
    if (R(2) * term * nrm < tol * R(n + 1) && nrm < R(0.5) * R(n + 2)) break;
  }
  // r = f0 1 + f1 a + f2 a^2, with (a^2)_ji = conj((a^2)_ij)
  M3<R> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      Cx<R> q2;
      if (i == j) q2 = cx<R>(h[i], R(0));
      else if (i < j) q2 = u[i + j - 1];
      else q2 = cx<R>(u[i + j - 1].re, -u[i + j - 1].im);
      const Cx<R> ae = a.e[3 * i + j];
      R re = fma(f1.re, ae.re, fma(-f1.im, ae.im, fma(f2.re, q2.re, -f2.im * q2.im)));
      R im = fma(f1.re, ae.im, fma(f1.im, ae.re, fma(f2.re, q2.im, f2.im * q2.re)));
      if (i == j) {
        re += f0.re;
        im += f0.im;
      }
      r.e[3 * i + j] = cx<R>(re, im);
    }
  return r;
}

// The exponential of the fused epilogues (both precisions).
template <typename R>
QGB_HD M3<R> exp_md(const M3<R>& a)
{
  return exp_su3(a);
}

}  // namespace qgb
