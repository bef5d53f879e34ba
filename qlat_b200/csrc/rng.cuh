// rng.cuh -- Qlattice's SHA-256 counter RNG (RngState), bit-exact on the GPU.
//
// Restates qlat-utils rng-state.h:12-99, lib/rng-state.cpp:150-281 and the
// SHA-256 compression of lib/sha256.cpp:71-507 (FIPS 180-4).  All of it is
// __host__ __device__: the host copy serves the library's RngState API, the
// device copy generates per-site streams (RngState(rs, gindex), qcd-utils.cpp:47-92).
//
// Bit-exactness.  Integer work (hashing, counters, u64 -> double) is exact by
// construction.  The floating-point steps of the Gaussian draw use explicitly
// rounded operations (no fused multiply-add contraction) in the reference's
// order.  The reference takes the logarithm from the C library; on the GPU we
// use qgb::log_cr below, which is correctly rounded.  The C library's log
// agrees with the correctly rounded value on all but ~0.08% of the inputs
// drawn here (it is accurate to 0.52 ulp, not 0.5); those draws differ by one
// unit in the last place.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "crlog_table.h"
#include "su3.cuh"

#if defined(__CUDA_ARCH__)
#define QGB_DMUL(a, b) __dmul_rn((a), (b))
#define QGB_DADD(a, b) __dadd_rn((a), (b))
#define QGB_DSUB(a, b) __dsub_rn((a), (b))
#define QGB_DDIV(a, b) __ddiv_rn((a), (b))
#define QGB_DSQRT(a) __dsqrt_rn((a))
#define QGB_DFMA(a, b, c) __fma_rn((a), (b), (c))
#define QGB_U2D(u) __ull2double_rn((u))
#else
// Host builds use -ffp-contract=off, so plain operators round once each.
#define QGB_DMUL(a, b) ((a) * (b))
#define QGB_DADD(a, b) ((a) + (b))
#define QGB_DSUB(a, b) ((a) - (b))
#define QGB_DDIV(a, b) ((a) / (b))
#define QGB_DSQRT(a) sqrt((a))
#define QGB_DFMA(a, b, c) fma((a), (b), (c))
#define QGB_U2D(u) ((double)(u))
#endif

namespace qgb
{

// ------------------------------------------------------------------------
// correctly rounded natural logarithm
//
// x = 2^e m with m in [sqrt(1/2), sqrt(2)); c = j/128 nearest to m;
// log x = e log 2 + log c + 2 atanh(s), s = (m - c)/(m + c), |s| < 2^-8.5.
// m - c is exact; s and the series 2s(1 + s^2/3 + s^4/5 + ...) are carried
// in double-double, giving |error| < 2^-96 |log x| (including the table and
// log 2 constants, each exact to 2^-105, and the worst cancellation between
// log c and the series, a factor below 2^7.3).  The bound used is 2^-94.  The double-double result
// (hi, lo) is rounded once; if hi + lo lies within that error bound of a
// rounding boundary the result cannot be certified and *ambiguous is set
// (probability ~2^-40 per call; counted and reported by the library).

struct DD {
  double hi, lo;
};

QGB_HD DD dd_two_sum(double a, double b)
{
  const double s = QGB_DADD(a, b);
  const double bb = QGB_DSUB(s, a);
  const double err = QGB_DADD(QGB_DSUB(a, QGB_DSUB(s, bb)), QGB_DSUB(b, bb));
  return DD{s, err};
}
QGB_HD DD dd_fast_two_sum(double a, double b)
{
  const double s = QGB_DADD(a, b);
  return DD{s, QGB_DSUB(b, QGB_DSUB(s, a))};
}
QGB_HD DD dd_add(DD a, DD b)
{
  DD s = dd_two_sum(a.hi, b.hi);
  DD t = dd_two_sum(a.lo, b.lo);
  s.lo = QGB_DADD(s.lo, t.hi);
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo = QGB_DADD(s.lo, t.lo);
  return dd_fast_two_sum(s.hi, s.lo);
}
QGB_HD DD dd_mul(DD a, DD b)
{
  const double p = QGB_DMUL(a.hi, b.hi);
  double e = QGB_DFMA(a.hi, b.hi, -p);
  e = QGB_DADD(e, QGB_DADD(QGB_DMUL(a.hi, b.lo), QGB_DMUL(a.lo, b.hi)));
  return dd_fast_two_sum(p, e);
}
QGB_HD DD dd_mul_d(DD a, double b)
{
  const double p = QGB_DMUL(a.hi, b);
  double e = QGB_DFMA(a.hi, b, -p);
  e = QGB_DADD(e, QGB_DMUL(a.lo, b));
  return dd_fast_two_sum(p, e);
}

QGB_HD uint64_t d2u(double x)
{
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, 8);
  return u;
#endif
}
QGB_HD double u2d_bits(uint64_t u)
{
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, 8);
  return x;
#endif
}

#if defined(__CUDACC__)
__constant__ double qgb_logtab_dev[QGB_LOGTAB_N][2];
#endif

QGB_HD void logtab_get(int j, double& hi, double& lo)
{
#if defined(__CUDA_ARCH__)
  hi = qgb_logtab_dev[j - QGB_LOGTAB_J0][0];
  lo = qgb_logtab_dev[j - QGB_LOGTAB_J0][1];
#else
  hi = qgb_logtab_host[j - QGB_LOGTAB_J0][0];
  lo = qgb_logtab_host[j - QGB_LOGTAB_J0][1];
#endif
}

// log(x) for finite x > 0 (the RNG only asks for x in (0, 1)).
QGB_HD double log_cr(double x, int* ambiguous)
{
  uint64_t u = d2u(x);
  int e = 0;
  if ((u >> 52) == 0) {  // subnormal: scale into the normal range
    x = QGB_DMUL(x, 18014398509481984.0);  // 2^54
    u = d2u(x);
    e = -54;
  }
  e += (int)(u >> 52) - 1023;
  double m = u2d_bits((u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);  // [1, 2)
  if (m > 1.4142135623730951) {  // above sqrt(2) rounded up: use m/2 in [0.707, 1)
    m = QGB_DMUL(m, 0.5);
    e += 1;
  }
  const int j = (int)rint(QGB_DMUL(m, 128.0));
  const double c = QGB_DMUL((double)j, 0.0078125);
  const double d = QGB_DSUB(m, c);  // exact
  const DD sum = dd_two_sum(m, c);
  // s = d / (m + c) in double-double
  const double sh = QGB_DDIV(d, sum.hi);
  double r = QGB_DFMA(-sh, sum.hi, d);
  r = QGB_DSUB(r, QGB_DMUL(sh, sum.lo));
  const DD s = dd_fast_two_sum(sh, QGB_DDIV(r, sum.hi));
  // z = s^2
  const DD z = dd_mul(s, s);
  // q = z/3 + z^2/5 + z^3 (1/7 + z (1/9 + z (1/11 + z/13))); the
  // coefficients are generated constants (gen_log_table.py): 1/3 and 1/5 as
  // (RN(1/k), RN((1 - k RN(1/k))/k)), the others RN(1/k)
  const DD third = dd_fast_two_sum(QGB_INV3_HI, QGB_INV3_LO);
  const DD fifth = dd_fast_two_sum(QGB_INV5_HI, QGB_INV5_LO);
  const DD q1 = dd_mul(z, third);
  const DD z2 = dd_mul(z, z);
  const DD q2 = dd_mul(z2, fifth);
  double t = QGB_DADD(QGB_INV11_HI, QGB_DMUL(z.hi, QGB_INV13_HI));
  t = QGB_DADD(QGB_INV9_HI, QGB_DMUL(z.hi, t));
  t = QGB_DADD(QGB_INV7_HI, QGB_DMUL(z.hi, t));
  t = QGB_DMUL(QGB_DMUL(z2.hi, z.hi), t);
  DD q = dd_add(q1, q2);
  q = dd_add(q, DD{t, 0.0});
  // L = 2 (s + s q)
  DD L = dd_add(s, dd_mul(s, q));
  L.hi = QGB_DMUL(L.hi, 2.0);
  L.lo = QGB_DMUL(L.lo, 2.0);
  // e log 2 + log c
  double th, tl;
  logtab_get(j, th, tl);
  DD acc = dd_mul_d(DD{QGB_LOG2_HI, QGB_LOG2_LO}, (double)e);
  acc = dd_add(acc, DD{th, tl});
  acc = dd_add(acc, L);
  // round once and certify
  const DD rs = dd_two_sum(acc.hi, acc.lo);
  const double res = rs.hi;
  const double resid = rs.lo;  // value = res + resid + err
  if (res != 0.0) {
    const double up = u2d_bits(d2u(fabs(res)) + 1) - fabs(res);
    const double dn = fabs(res) - u2d_bits(d2u(fabs(res)) - 1);
    const bool toward_zero = (resid < 0) == (res > 0);
    const double half_gap = 0.5 * (toward_zero ? dn : up);
    const double bound = fabs(res) * 5.048709793414476e-29;  // 2^-94
    if (fabs(resid) + bound >= half_gap && ambiguous) *ambiguous = 1;
  }
  return res;
}

// ------------------------------------------------------------------------
// SHA-256

struct ShaConst {
  uint32_t k[64];
  uint32_t h0[8];
};

#if defined(__CUDACC__)
__constant__ ShaConst qgb_sha_dev;
#endif

// Host copy, filled by sha_const_init().
extern ShaConst qgb_sha_host;

QGB_HD uint32_t sha_k(int i)
{
#if defined(__CUDA_ARCH__)
  return qgb_sha_dev.k[i];
#else
  return qgb_sha_host.k[i];
#endif
}

QGB_HD uint32_t rotr32(uint32_t a, int c) { return (a >> c) | (a << (32 - c)); }

// One compression of a 64-byte block given as 16 big-endian words.
QGB_HD void sha256_compress(uint32_t out[8], const uint32_t in[8], const uint32_t wb[16])
{
  uint32_t w[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) w[i] = wb[i];
  uint32_t a = in[0], b = in[1], c = in[2], d = in[3], e = in[4], f = in[5], g = in[6], h = in[7];
#pragma unroll 16
  for (int i = 0; i < 64; ++i) {
    uint32_t wi;
    if (i < 16) {
      wi = w[i & 15];
    } else {
      const uint32_t w15 = w[(i - 15) & 15], w2 = w[(i - 2) & 15];
      const uint32_t s0 = rotr32(w15, 7) ^ rotr32(w15, 18) ^ (w15 >> 3);
      const uint32_t s1 = rotr32(w2, 17) ^ rotr32(w2, 19) ^ (w2 >> 10);
      wi = w[i & 15] + s0 + w[(i - 7) & 15] + s1;
      w[i & 15] = wi;
    }
    const uint32_t S1 = rotr32(e, 6) ^ rotr32(e, 11) ^ rotr32(e, 25);
    const uint32_t ch = (e & f) ^ (~e & g);
    const uint32_t t1 = h + S1 + ch + sha_k(i) + wi;
    const uint32_t S0 = rotr32(a, 2) ^ rotr32(a, 13) ^ rotr32(a, 22);
    const uint32_t maj = (a & b) ^ (a & c) ^ (b & c);
    h = g;
    g = f;
    f = e;
    e = d + t1;
    d = c;
    c = b;
    b = a;
    a = t1 + S0 + maj;
  }
  out[0] = in[0] + a;
  out[1] = in[1] + b;
  out[2] = in[2] + c;
  out[3] = in[3] + d;
  out[4] = in[4] + e;
  out[5] = in[5] + f;
  out[6] = in[6] + g;
  out[7] = in[7] + h;
}

// Byte buffer -> big-endian words.
QGB_HD void bytes_to_words(uint32_t w[16], const uint8_t* p)
{
#pragma unroll
  for (int i = 0; i < 16; ++i)
    w[i] = ((uint32_t)p[4 * i] << 24) | ((uint32_t)p[4 * i + 1] << 16) | ((uint32_t)p[4 * i + 2] << 8) |
           (uint32_t)p[4 * i + 3];
}

// Decimal digits of v into buf (no terminator); returns the length.
QGB_HD int u64_to_dec(uint8_t* buf, uint64_t v)
{
  uint8_t tmp[20];
  int n = 0;
  do {
    tmp[n++] = (uint8_t)('0' + (int)(v % 10));
    v /= 10;
  } while (v != 0);
  for (int i = 0; i < n; ++i) buf[i] = tmp[n - 1 - i];
  return n;
}

// ------------------------------------------------------------------------
// RngState

struct Rng {
  uint64_t numBytes;
  uint32_t hash[8];
  uint64_t type;
  uint64_t index;
  uint64_t cache[3];
  double gaussian;
  int32_t cacheAvail;
  int32_t gaussianAvail;
};

static const uint64_t RNG_NO_TYPE = ~(uint64_t)0;

QGB_HD void rng_import(Rng& rs, const uint32_t* v)
{
  rs.numBytes = ((uint64_t)v[0] << 32) | v[1];
  for (int i = 0; i < 8; ++i) rs.hash[i] = v[2 + i];
  rs.type = ((uint64_t)v[10] << 32) | v[11];
  rs.index = ((uint64_t)v[12] << 32) | v[13];
  for (int i = 0; i < 3; ++i) rs.cache[i] = ((uint64_t)v[14 + 2 * i] << 32) | v[15 + 2 * i];
  rs.gaussian = u2d_bits(((uint64_t)v[20] << 32) | v[21]);
  rs.cacheAvail = (int32_t)v[22];
  rs.gaussianAvail = (int32_t)v[23];
}

QGB_HD void rng_export(uint32_t* v, const Rng& rs)
{
  v[0] = (uint32_t)(rs.numBytes >> 32);
  v[1] = (uint32_t)rs.numBytes;
  for (int i = 0; i < 8; ++i) v[2 + i] = rs.hash[i];
  v[10] = (uint32_t)(rs.type >> 32);
  v[11] = (uint32_t)rs.type;
  v[12] = (uint32_t)(rs.index >> 32);
  v[13] = (uint32_t)rs.index;
  for (int i = 0; i < 3; ++i) {
    v[14 + 2 * i] = (uint32_t)(rs.cache[i] >> 32);
    v[15 + 2 * i] = (uint32_t)rs.cache[i];
  }
  const uint64_t g = d2u(rs.gaussian);
  v[20] = (uint32_t)(g >> 32);
  v[21] = (uint32_t)g;
  v[22] = (uint32_t)rs.cacheAvail;
  v[23] = (uint32_t)rs.gaussianAvail;
}

// split_rng_state(rs, rs0, sindex) (rng-state.cpp:173-201) where sindex is
// given as bytes: hash the string "[index] {sindex}" (or "[type,index] {..}")
// padded with spaces to whole 64-byte blocks, continuing rs0's hash.
// Supports strings of up to 4 blocks.
QGB_HD bool rng_split_bytes(Rng& out, const Rng& rs0, const uint8_t* sidx, int slen)
{
  uint8_t data[256];
  int n = 0;
  data[n++] = '[';
  if (rs0.type != RNG_NO_TYPE) {
    n += u64_to_dec(data + n, rs0.type);
    data[n++] = ',';
  }
  n += u64_to_dec(data + n, rs0.index);
  data[n++] = ']';
  data[n++] = ' ';
  data[n++] = '{';
  if (n + slen + 1 > 256) return false;
  for (int i = 0; i < slen; ++i) data[n++] = sidx[i];
  data[n++] = '}';
  const int nblocks = (n - 1) / 64 + 1;
  for (int i = n; i < nblocks * 64; ++i) data[i] = ' ';
  uint32_t h[8], w[16];
  bytes_to_words(w, data);
  sha256_compress(h, rs0.hash, w);
  for (int b = 1; b < nblocks; ++b) {
    bytes_to_words(w, data + 64 * b);
    sha256_compress(h, h, w);
  }
  out.numBytes = rs0.numBytes + (uint64_t)nblocks * 64;
  for (int i = 0; i < 8; ++i) out.hash[i] = h[i];
  out.type = RNG_NO_TYPE;
  out.index = 0;
  out.cache[0] = out.cache[1] = out.cache[2] = 0;
  out.gaussian = 0.0;
  out.cacheAvail = 0;
  out.gaussianAvail = 0;
  return true;
}

// RngState(rs0, (Long)sindex): the index is printed with "%ld".
QGB_HD void rng_split_long(Rng& out, const Rng& rs0, int64_t sindex)
{
  uint8_t s[24];
  int n = 0;
  uint64_t v = (uint64_t)sindex;
  if (sindex < 0) {
    s[n++] = '-';
    v = (uint64_t)(-(sindex + 1)) + 1;
  }
  n += u64_to_dec(s + n, v);
  rng_split_bytes(out, rs0, s, n);
}

// rand_gen (rng-state.cpp:203-238): three cached u64 per hash of "[index]".
// New cache block of rand_gen: SHA-256 of "[index]" (or "[type,index]")
// appended to the state, with the already advanced index; caches three of the
// four 64-bit words and returns the fourth.
// The block of an untyped state, built in registers: "[" dec(index) "]"
// (at most 22 bytes) and the 0x80 pad byte fill words 0-5 from the left,
// words 14-15 hold the message length in bits.
QGB_HD void refill_words_untyped(uint32_t w[16], uint64_t index, uint64_t numBytes)
{
  int nd = 1;
  for (uint64_t t = index; t >= 10; t /= 10) ++nd;
  uint64_t q0 = (uint64_t)'[' << 56, q1 = 0, q2 = 0;  // bytes 0-7, 8-15, 16-23, big-endian
  auto put = [&](int p, uint64_t byte) {
    const uint64_t v = byte << (56 - 8 * (p & 7));
    if (p < 8) q0 |= v;
    else if (p < 16) q1 |= v;
    else q2 |= v;
  };
  uint64_t v = index;
  for (int p = nd; p >= 1; --p) {
    put(p, '0' + v % 10);
    v /= 10;
  }
  put(nd + 1, ']');
  put(nd + 2, 0x80);
  const uint64_t bits = 8 * (numBytes + (uint64_t)(nd + 2));
  w[0] = (uint32_t)(q0 >> 32);
  w[1] = (uint32_t)q0;
  w[2] = (uint32_t)(q1 >> 32);
  w[3] = (uint32_t)q1;
  w[4] = (uint32_t)(q2 >> 32);
  w[5] = (uint32_t)q2;
#pragma unroll
  for (int i = 6; i < 14; ++i) w[i] = 0;
  w[14] = (uint32_t)(bits >> 32);
  w[15] = (uint32_t)bits;
}

QGB_HD uint64_t rng_refill(Rng& rs)
{
  uint32_t w[16], h[8];
  if (rs.type == RNG_NO_TYPE) {
    refill_words_untyped(w, rs.index, rs.numBytes);
    sha256_compress(h, rs.hash, w);
    rs.cache[0] = ((uint64_t)h[0] << 32) | h[1];
    rs.cache[1] = ((uint64_t)h[2] << 32) | h[3];
    rs.cache[2] = ((uint64_t)h[4] << 32) | h[5];
    rs.cacheAvail = 3;
    return ((uint64_t)h[6] << 32) | h[7];
  }
  uint8_t blk[64];
  for (int i = 0; i < 64; ++i) blk[i] = 0;
  int n = 0;
  blk[n++] = '[';
  if (rs.type != RNG_NO_TYPE) {
    n += u64_to_dec(blk + n, rs.type);
    blk[n++] = ',';
  }
  n += u64_to_dec(blk + n, rs.index);
  blk[n++] = ']';
  blk[n] = 0x80;
  const uint64_t bits = 8 * (rs.numBytes + (uint64_t)n);
  for (int i = 0; i < 8; ++i) blk[63 - i] = (uint8_t)(bits >> (8 * i));
  bytes_to_words(w, blk);
  sha256_compress(h, rs.hash, w);
  rs.cache[0] = ((uint64_t)h[0] << 32) | h[1];
  rs.cache[1] = ((uint64_t)h[2] << 32) | h[3];
  rs.cache[2] = ((uint64_t)h[4] << 32) | h[5];
  rs.cacheAvail = 3;
  return ((uint64_t)h[6] << 32) | h[7];
}

// Takes cache[--cacheAvail] and clears it, with constant indices (a
// run-time index would put the cache in local memory).
QGB_HD uint64_t rng_cache_pop(Rng& rs)
{
  const int k = --rs.cacheAvail;
  uint64_t r;
  if (k == 2) {
    r = rs.cache[2];
    rs.cache[2] = 0;
  } else if (k == 1) {
    r = rs.cache[1];
    rs.cache[1] = 0;
  } else {
    r = rs.cache[0];
    rs.cache[0] = 0;
  }
  return r;
}

// rand_gen (rng-state.cpp:215-238)
QGB_HD uint64_t rng_rand_gen(Rng& rs)
{
  rs.index += 1;
  if (rs.cacheAvail > 0) return rng_cache_pop(rs);
  return rng_refill(rs);
}

// u_rand_gen (rng-state.cpp:240-246): u * 2^-64 * (upper - lower) + lower.
QGB_HD double rng_u_rand_gen(Rng& rs, double upper, double lower)
{
  const uint64_t u = rng_rand_gen(rs);
  const double fac = 5.421010862427522e-20;  // 2^-64
  return QGB_DADD(QGB_DMUL(QGB_DMUL(QGB_U2D(u), fac), QGB_DSUB(upper, lower)), lower);
}

// g_rand_gen (rng-state.cpp:248-281), Marsaglia polar method.  LOG selects
// the logarithm: the device uses log_cr; the host API uses the C library's
// log like the reference.
template <bool DEVICE_LOG>
QGB_HD double rng_g_rand_gen(Rng& rs, double center, double sigma, int* ambiguous)
{
  rs.index += 1;
  if (rs.gaussianAvail) {
    rs.gaussianAvail = 0;
    return QGB_DADD(QGB_DMUL(rs.gaussian, sigma), center);
  }
  int num_try = 1;
  double v1, v2, rsq;
  do {
    v1 = rng_u_rand_gen(rs, 1.0, -1.0);
    v2 = rng_u_rand_gen(rs, 1.0, -1.0);
    rsq = QGB_DADD(QGB_DMUL(v1, v1), QGB_DMUL(v2, v2));
    num_try++;
  } while ((num_try < 10000) && (rsq >= 1.0 || rsq == 0));
  if (num_try > 9999) return 1e+10;
  double lg;
  if (DEVICE_LOG) {
    lg = log_cr(rsq, ambiguous);
  } else {
    lg = log(rsq);
  }
  const double fac = QGB_DSQRT(QGB_DDIV(QGB_DMUL(-2.0, lg), rsq));
  rs.gaussian = QGB_DMUL(v1, fac);
  rs.gaussianAvail = 1;
  return QGB_DADD(QGB_DMUL(QGB_DMUL(v2, fac), sigma), center);
}

#if defined(__CUDACC__)
// N successive g_rand_gen(rs, 0, sigma) values of each lane's own stream,
// handed to sink(i, value) in order -- the same values and the same final
// state as N calls of rng_g_rand_gen<true> -- with the SHA-256 refills of a
// warp executed together.  Called by all 32 lanes of a warp (lanes with
// active == false take part in the synchronisation only).
//
// Each lane advances its stream through the cheap steps (index increments,
// cache pops, the polar accept test, the logarithm) until it needs a new cache
// block; then every lane that is blocked computes its block at once.  Drawing
// stream by stream instead leaves the lanes' refills at different times, and a
// warp runs each lane's 64-round compression with most lanes idle.
template <int N, typename Sink>
__device__ __forceinline__ void rng_gaussians_converged(Rng& rs, double sigma, bool active, int* ambiguous,
                                                        Sink&& sink)
{
  int produced = 0;
  if (active && rs.gaussianAvail && N > 0) {  // a Gaussian cached by an earlier call comes first
    rs.index += 1;
    rs.gaussianAvail = 0;
    sink(produced++, QGB_DADD(QGB_DMUL(rs.gaussian, sigma), 0.0));
  }
  int stage = 0;  // 0: next call starts a pair; 1: v1 next; 2: v2 next
  int num_try = 1;
  double v1 = 0.0;
  bool done = !active || produced >= N;
  bool need = false;
  // take one uniform of [-1, 1) (u_rand_gen(rs, 1, -1)) into the polar step
  auto consume = [&](uint64_t u) {
    const double x = QGB_DADD(QGB_DMUL(QGB_DMUL(QGB_U2D(u), 5.421010862427522e-20), 2.0), -1.0);
    if (stage == 1) {
      v1 = x;
      stage = 2;
      return;
    }
    const double v2 = x;
    const double rsq = QGB_DADD(QGB_DMUL(v1, v1), QGB_DMUL(v2, v2));
    num_try++;
    if (num_try < 10000 && (rsq >= 1.0 || rsq == 0)) {
      stage = 1;
      return;
    }
    stage = 0;
    if (num_try > 9999) {
      sink(produced++, 1e+10);
    } else {
      const double lg = log_cr(rsq, ambiguous);
      const double fac = QGB_DSQRT(QGB_DDIV(QGB_DMUL(-2.0, lg), rsq));
      sink(produced++, QGB_DADD(QGB_DMUL(QGB_DMUL(v2, fac), sigma), 0.0));
      const double g1 = QGB_DMUL(v1, fac);
      if (produced < N) {
        rs.index += 1;  // the next g_rand_gen call returns the cached value
        sink(produced++, QGB_DADD(QGB_DMUL(g1, sigma), 0.0));
      } else {
        rs.gaussian = g1;
        rs.gaussianAvail = 1;
      }
    }
    if (produced >= N) done = true;
  };
  while (true) {
    while (!done && !need) {
      if (stage == 0) {
        rs.index += 1;  // g_rand_gen call that starts a pair
        num_try = 1;
        stage = 1;
      }
      rs.index += 1;  // rand_gen
      if (rs.cacheAvail > 0) {
        consume(rng_cache_pop(rs));
      } else {
        need = true;
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (need) {
      need = false;
      consume(rng_refill(rs));
    }
  }
}
#endif

// ------------------------------------------------------------------------
// Exactly rounded complex / matrix arithmetic in the reference's order
// (used where results must match the reference bit for bit: the random
// momentum and the hot start).

QGB_HD Cx<double> xc_mul(Cx<double> a, Cx<double> b)
{
  return cx<double>(QGB_DSUB(QGB_DMUL(a.re, b.re), QGB_DMUL(a.im, b.im)),
                    QGB_DADD(QGB_DMUL(a.re, b.im), QGB_DMUL(a.im, b.re)));
}
QGB_HD Cx<double> xc_add(Cx<double> a, Cx<double> b)
{
  return cx<double>(QGB_DADD(a.re, b.re), QGB_DADD(a.im, b.im));
}
QGB_HD Cx<double> xc_sub(Cx<double> a, Cx<double> b)
{
  return cx<double>(QGB_DSUB(a.re, b.re), QGB_DSUB(a.im, b.im));
}

QGB_HD M3<double> xm_mul(const M3<double>& x, const M3<double>& y)
{
  M3<double> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Cx<double> s = xc_mul(x.e[3 * i], y.e[j]);
      s = xc_add(s, xc_mul(x.e[3 * i + 1], y.e[3 + j]));
      s = xc_add(s, xc_mul(x.e[3 * i + 2], y.e[6 + j]));
      r.e[3 * i + j] = s;
    }
  return r;
}

// matrix-hmc.h:11-74 with exactly rounded operations.
QGB_HD void x_normalize_row(Cx<double>* p)
{
  double norm = 0;
  for (int k = 0; k < 3; ++k) {
    norm = QGB_DADD(norm, QGB_DMUL(p[k].re, p[k].re));
    norm = QGB_DADD(norm, QGB_DMUL(p[k].im, p[k].im));
  }
  if (!(norm == 1.0)) {
    norm = QGB_DDIV(1.0, QGB_DSQRT(norm));
    for (int k = 0; k < 3; ++k) {
      p[k].re = QGB_DMUL(p[k].re, norm);
      p[k].im = QGB_DMUL(p[k].im, norm);
    }
  }
}
QGB_HD void x_unitarize(M3<double>& m)
{
  Cx<double>* p1 = m.e;
  Cx<double>* p2 = m.e + 3;
  Cx<double>* p3 = m.e + 6;
  x_normalize_row(p1);
  Cx<double> c = cx<double>(0.0, 0.0);
  for (int k = 0; k < 3; ++k) c = xc_add(c, xc_mul(cx<double>(p1[k].re, -p1[k].im), p2[k]));
  if (!(c.re == 0.0 && c.im == 0.0)) {
    for (int k = 0; k < 3; ++k) p2[k] = xc_sub(p2[k], xc_mul(c, p1[k]));
  }
  x_normalize_row(p2);
  Cx<double> t;
  t = xc_sub(xc_mul(p1[1], p2[2]), xc_mul(p1[2], p2[1]));
  p3[0] = cx<double>(t.re, -t.im);
  t = xc_sub(xc_mul(p1[2], p2[0]), xc_mul(p1[0], p2[2]));
  p3[1] = cx<double>(t.re, -t.im);
  t = xc_sub(xc_mul(p1[0], p2[1]), xc_mul(p1[1], p2[0]));
  p3[2] = cx<double>(t.re, -t.im);
}

// matrix-hmc.h:155-167 with exactly rounded operations.
QGB_HD M3<double> x_exp_taylor20(const M3<double>& a)
{
  M3<double> t2 = a, t3;
  for (int j = 20; j > 1; --j) {
    const double f = QGB_DDIV(1.0, (double)j);
    for (int i = 0; i < 9; ++i) {
      t3.e[i] = cx<double>(QGB_DMUL(f, t2.e[i].re), QGB_DMUL(f, t2.e[i].im));
      if (i % 4 == 0) t3.e[i].re = QGB_DADD(1.0, t3.e[i].re);
    }
    t2 = xm_mul(a, t3);
  }
  t3 = t2;
  for (int i = 0; i < 9; i += 4) t3.e[i].re = QGB_DADD(1.0, t3.e[i].re);
  return t3;
}

// make_anti_hermitian_matrix (matrix-hmc.h:76-106); inv_sqrt3 = 1/sqrt(3).
QGB_HD M3<double> x_make_anti_hermitian(const double b[8], double inv_sqrt3)
{
  M3<double> m;
  const double s3 = QGB_DMUL(inv_sqrt3, b[7]);
  m.e[0] = cx<double>(0.0, QGB_DADD(b[2], s3));
  m.e[4] = cx<double>(0.0, QGB_DADD(-b[2], s3));
  m.e[8] = cx<double>(0.0, QGB_DMUL(-2.0, s3));
  m.e[1] = cx<double>(b[1], b[0]);
  m.e[2] = cx<double>(b[4], b[3]);
  m.e[3] = cx<double>(-b[1], b[0]);
  m.e[5] = cx<double>(b[6], b[5]);
  m.e[6] = cx<double>(-b[4], b[3]);
  m.e[7] = cx<double>(-b[6], b[5]);
  return m;
}

}  // namespace qgb
