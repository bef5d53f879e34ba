/* qgauge_oracle.c -- CPU restatement of Qlattice's pure-gauge SU(3) hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of
 * it.  Written from the reference's published algorithm; each function cites
 * the reference file:line it restates (paths inside the Qlattice project).
 *
 * Floating-point order follows the reference so that results agree to the
 * last bit where the reference is itself deterministic: complex products are
 * (ac - bd, ad + bc), matrix products sum k = 0, 1, 2 from zero, Wilson lines
 * multiply left to right from the unit matrix.  Build with
 * -ffp-contract=off (no fused multiply-add), like the x86-64 baseline build
 * of the reference. */
#include "qgauge_oracle.h"

#include <math.h>
#include <quadmath.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* complex 3x3 algebra (qlat-utils mat-vec.h:115, matrix.h:45-260)     */

typedef struct {
  double re, im;
} cd;
typedef struct {
  cd p[9];
} cm;

static inline cd c_add(cd a, cd b) { return (cd){a.re + b.re, a.im + b.im}; }
static inline cd c_sub(cd a, cd b) { return (cd){a.re - b.re, a.im - b.im}; }
static inline cd c_mul(cd a, cd b)
{
  return (cd){a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
static inline cd c_conj(cd a) { return (cd){a.re, -a.im}; }
static inline cd c_rscale(double s, cd a) { return (cd){s * a.re, s * a.im}; }

static cm m_zero(void)
{
  cm r;
  memset(&r, 0, sizeof(r));
  return r;
}
static cm m_unit(void)
{
  cm r = m_zero();
  r.p[0].re = r.p[4].re = r.p[8].re = 1.0;
  return r;
}
/* matrix.h:45-61: ret[i][j] = sum_k x[i][k] y[k][j], accumulated from 0 */
static cm m_mul(const cm* x, const cm* y)
{
  cm r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      cd s = {0.0, 0.0};
      for (int k = 0; k < 3; ++k) {
        s = c_add(s, c_mul(x->p[i * 3 + k], y->p[k * 3 + j]));
      }
      r.p[i * 3 + j] = s;
    }
  }
  return r;
}
static cm m_adj(const cm* x)
{
  cm r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.p[i * 3 + j] = c_conj(x->p[j * 3 + i]);
  return r;
}
static void m_add_to(cm* acc, const cm* x)
{
  for (int i = 0; i < 9; ++i) acc->p[i] = c_add(acc->p[i], x->p[i]);
}
static void m_sub_to(cm* acc, const cm* x)
{
  for (int i = 0; i < 9; ++i) acc->p[i] = c_sub(acc->p[i], x->p[i]);
}
static cm m_rscale(double s, const cm* x)
{
  cm r;
  for (int i = 0; i < 9; ++i) r.p[i] = c_rscale(s, x->p[i]);
  return r;
}
/* matrix.h:220-227 */
static cd m_trace(const cm* x)
{
  cd s = {0.0, 0.0};
  for (int i = 0; i < 3; ++i) s = c_add(s, x->p[i * 4]);
  return s;
}
/* matrix.h:230-240: tr(x y) = sum_i sum_j x[i][j] y[j][i] */
static cd m_trace2(const cm* x, const cm* y)
{
  cd s = {0.0, 0.0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s = c_add(s, c_mul(x->p[i * 3 + j], y->p[j * 3 + i]));
  return s;
}

/* matrix-hmc.h:11-74 (Gram-Schmidt unitarisation, third row = (r1 x r2)^*) */
static void normalize_row(cd* p)
{
  double norm = 0;
  const double* r = (const double*)p;
  for (int i = 0; i < 6; ++i) norm += r[i] * r[i];
  if (!(norm == 1.0)) {
    norm = 1.0 / sqrt(norm);
    double* w = (double*)p;
    for (int i = 0; i < 6; ++i) w[i] *= norm;
  }
}
static void unitarize_cm(cm* m)
{
  cd* p1 = m->p;
  cd* p2 = m->p + 3;
  cd* p3 = m->p + 6;
  normalize_row(p1);
  cd c = {0.0, 0.0};
  for (int i = 0; i < 3; ++i) c = c_add(c, c_mul(c_conj(p1[i]), p2[i]));
  if (!(c.re == 0.0 && c.im == 0.0)) {
    for (int i = 0; i < 3; ++i) p2[i] = c_sub(p2[i], c_mul(c, p1[i]));
  }
  normalize_row(p2);
  p3[0] = c_conj(c_sub(c_mul(p1[1], p2[2]), c_mul(p1[2], p2[1])));
  p3[1] = c_conj(c_sub(c_mul(p1[2], p2[0]), c_mul(p1[0], p2[2])));
  p3[2] = c_conj(c_sub(c_mul(p1[0], p2[1]), c_mul(p1[1], p2[0])));
}

/* matrix-hmc.h:155-167: Horner form of the order-20 Taylor series */
static cm make_matrix_exp(const cm* a, int max_order)
{
  const cm unit = m_unit();
  cm t2 = *a;
  cm t3;
  for (int j = max_order; j > 1; --j) {
    cm s = m_rscale(1.0 / j, &t2);
    t3 = unit;
    m_add_to(&t3, &s);
    t2 = m_mul(a, &t3);
  }
  t3 = unit;
  m_add_to(&t3, &t2);
  return t3;
}

/* matrix-hmc.h:179-188 */
static cm matrix_evolve(const cm* gf, const cm* gm, double step)
{
  cm t = m_rscale(step, gm);
  cm e = make_matrix_exp(&t, 20);
  t = m_mul(&e, gf);
  unitarize_cm(&t);
  return t;
}

/* matrix-hmc.h:202-213 */
static cm make_tr_less_anti_herm(const cm* m)
{
  cm ad = m_adj(m);
  cm r = *m;
  m_sub_to(&r, &ad);
  r = m_rscale(0.5, &r);
  double* p = (double*)r.p;
  const double c = (p[1] + p[9] + p[17]) / 3.0;
  p[1] -= c;
  p[9] -= c;
  p[17] -= c;
  return r;
}

/* matrix-hmc.h:76-106 */
static cm make_anti_hermitian_matrix(const double b[8])
{
  cm m;
  double* p = (double*)m.p;
  const double s3 = (1.0 / sqrt(3.0)) * b[7];
  p[0] = 0.0;
  p[8] = 0.0;
  p[16] = 0.0;
  p[1] = b[2] + s3;
  p[9] = -b[2] + s3;
  p[17] = -2.0 * s3;
  p[2] = b[1];
  p[3] = b[0];
  p[4] = b[4];
  p[5] = b[3];
  p[6] = -b[1];
  p[7] = b[0];
  p[10] = b[6];
  p[11] = b[5];
  p[12] = -b[4];
  p[13] = b[3];
  p[14] = -b[6];
  p[15] = b[5];
  return m;
}

/* matrix-hmc.h:144-152 */
static double neg_half_tr_square(const cm* m)
{
  const double* p = (const double*)m->p;
  return p[3] * p[3] + p[2] * p[2] + (p[1] - p[9]) * (p[1] - p[9]) * 0.25 + p[5] * p[5] +
         p[4] * p[4] + p[11] * p[11] + p[10] * p[10] + p[17] * p[17] * 0.75;
}

/* ------------------------------------------------------------------ */
/* SHA-256 (FIPS 180-4) as used by qlat-utils lib/sha256.cpp:71-507     */
/* The round constants are derived here from their definition (first  */
/* 32 fractional bits of the cube roots of the first 64 primes, and of */
/* the square roots of the first 8 primes for the initial hash).        */

static uint32_t K256[64];
static uint32_t H256[8];
static int sha_ready = 0;

static void sha_init_constants(void)
{
  if (sha_ready) return;
  int primes[64];
  int n = 0;
  for (int c = 2; n < 64; ++c) {
    int is_p = 1;
    for (int d = 2; d * d <= c; ++d)
      if (c % d == 0) {
        is_p = 0;
        break;
      }
    if (is_p) primes[n++] = c;
  }
  for (int i = 0; i < 64; ++i) {
    /* k = floor(cbrt(p) * 2^32) = max k with k^3 <= p * 2^96 */
    unsigned __int128 target = ((unsigned __int128)primes[i]) << 96;
    uint64_t lo = 0, hi = (uint64_t)1 << 36;
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) / 2;
      unsigned __int128 m3 = (unsigned __int128)mid * mid * mid;
      if (m3 <= target) lo = mid; else hi = mid;
    }
    K256[i] = (uint32_t)lo;
  }
  for (int i = 0; i < 8; ++i) {
    unsigned __int128 target = ((unsigned __int128)primes[i]) << 64;
    uint64_t lo = 0, hi = (uint64_t)1 << 36;
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) / 2;
      unsigned __int128 m2 = (unsigned __int128)mid * mid;
      if (m2 <= target) lo = mid; else hi = mid;
    }
    H256[i] = (uint32_t)lo;
  }
  sha_ready = 1;
}

static inline uint32_t rotr(uint32_t a, int c) { return (a >> c) | (a << (32 - c)); }

void or_sha256_initial(uint32_t h[8])
{
  sha_init_constants();
  memcpy(h, H256, 32);
}

/* sha256.cpp:71-420: one 64-byte block, big-endian words */
void or_sha256_block(uint32_t out[8], const uint32_t in[8], const uint8_t data[64])
{
  sha_init_constants();
  uint32_t w[64];
  for (int i = 0; i < 16; ++i) {
    w[i] = ((uint32_t)data[4 * i] << 24) | ((uint32_t)data[4 * i + 1] << 16) |
           ((uint32_t)data[4 * i + 2] << 8) | (uint32_t)data[4 * i + 3];
  }
  for (int i = 16; i < 64; ++i) {
    const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
    const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
    w[i] = w[i - 16] + s0 + w[i - 7] + s1;
  }
  uint32_t a = in[0], b = in[1], c = in[2], d = in[3], e = in[4], f = in[5], g = in[6], h = in[7];
  for (int i = 0; i < 64; ++i) {
    const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
    const uint32_t ch = (e & f) ^ (~e & g);
    const uint32_t t1 = h + S1 + ch + K256[i] + w[i];
    const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
    const uint32_t maj = (a & b) ^ (a & c) ^ (b & c);
    const uint32_t t2 = S0 + maj;
    h = g;
    g = f;
    f = e;
    e = d + t1;
    d = c;
    c = b;
    b = a;
    a = t1 + t2;
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

/* sha256.cpp:422-495: whole blocks, then padding carrying the total bit
 * length (num_bytes already hashed + input_size) */
void or_sha256_final(uint32_t out[8], const uint32_t in[8], uint64_t num_bytes,
                     const uint8_t* input, uint64_t input_size)
{
  uint32_t h[8];
  memcpy(h, in, 32);
  uint64_t nb = input_size / 64;
  for (uint64_t i = 0; i < nb; ++i) or_sha256_block(h, h, input + 64 * i);
  uint8_t buf[128];
  memset(buf, 0, sizeof(buf));
  const uint64_t rem = input_size - nb * 64;
  memcpy(buf, input + nb * 64, rem);
  buf[rem] = 0x80;
  const int nblk = (rem + 1 + 8 <= 64) ? 1 : 2;
  const uint64_t bits = 8 * (num_bytes + input_size);
  for (int i = 0; i < 8; ++i) buf[nblk * 64 - 1 - i] = (uint8_t)(bits >> (8 * i));
  or_sha256_block(h, h, buf);
  if (nblk == 2) or_sha256_block(h, h, buf + 64);
  memcpy(out, h, 32);
}

/* ------------------------------------------------------------------ */
/* RngState (rng-state.cpp:150-281)                                     */

static const uint64_t U64MAX = ~(uint64_t)0;
static int g_log_mode = 0;

void or_set_log_mode(int mode) { g_log_mode = mode; }

static double rng_log(double x)
{
  if (g_log_mode == 1) return (double)logq((__float128)x);
  return log(x);
}

void or_rng_reset(or_rng* rs)
{
  memset(rs, 0, sizeof(*rs));
  or_sha256_initial(rs->hash);
  rs->type = U64MAX;
}

/* rng-state.cpp:173-201: hash of "[index] {sindex}" (or "[type,index] {..}")
 * padded with spaces to whole 64-byte blocks */
void or_rng_split(or_rng* out, const or_rng* rs0, const char* sindex)
{
  char data[1024];
  int len;
  if (rs0->type == U64MAX) {
    len = snprintf(data, sizeof(data) - 64, "[%lu] {%s}", (unsigned long)rs0->index, sindex);
  } else {
    len = snprintf(data, sizeof(data) - 64, "[%lu,%lu] {%s}", (unsigned long)rs0->type,
                   (unsigned long)rs0->index, sindex);
  }
  const int nblocks = (len - 1) / 64 + 1;
  for (int i = len; i < nblocks * 64; ++i) data[i] = ' ';
  uint32_t h[8];
  or_sha256_block(h, rs0->hash, (const uint8_t*)data);
  for (int i = 1; i < nblocks; ++i) or_sha256_block(h, h, (const uint8_t*)data + 64 * i);
  const uint64_t nbytes = rs0->numBytes + (uint64_t)nblocks * 64;
  memset(out, 0, sizeof(*out));
  memcpy(out->hash, h, 32);
  out->numBytes = nbytes;
  out->type = U64MAX;
}

void or_rng_seed(or_rng* rs, const char* seed)
{
  or_rng r;
  or_rng_reset(&r);
  or_rng_split(rs, &r, seed);
}

void or_rng_split_long(or_rng* out, const or_rng* rs0, int64_t sindex)
{
  char s[32];
  snprintf(s, sizeof(s), "%ld", (long)sindex);
  or_rng_split(out, rs0, s);
}

/* rng-state.cpp:203-238 */
uint64_t or_rand_gen(or_rng* rs)
{
  rs->index += 1;
  if (rs->cacheAvail > 0) {
    rs->cacheAvail -= 1;
    const uint64_t r = rs->cache[rs->cacheAvail];
    rs->cache[rs->cacheAvail] = 0;
    return r;
  }
  char in[64];
  int len;
  if (rs->type == U64MAX) {
    len = snprintf(in, sizeof(in), "[%lu]", (unsigned long)rs->index);
  } else {
    len = snprintf(in, sizeof(in), "[%lu,%lu]", (unsigned long)rs->type, (unsigned long)rs->index);
  }
  uint32_t h[8];
  or_sha256_final(h, rs->hash, rs->numBytes, (const uint8_t*)in, (uint64_t)len);
  rs->cache[0] = ((uint64_t)h[0] << 32) | h[1];
  rs->cache[1] = ((uint64_t)h[2] << 32) | h[3];
  rs->cache[2] = ((uint64_t)h[4] << 32) | h[5];
  rs->cacheAvail = 3;
  return ((uint64_t)h[6] << 32) | h[7];
}

/* rng-state.cpp:240-246 */
double or_u_rand_gen(or_rng* rs, double upper, double lower)
{
  const uint64_t u = or_rand_gen(rs);
  const double fac = 1.0 / (256.0 * 256.0 * 256.0 * 256.0) / (256.0 * 256.0 * 256.0 * 256.0);
  return (double)u * fac * (upper - lower) + lower;
}

/* rng-state.cpp:248-281: Marsaglia polar method, one cached partner */
double or_g_rand_gen(or_rng* rs, double center, double sigma)
{
  rs->index += 1;
  if (rs->gaussianAvail) {
    rs->gaussianAvail = 0;
    return rs->gaussian * sigma + center;
  }
  int num_try = 1;
  double v1, v2, rsq;
  do {
    v1 = or_u_rand_gen(rs, 1.0, -1.0);
    v2 = or_u_rand_gen(rs, 1.0, -1.0);
    rsq = v1 * v1 + v2 * v2;
    num_try++;
  } while ((num_try < 10000) && (rsq >= 1.0 || rsq == 0));
  if (num_try > 9999) return 1e+10;
  const double fac = sqrt(-2.0 * rng_log(rsq) / rsq);
  rs->gaussian = v1 * fac;
  rs->gaussianAvail = 1;
  return v2 * fac * sigma + center;
}

/* rng-state.cpp:61-103 */
void or_rng_export(uint32_t v[24], const or_rng* rs)
{
  v[0] = (uint32_t)(rs->numBytes >> 32);
  v[1] = (uint32_t)rs->numBytes;
  for (int i = 0; i < 8; ++i) v[2 + i] = rs->hash[i];
  v[10] = (uint32_t)(rs->type >> 32);
  v[11] = (uint32_t)rs->type;
  v[12] = (uint32_t)(rs->index >> 32);
  v[13] = (uint32_t)rs->index;
  for (int i = 0; i < 3; ++i) {
    v[14 + 2 * i] = (uint32_t)(rs->cache[i] >> 32);
    v[15 + 2 * i] = (uint32_t)rs->cache[i];
  }
  uint64_t g;
  memcpy(&g, &rs->gaussian, 8);
  v[20] = (uint32_t)(g >> 32);
  v[21] = (uint32_t)g;
  v[22] = (uint32_t)rs->cacheAvail;
  v[23] = (uint32_t)rs->gaussianAvail;
}

void or_rng_import(or_rng* rs, const uint32_t v[24])
{
  rs->numBytes = ((uint64_t)v[0] << 32) | v[1];
  for (int i = 0; i < 8; ++i) rs->hash[i] = v[2 + i];
  rs->type = ((uint64_t)v[10] << 32) | v[11];
  rs->index = ((uint64_t)v[12] << 32) | v[13];
  for (int i = 0; i < 3; ++i) rs->cache[i] = ((uint64_t)v[14 + 2 * i] << 32) | v[15 + 2 * i];
  const uint64_t g = ((uint64_t)v[20] << 32) | v[21];
  memcpy(&rs->gaussian, &g, 8);
  rs->cacheAvail = (int32_t)v[22];
  rs->gaussianAvail = (int32_t)v[23];
}

/* matrix-hmc.h:125-142 */
static cm make_g_rand_anti_hermitian_matrix(or_rng* rs, double sigma)
{
  const double s = sigma / sqrt(2.0);
  double a[8];
  for (int i = 0; i < 8; ++i) a[i] = or_g_rand_gen(rs, 0.0, s);
  return make_anti_hermitian_matrix(a);
}

/* ------------------------------------------------------------------ */
/* lattice geometry: x fastest (coordinate.h:182-188), periodic          */

typedef struct {
  int d[4];
  long vol;
} geo_t;

static geo_t mk_geo(const int dims[4])
{
  geo_t g;
  for (int i = 0; i < 4; ++i) g.d[i] = dims[i];
  g.vol = (long)dims[0] * dims[1] * dims[2] * dims[3];
  return g;
}
static inline void coor_from_index(const geo_t* g, long idx, int x[4])
{
  for (int i = 0; i < 4; ++i) {
    x[i] = (int)(idx % g->d[i]);
    idx /= g->d[i];
  }
}
static inline long index_from_coor(const geo_t* g, const int x[4])
{
  int y[4];
  for (int i = 0; i < 4; ++i) y[i] = ((x[i] % g->d[i]) + g->d[i]) % g->d[i];
  return (((long)y[3] * g->d[2] + y[2]) * g->d[1] + y[1]) * g->d[0] + y[0];
}
static inline cm get_link(const double* gf, const geo_t* g, const int x[4], int mu)
{
  cm m;
  memcpy(&m, gf + (index_from_coor(g, x) * 4 + mu) * 18, sizeof(cm));
  return m;
}
static inline void put_link(double* gf, long idx, int mu, const cm* m)
{
  memcpy(gf + (idx * 4 + mu) * 18, m, sizeof(cm));
}

/* qcd-acc.h:23-41: ordered product along a path; dir < 0 means the link
 * -dir-1 traversed backwards (its adjoint, one site back) */
static cm wilson_line(const double* gf, const geo_t* g, const int x0[4], const int* path, int n)
{
  cm ret = m_unit();
  int x[4] = {x0[0], x0[1], x0[2], x0[3]};
  for (int i = 0; i < n; ++i) {
    const int dir = path[i];
    if (dir >= 0) {
      cm l = get_link(gf, g, x, dir);
      ret = m_mul(&ret, &l);
      x[dir] += 1;
    } else {
      x[-dir - 1] -= 1;
      cm l = get_link(gf, g, x, -dir - 1);
      cm la = m_adj(&l);
      ret = m_mul(&ret, &la);
    }
  }
  return ret;
}

/* qcd-acc.h:152-165 */
static cm plaq_staple(const double* gf, const geo_t* g, const int x[4], int mu)
{
  cm acc = m_zero();
  for (int nu = -4; nu < 4; ++nu) {
    if (nu == mu || -nu - 1 == mu) continue;
    const int path[3] = {nu, mu, -nu - 1};
    cm w = wilson_line(gf, g, x, path, 3);
    m_add_to(&acc, &w);
  }
  return acc;
}

/* hmc.cpp:27-46 */
static cm rect_staple(const double* gf, const geo_t* g, const int x[4], int mu)
{
  cm acc = m_zero();
  for (int nu = -4; nu < 4; ++nu) {
    if (nu == mu || -nu - 1 == mu) continue;
    const int p1[5] = {nu, nu, mu, -nu - 1, -nu - 1};
    const int p2[5] = {nu, mu, mu, -nu - 1, -mu - 1};
    const int p3[5] = {-mu - 1, nu, mu, mu, -nu - 1};
    cm w = wilson_line(gf, g, x, p1, 5);
    m_add_to(&acc, &w);
    w = wilson_line(gf, g, x, p2, 5);
    m_add_to(&acc, &w);
    w = wilson_line(gf, g, x, p3, 5);
    m_add_to(&acc, &w);
  }
  return acc;
}

/* hmc.cpp:48-75 */
static cm force_site(const double* gf, const geo_t* g, const int x[4], int mu, double beta, double c1)
{
  cm acc = m_zero();
  cm ps = plaq_staple(gf, g, x, mu);
  cm t = m_rscale(1.0 - 8.0 * c1, &ps);
  m_add_to(&acc, &t);
  if (c1 != 0.0) {
    cm rs = rect_staple(gf, g, x, mu);
    t = m_rscale(c1, &rs);
    m_add_to(&acc, &t);
  }
  cm ad = m_adj(&acc);
  cm u = get_link(gf, g, x, mu);
  cm prod = m_mul(&u, &ad);
  cm f = m_rscale(-beta / 3.0, &prod);
  return make_tr_less_anti_herm(&f);
}

/* ------------------------------------------------------------------ */
/* field operations                                                     */

void or_set_unit(double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  const cm u = m_unit();
  for (long i = 0; i < g.vol; ++i)
    for (int mu = 0; mu < 4; ++mu) put_link(gf, i, mu, &u);
}

/* qcd-utils.cpp:47-69 (per-site RngState(rs, gindex)) */
void or_set_rand_gauge_momentum(double* gm, const int dims[4], const or_rng* rs, double sigma)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    or_rng rsi;
    or_rng_split_long(&rsi, rs, i);
    for (int mu = 0; mu < 4; ++mu) {
      cm m = make_g_rand_anti_hermitian_matrix(&rsi, sigma);
      put_link(gm, i, mu, &m);
    }
  }
}

/* qcd-utils.cpp:71-92 */
void or_set_g_rand_color_matrix_field(double* gf, const int dims[4], const or_rng* rs, double sigma,
                                      int n_step)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    or_rng rsi;
    or_rng_split_long(&rsi, rs, i);
    for (int mu = 0; mu < 4; ++mu) {
      cm a = make_g_rand_anti_hermitian_matrix(&rsi, sigma);
      cm v = make_matrix_exp(&a, 20);
      unitarize_cm(&v);
      for (int k = 1; k < n_step; ++k) {
        cm b = make_g_rand_anti_hermitian_matrix(&rsi, sigma);
        cm e = make_matrix_exp(&b, 20);
        unitarize_cm(&e);
        v = m_mul(&v, &e);
      }
      put_link(gf, i, mu, &v);
    }
  }
}

/* qcd.cpp:81-129: mean of Re Tr U_P / 3 over the 6 planes */
double or_gf_avg_plaq(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double total = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    cm v[4], vms[4][4];
    for (int m = 0; m < 4; ++m) v[m] = get_link(gf, &g, x, m);
    for (int m = 0; m < 4; ++m) {
      int y[4] = {x[0], x[1], x[2], x[3]};
      y[m] += 1;
      for (int n = 0; n < 4; ++n) vms[m][n] = get_link(gf, &g, y, n);
    }
    double sum = 0.0;
    for (int m1 = 0; m1 < 3; ++m1) {
      for (int m2 = m1 + 1; m2 < 4; ++m2) {
        cm a = m_mul(&v[m1], &vms[m1][m2]);
        cm b = m_mul(&v[m2], &vms[m2][m1]);
        cm bd = m_adj(&b);
        cm c = m_mul(&a, &bd);
        sum += m_trace(&c).re / 3;
      }
    }
    sum *= 2.0 / (4 * 3);
    total += sum;
  }
  return total / (double)g.vol;
}

/* hmc.cpp:151-173 */
double or_gm_hamilton_node(const double* gm, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double sum = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    double s = 0.0;
    for (int mu = 0; mu < 4; ++mu) {
      cm m;
      memcpy(&m, gm + (i * 4 + mu) * 18, sizeof(cm));
      s += neg_half_tr_square(&m);
    }
    sum += s;
  }
  return sum;
}

/* hmc.cpp:203-226 */
double or_gf_sum_re_tr_plaq(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double sum = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    double s = 0.0;
    for (int mu = 0; mu < 3; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int path[4] = {mu, nu, -mu - 1, -nu - 1};
        cm w = wilson_line(gf, &g, x, path, 4);
        s += m_trace(&w).re - 3.0;
      }
    sum += s;
  }
  return sum;
}

/* hmc.cpp:228-252 */
double or_gf_sum_re_tr_rect(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double sum = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    double s = 0.0;
    for (int mu = 0; mu < 3; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int p1[6] = {mu, mu, nu, -mu - 1, -mu - 1, -nu - 1};
        cm w = wilson_line(gf, &g, x, p1, 6);
        s += m_trace(&w).re - 3.0;
        const int p2[6] = {nu, nu, mu, -nu - 1, -nu - 1, -mu - 1};
        w = wilson_line(gf, &g, x, p2, 6);
        s += m_trace(&w).re - 3.0;
      }
    sum += s;
  }
  return sum;
}

/* hmc.cpp:254-277 */
double or_gf_hamilton_node(const double* gf, const int dims[4], double beta, double c1)
{
  const double sp = or_gf_sum_re_tr_plaq(gf, dims);
  const double sr = c1 == 0.0 ? 0.0 : or_gf_sum_re_tr_rect(gf, dims);
  return -beta / 3.0 * ((1.0 - 8.0 * c1) * sp + c1 * sr);
}

/* hmc.cpp:446-490 */
void or_set_gm_force(double* gm_force, const double* gf, const int dims[4], double beta, double c1)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int mu = 0; mu < 4; ++mu) {
      cm f = force_site(gf, &g, x, mu, beta, c1);
      put_link(gm_force, i, mu, &f);
    }
  }
}

/* hmc.cpp:311-328 */
void or_gf_evolve(double* gf, const double* gm, const int dims[4], double step_size)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    for (int mu = 0; mu < 4; ++mu) {
      cm u, p;
      memcpy(&u, gf + (i * 4 + mu) * 18, sizeof(cm));
      memcpy(&p, gm + (i * 4 + mu) * 18, sizeof(cm));
      cm r = matrix_evolve(&u, &p, step_size);
      put_link(gf, i, mu, &r);
    }
  }
}

/* qcd.cpp:346-359 */
void or_unitarize_field(double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  for (long i = 0; i < g.vol * 4; ++i) {
    cm u;
    memcpy(&u, gf + i * 18, sizeof(cm));
    unitarize_cm(&u);
    memcpy(gf + i * 18, &u, sizeof(cm));
  }
}

static void field_scale(double* f, long n, double s)
{
  for (long i = 0; i < n; ++i) f[i] *= s;
}

/* wilson-flow.cpp:29-50: Luescher RK3 with Z = force at beta = 3 */
void or_gf_wilson_flow_step(double* gf, const int dims[4], double epsilon, double c1)
{
  const geo_t g = mk_geo(dims);
  const long n = g.vol * 72;
  double* z = (double*)malloc(n * sizeof(double));
  double* zp = (double*)malloc(n * sizeof(double));
  or_set_gm_force(z, gf, dims, 3.0, c1);
  field_scale(z, n, 1.0 / 4.0);
  or_gf_evolve(gf, z, dims, epsilon);
  double* t = z;
  z = zp;
  zp = t;
  field_scale(zp, n, 17.0 / 9.0);
  or_set_gm_force(z, gf, dims, 3.0, c1);
  field_scale(z, n, 8.0 / 9.0);
  for (long i = 0; i < n; ++i) z[i] -= zp[i];
  or_gf_evolve(gf, z, dims, epsilon);
  t = z;
  z = zp;
  zp = t;
  or_set_gm_force(z, gf, dims, 3.0, c1);
  field_scale(z, n, 3.0 / 4.0);
  for (long i = 0; i < n; ++i) z[i] -= zp[i];
  or_gf_evolve(gf, z, dims, epsilon);
  free(z);
  free(zp);
}

/* wilson-flow.cpp:19-27 */
void or_gf_wilson_flow_step_euler(double* gf, const int dims[4], double epsilon, double c1)
{
  const geo_t g = mk_geo(dims);
  double* z = (double*)malloc(g.vol * 72 * sizeof(double));
  or_set_gm_force(z, gf, dims, 3.0, c1);
  or_gf_evolve(gf, z, dims, epsilon);
  free(z);
}

/* qcd-acc.h:135-150 */
static cm clover_leaf(const double* gf, const geo_t* g, const int x[4], int mu, int nu)
{
  cm m = m_zero();
  const int p1[4] = {mu, nu, -mu - 1, -nu - 1};
  const int p2[4] = {-mu - 1, -nu - 1, mu, nu};
  const int p3[4] = {nu, -mu - 1, -nu - 1, mu};
  const int p4[4] = {-nu - 1, mu, nu, -mu - 1};
  cm w = wilson_line(gf, g, x, p1, 4);
  m_add_to(&m, &w);
  w = wilson_line(gf, g, x, p2, 4);
  m_add_to(&m, &w);
  w = wilson_line(gf, g, x, p3, 4);
  m_add_to(&m, &w);
  w = wilson_line(gf, g, x, p4, 4);
  m_add_to(&m, &w);
  return m_rscale(0.25, &m);
}

/* wilson-flow.cpp:99-129: sum over mu<nu of -Tr(G_mu_nu^2), G = TA(clover) */
void or_gf_energy_density_field(double* fd, const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    double s = 0.0;
    for (int mu = 0; mu < 3; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        cm c = clover_leaf(gf, &g, x, mu, nu);
        cm gmn = make_tr_less_anti_herm(&c);
        s += -m_trace2(&gmn, &gmn).re;
      }
    fd[i] = s;
  }
}

/* wilson-flow.cpp:131-141 */
double or_gf_energy_density(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double* fd = (double*)malloc(g.vol * sizeof(double));
  or_gf_energy_density_field(fd, gf, dims);
  double s = 0.0;
  for (long i = 0; i < g.vol; ++i) s += fd[i];
  free(fd);
  return s / (double)g.vol;
}

/* qcd.cpp:64-79 and 515-534: clover-leaf topological charge density */
void or_clf_topology_field(double* topf, const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  const double PI = 3.141592653589793;
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    const int pl[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    cm arr[6];
    for (int k = 0; k < 6; ++k) {
      cm v = clover_leaf(gf, &g, x, pl[k][0], pl[k][1]);
      cm va = m_adj(&v);
      cm d = v;
      m_sub_to(&d, &va);
      arr[k] = m_rscale(0.5, &d);
    }
    const double fac = -1.0 / (4.0 * PI * PI);
    double sum = 0.0;
    cm t = m_mul(&arr[1], &arr[4]);
    sum -= m_trace(&t).re;
    t = m_mul(&arr[2], &arr[3]);
    sum += m_trace(&t).re;
    t = m_mul(&arr[5], &arr[0]);
    sum += m_trace(&t).re;
    topf[i] = fac * sum;
  }
}

/* qcd.cpp:11-31: the four m x n leaves at x in the (mu, nu) plane, times 1/4;
 * each path of qcd-acc.h:23-41 with direction counts (m, n, m, n) expanded
 * into unit steps */
static cm clover_leaf_mn(const double* gf, const geo_t* g, const int x[4], int mu, int m, int nu, int n)
{
  const int dirs[4][4] = {{mu, nu, -mu - 1, -nu - 1},
                          {-mu - 1, -nu - 1, mu, nu},
                          {nu, -mu - 1, -nu - 1, mu},
                          {-nu - 1, mu, nu, -mu - 1}};
  const int reps[4][4] = {{m, n, m, n}, {m, n, m, n}, {n, m, n, m}, {n, m, n, m}};
  cm acc = m_zero();
  for (int l = 0; l < 4; ++l) {
    int path[32];
    int len = 0;
    for (int i = 0; i < 4; ++i)
      for (int r = 0; r < reps[l][i]; ++r) path[len++] = dirs[l][i];
    cm w = wilson_line(gf, g, x, path, len);
    m_add_to(&acc, &w);
  }
  return m_rscale(0.25, &acc);
}

/* qcd.cpp:64-79 on the six planes' leaves of qcd.cpp:536-568 (m != n: the
 * average of the m x n and n x m leaves) */
static double clf_topology_density_mn(const double* gf, const geo_t* g, const int x[4], int m, int n)
{
  const int pl[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  const double PI = 3.141592653589793;
  cm arr[6];
  for (int k = 0; k < 6; ++k) {
    cm v = clover_leaf_mn(gf, g, x, pl[k][0], m, pl[k][1], n);
    if (m != n) {
      cm w = clover_leaf_mn(gf, g, x, pl[k][0], n, pl[k][1], m);
      m_add_to(&v, &w);
      v = m_rscale(0.5, &v);
    }
    cm va = m_adj(&v);
    cm d = v;
    m_sub_to(&d, &va);
    arr[k] = m_rscale(0.5, &d);
  }
  const double fac = -1.0 / (4.0 * PI * PI);
  double sum = 0.0;
  cm t = m_mul(&arr[1], &arr[4]);
  sum -= m_trace(&t).re;
  t = m_mul(&arr[2], &arr[3]);
  sum += m_trace(&t).re;
  t = m_mul(&arr[5], &arr[0]);
  sum += m_trace(&t).re;
  return fac * sum;
}

/* qcd.cpp:425-489 (hep-lat/9701012 Eq. 2-7): the five terms of the improved
 * topological charge density, topf[5 * site + k] */
void or_clf_topology_field_5_terms(double* topf, const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  const double c5 = 1.0 / 20.0;
  const double c1 = (19.0 - 55.0 * c5) / 9.0;
  const double c2 = (1.0 - 64.0 * c5) / 9.0;
  const double c3 = (-64.0 + 640.0 * c5) / 45.0;
  const double c4 = 1.0 / 5.0 - 2.0 * c5;
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    double* v = topf + 5 * i;
    v[0] = c1 * clf_topology_density_mn(gf, &g, x, 1, 1);
    v[1] = c2 / 16.0 * clf_topology_density_mn(gf, &g, x, 2, 2);
    v[2] = c3 / 4.0 * clf_topology_density_mn(gf, &g, x, 1, 2);
    v[3] = c4 / 9.0 * clf_topology_density_mn(gf, &g, x, 1, 3);
    v[4] = c5 / 81.0 * clf_topology_density_mn(gf, &g, x, 3, 3);
  }
}

/* topology.pyx:98-108 -> qcd.cpp:491-509: the improved charge (sum of the
 * five terms over all sites) */
double or_gf_topology(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double* t = (double*)malloc(5 * g.vol * sizeof(double));
  or_clf_topology_field_5_terms(t, gf, dims);
  double s = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    double si = 0.0;
    for (int k = 0; k < 5; ++k) si += t[5 * i + k];
    s += si;
  }
  free(t);
  return s;
}

double or_gf_topology_clf(const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double* tf = (double*)malloc(g.vol * sizeof(double));
  or_clf_topology_field(tf, gf, dims);
  double s = 0.0;
  for (long i = 0; i < g.vol; ++i) s += tf[i];
  free(tf);
  return s;
}

/* ------------------------------------------------------------------ */
/* integrators                                                          */

/* hmc.pyx:157-167 */
static void gm_evolve_fg(double* gm, const double* gf_init, const int dims[4], double beta, double c1,
                         double fg_dt, double dt, double* scratch_gf, double* scratch_f)
{
  const geo_t g = mk_geo(dims);
  const long n = g.vol * 72;
  memcpy(scratch_gf, gf_init, n * sizeof(double));
  or_set_gm_force(scratch_f, scratch_gf, dims, beta, c1);
  or_gf_evolve(scratch_gf, scratch_f, dims, fg_dt);
  or_set_gm_force(scratch_f, scratch_gf, dims, beta, c1);
  field_scale(scratch_f, n, dt);
  for (long i = 0; i < n; ++i) gm[i] += scratch_f[i];
}

/* hmc.pyx:169-188 */
double or_run_hmc_evolve_fg(double* gm, double* gf, const int dims[4], double beta, double c1, int n_step,
                            double md_time)
{
  const geo_t g = mk_geo(dims);
  const long n = g.vol * 72;
  double* sgf = (double*)malloc(n * sizeof(double));
  double* sf = (double*)malloc(n * sizeof(double));
  const double energy = or_gm_hamilton_node(gm, dims) + or_gf_hamilton_node(gf, dims, beta, c1);
  const double dt = md_time / n_step;
  const double lam = 0.5 * (1.0 - 1.0 / sqrt(3.0));
  const double theta = (2.0 - sqrt(3.0)) / 48.0;
  const double ttheta = theta * dt * dt * dt;
  or_gf_evolve(gf, gm, dims, lam * dt);
  for (int i = 0; i < n_step; ++i) {
    gm_evolve_fg(gm, gf, dims, beta, c1, 4.0 * ttheta / dt, 0.5 * dt, sgf, sf);
    or_gf_evolve(gf, gm, dims, (1.0 - 2.0 * lam) * dt);
    gm_evolve_fg(gm, gf, dims, beta, c1, 4.0 * ttheta / dt, 0.5 * dt, sgf, sf);
    if (i < n_step - 1) {
      or_gf_evolve(gf, gm, dims, 2.0 * lam * dt);
    } else {
      or_gf_evolve(gf, gm, dims, lam * dt);
    }
  }
  or_unitarize_field(gf, dims);
  const double delta_h = or_gm_hamilton_node(gm, dims) + or_gf_hamilton_node(gf, dims, beta, c1) - energy;
  free(sgf);
  free(sf);
  return delta_h;
}

/* examples-py/hmc-pure-gauge-fgf.py:57-69 composed with gf_evolve / set_gm_force */
double or_run_hmc_evolve_leapfrog(double* gm, double* gf, const int dims[4], double beta, double c1,
                                  int n_step, double md_time)
{
  const geo_t g = mk_geo(dims);
  const long n = g.vol * 72;
  double* sf = (double*)malloc(n * sizeof(double));
  const double energy = or_gm_hamilton_node(gm, dims) + or_gf_hamilton_node(gf, dims, beta, c1);
  const double dt = md_time / n_step;
  for (int i = 0; i < n_step; ++i) {
    or_gf_evolve(gf, gm, dims, 0.5 * dt);
    or_set_gm_force(sf, gf, dims, beta, c1);
    field_scale(sf, n, dt);
    for (long k = 0; k < n; ++k) gm[k] += sf[k];
    or_gf_evolve(gf, gm, dims, 0.5 * dt);
  }
  or_unitarize_field(gf, dims);
  const double delta_h = or_gm_hamilton_node(gm, dims) + or_gf_hamilton_node(gf, dims, beta, c1) - energy;
  free(sf);
  return delta_h;
}

/* ------------------------------------------------------------------ */
/* field-accelerated HMC                                                */

/* rng-state.h:71-76 newtype + rng-state.cpp:38-45 set_type */
static void rng_newtype(or_rng* out, const or_rng* rs, uint64_t type)
{
  *out = *rs;
  out->type = type;
  out->cacheAvail = 0;
  out->gaussianAvail = 0;
}

/* core.h:1585-1603 */
void or_field_set_u_rand(double* f, const int dims[4], int n_per_site, const or_rng* rs, double upper, double lower)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    or_rng rsi;
    rng_newtype(&rsi, rs, (uint64_t)i);
    for (int m = 0; m < n_per_site; ++m) f[i * n_per_site + m] = or_u_rand_gen(&rsi, upper, lower);
  }
}

/* core.h:1617-1636 */
void or_field_set_g_rand(double* f, const int dims[4], int n_per_site, const or_rng* rs, double center, double sigma)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    or_rng rsi;
    rng_newtype(&rsi, rs, (uint64_t)i);
    for (int m = 0; m < n_per_site; ++m) f[i * n_per_site + m] = or_g_rand_gen(&rsi, center, sigma);
  }
}

/* hmc.cpp:121-149 */
void or_set_rand_gauge_momentum_fa(double* gm, const double* mf, const int dims[4], const or_rng* rs)
{
  or_set_rand_gauge_momentum(gm, dims, rs, 1.0);
  const geo_t g = mk_geo(dims);
  for (long i = 0; i < g.vol; ++i)
    for (int m = 0; m < 4; ++m) {
      double* p = gm + (i * 4 + m) * 18;
      const double v = mf[i * 4 + m];
      if (v != INFINITY) {
        const double s = sqrt(v);
        for (int k = 0; k < 18; ++k) p[k] *= s;
      } else {
        for (int k = 0; k < 18; ++k) p[k] = 0.0;
      }
    }
}

/* hmc.cpp:175-201 */
double or_gm_hamilton_node_fa(const double* gm, const double* mf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  double sum = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    double s = 0.0;
    for (int mu = 0; mu < 4; ++mu) {
      cm p;
      memcpy(&p, gm + (i * 4 + mu) * 18, sizeof(cm));
      s += neg_half_tr_square(&p) / mf[i * 4 + mu];
    }
    sum += s;
  }
  return sum;
}

/* hmc.cpp:311-396 with matrix_evolve / matrix_evolve_dual (matrix-hmc.h:178-200) */
void or_gf_evolve_fa(double* gf, const double* gm, const double* mf, const int dims[4], double step_size, int dual)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    for (int mu = 0; mu < 4; ++mu) {
      cm u, p;
      memcpy(&u, gf + (i * 4 + mu) * 18, sizeof(cm));
      memcpy(&p, gm + (i * 4 + mu) * 18, sizeof(cm));
      const double dt_m = mf ? step_size / mf[i * 4 + mu] : step_size;
      cm r;
      if (!dual) {
        r = matrix_evolve(&u, &p, dt_m);
      } else {
        cm t = m_rscale(-dt_m, &p);
        cm e = make_matrix_exp(&t, 20);
        r = m_mul(&u, &e);
        unitarize_cm(&r);
      }
      put_link(gf, i, mu, &r);
    }
  }
}

/* hmc.cpp:492-513: -U^+ F U, evaluated as ((-U^+) F) U */
void or_set_gm_force_dual(double* fd, const double* gf, const double* f, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  for (long i = 0; i < g.vol; ++i)
    for (int mu = 0; mu < 4; ++mu) {
      cm u, x;
      memcpy(&u, gf + (i * 4 + mu) * 18, sizeof(cm));
      memcpy(&x, f + (i * 4 + mu) * 18, sizeof(cm));
      cm a = m_adj(&u);
      a = m_rscale(-1.0, &a);
      cm t = m_mul(&a, &x);
      t = m_mul(&t, &u);
      put_link(fd, i, mu, &t);
    }
}

/* hmc.cpp:515-589 */
double or_project_gauge_transform(double* gm, double* gmd, const double* mf, const double* mfd, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  cm* ag = (cm*)malloc(sizeof(cm) * (size_t)g.vol);
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    cm sum = m_zero();
    for (int m = 0; m < 4; ++m) {
      int xm[4] = {x[0], x[1], x[2], x[3]};
      xm[m] -= 1;
      const long im = index_from_coor(&g, xm);
      const double m1 = mf[i * 4 + m];
      const double m2 = mfd[im * 4 + m];
      cm c1, c2;
      memcpy(&c1, gm + (i * 4 + m) * 18, sizeof(cm));
      memcpy(&c2, gmd + (im * 4 + m) * 18, sizeof(cm));
      if (m1 != INFINITY) {
        cm t = m_rscale(1.0 / sqrt(m1), &c1);
        m_add_to(&sum, &t);
      }
      if (m2 != INFINITY) {
        cm t = m_rscale(1.0 / sqrt(m2), &c2);
        m_add_to(&sum, &t);
      }
    }
    ag[i] = m_rscale(1.0 / 8.0, &sum);
  }
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int m = 0; m < 4; ++m) {
      int xp[4] = {x[0], x[1], x[2], x[3]};
      xp[m] += 1;
      const long ip = index_from_coor(&g, xp);
      if (mf[i * 4 + m] != INFINITY) {
        cm v;
        memcpy(&v, gm + (i * 4 + m) * 18, sizeof(cm));
        cm t = m_rscale(sqrt(mf[i * 4 + m]), &ag[i]);
        m_sub_to(&v, &t);
        put_link(gm, i, m, &v);
      }
      if (mfd[i * 4 + m] != INFINITY) {
        cm v;
        memcpy(&v, gmd + (i * 4 + m) * 18, sizeof(cm));
        cm t = m_rscale(sqrt(mfd[i * 4 + m]), &ag[ip]);
        m_sub_to(&v, &t);
        put_link(gmd, i, m, &v);
      }
    }
  }
  double qn = 0.0;
  for (long i = 0; i < g.vol; ++i) {
    const double* p = (const double*)ag[i].p;
    double s = 0.0;
    for (int k = 0; k < 9; ++k) s += p[2 * k] * p[2 * k] + p[2 * k + 1] * p[2 * k + 1];
    qn += s;
  }
  free(ag);
  return qn / (double)g.vol;
}

/* hmc.cpp:591-626 */
void or_set_gauge_transform_momentum(double* gm, double* gmd, const double* gtm, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int m = 0; m < 4; ++m) {
      int xp[4] = {x[0], x[1], x[2], x[3]};
      xp[m] += 1;
      const long ip = index_from_coor(&g, xp);
      memcpy(gm + (i * 4 + m) * 18, gtm + i * 18, sizeof(cm));
      memcpy(gmd + (i * 4 + m) * 18, gtm + ip * 18, sizeof(cm));
    }
  }
}

/* hmc.cpp:628-645 with qnorm(m1, m2) (matrix.h:209-217, complex.h:153-156) */
void or_dot_gauge_momentum(double* f, const double* gm1, const double* gm2, const int dims[4])
{
  const geo_t g = mk_geo(dims);
  for (long i = 0; i < g.vol * 4; ++i) {
    double s = 0.0;
    for (int k = 0; k < 9; ++k) s += gm1[i * 18 + 2 * k] * gm2[i * 18 + 2 * k] + gm1[i * 18 + 2 * k + 1] * gm2[i * 18 + 2 * k + 1];
    f[i] = s;
  }
}

/* ------------------------------------------------------------------ */
/* topology-measurement flows                                           */

static const int PLANE_A[6] = {0, 0, 0, 1, 1, 2};
static const int PLANE_B[6] = {1, 2, 3, 2, 3, 3};

/* qcd.cpp:84-91 gf_plaq_no_comm: Re tr(U_a(x) U_b(x+a) (U_b(x) U_a(x+b))^+) / 3 */
static double plaq_at(const double* gf, const geo_t* g, const int x[4], int a, int b)
{
  int xa[4] = {x[0], x[1], x[2], x[3]}, xb[4] = {x[0], x[1], x[2], x[3]};
  xa[a] += 1;
  xb[b] += 1;
  cm ua = get_link(gf, g, x, a), ub = get_link(gf, g, x, b);
  cm ub_a = get_link(gf, g, xa, b), ua_b = get_link(gf, g, xb, a);
  cm l = m_mul(&ua, &ub_a);
  cm r = m_mul(&ub, &ua_b);
  cm ra = m_adj(&r);
  cm p = m_mul(&l, &ra);
  return m_trace(&p).re / 3.0;
}

/* qcd.cpp:298-325 */
void or_gf_plaq_field(double* f_plaq, const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int p = 0; p < 6; ++p) f_plaq[i * 6 + p] = plaq_at(gf, &g, x, PLANE_A[p], PLANE_B[p]);
  }
}

/* qcd-utils.cpp:359-400 (make_wilson_loop_path: l along +i, t along +3, l along -i, t along -3) */
double or_gf_avg_wilson_loop_normalized_tr(const double* gf, const int dims[4], int l, int t)
{
  const geo_t g = mk_geo(dims);
  int path[256];
  double tot = 0.0;
  for (int i = 0; i < 3; ++i) {
    int n = 0;
    for (int k = 0; k < l && n < 256; ++k) path[n++] = i;
    for (int k = 0; k < t && n < 256; ++k) path[n++] = 3;
    for (int k = 0; k < l && n < 256; ++k) path[n++] = -i - 1;
    for (int k = 0; k < t && n < 256; ++k) path[n++] = -4;
    cd sum = {0.0, 0.0};
    for (long s = 0; s < g.vol; ++s) {
      int x[4];
      coor_from_index(&g, s, x);
      cm w = wilson_line(gf, &g, x, path, n);
      sum = c_add(sum, m_trace(&w));
    }
    tot += sum.re / (double)g.vol;
  }
  return tot / 3.0 / 3.0;
}

/* wilson-flow.cpp:53-95 */
void or_gf_energy_density_dir_field(double* fd, const double* gf, const int dims[4])
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int p = 0; p < 6; ++p) {
      cm c = clover_leaf(gf, &g, x, PLANE_A[p], PLANE_B[p]);
      cm gmn = make_tr_less_anti_herm(&c);
      fd[i * 6 + p] = -m_trace2(&gmn, &gmn).re;
    }
  }
}

/* qcd.cpp:33-62 with the clover leaves of qcd.cpp:10-31 */
void or_clf_plaq_action_density_field(double* paf, const double* gf, const int dims[4], int spatial)
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    double sum = 0.0;
    for (int p = 0; p < 6; ++p) {
      if (spatial && (p == 2 || p == 4 || p == 5)) continue;
      cm c = clover_leaf(gf, &g, x, PLANE_A[p], PLANE_B[p]);
      sum += 1.0 - 1.0 / 3.0 * m_trace(&c).re;
    }
    paf[i] = sum;
  }
}

static int plane_index(int mu, int nu)
{
  const int a = mu < nu ? mu : nu, b = mu < nu ? nu : mu;
  for (int p = 0; p < 6; ++p)
    if (PLANE_A[p] == a && PLANE_B[p] == b) return p;
  return -1;
}

/* wilson-flow.cpp:164-207 */
void or_set_plaq_flow_z(double* z, const double* gf, const double* plaq_factor, const int dims[4])
{
  const geo_t g = mk_geo(dims);
#pragma omp parallel for
  for (long i = 0; i < g.vol; ++i) {
    int x[4];
    coor_from_index(&g, i, x);
    for (int mu = 0; mu < 4; ++mu) {
      cm acc = m_zero();
      for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int xn[4] = {x[0], x[1], x[2], x[3]};
        xn[nu] -= 1;
        const long in = index_from_coor(&g, xn);
        const int m = plane_index(mu, nu);
        const int p1[3] = {nu, mu, -nu - 1};
        const int p2[3] = {-nu - 1, mu, nu};
        cm w1 = wilson_line(gf, &g, x, p1, 3);
        cm w2 = wilson_line(gf, &g, x, p2, 3);
        cm t1 = m_rscale(plaq_factor[i * 6 + m], &w1);
        m_add_to(&acc, &t1);
        cm t2 = m_rscale(plaq_factor[in * 6 + m], &w2);
        m_add_to(&acc, &t2);
      }
      cm ad = m_adj(&acc);
      cm u = get_link(gf, &g, x, mu);
      cm f = m_mul(&u, &ad);
      f = m_rscale(-1.0, &f);
      cm r = make_tr_less_anti_herm(&f);
      put_link(z, i, mu, &r);
    }
  }
}

/* instanton_map.py:162-190 */
double or_gf_flow_topo_plaq(double* gf, const int dims[4], double step_size, int kind)
{
  const geo_t g = mk_geo(dims);
  double* fp = (double*)malloc(sizeof(double) * 6 * (size_t)g.vol);
  double* pf = (double*)malloc(sizeof(double) * 6 * (size_t)g.vol);
  double* z = (double*)malloc(sizeof(double) * 72 * (size_t)g.vol);
  or_gf_plaq_field(fp, gf, dims);
  double pmin = fp[0], pmax = fp[0];
  for (long i = 0; i < 6 * g.vol; ++i) {
    if (fp[i] < pmin) pmin = fp[i];
    if (fp[i] > pmax) pmax = fp[i];
  }
  double norm = 1.0;
  for (long i = 0; i < 6 * g.vol; ++i) {
    const double p = fp[i];
    double v;
    if (kind == 1) v = 0.005 / (1 - p + 0.005) + 0.5;
    else if (kind == 2) v = 1 - p;
    else if (kind == 3) v = 0.002 / (1 - p + 0.002) + (50 * (1 - p));
    else { v = 50 * (1 - p); if (v < 1) v = 1; }
    pf[i] = v;
  }
  if (kind == 1) norm = 0.005 / (1 - pmax + 0.005) + 0.5;
  else if (kind == 2) norm = 1 - pmin;
  else if (kind == 3) {
    const double a = 0.002 / (1 - pmax + 0.002) + (50 * (1 - pmax));
    const double b = 0.002 / (1 - pmin + 0.002) + (50 * (1 - pmin));
    norm = a > b ? a : b;
  } else {
    norm = 50 * (1 - pmin);
    if (norm < 1) norm = 1;
  }
  or_set_plaq_flow_z(z, gf, pf, dims);
  or_gf_evolve(gf, z, dims, step_size / norm);
  free(fp);
  free(pf);
  free(z);
  return step_size / norm;
}

void or_make_matrix_exp(double out[18], const double a[18], int max_order)
{
  cm x;
  memcpy(&x, a, sizeof(cm));
  cm r = make_matrix_exp(&x, max_order);
  memcpy(out, &r, sizeof(cm));
}

void or_unitarize(double m[18])
{
  cm x;
  memcpy(&x, m, sizeof(cm));
  unitarize_cm(&x);
  memcpy(m, &x, sizeof(cm));
}

void or_make_tr_less_anti_herm(double out[18], const double m[18])
{
  cm x;
  memcpy(&x, m, sizeof(cm));
  cm r = make_tr_less_anti_herm(&x);
  memcpy(out, &r, sizeof(cm));
}
