// fa.cu -- field-accelerated HMC on the GPU: per-link masses, the dual
// momentum, and the projection of gauge-transformation motion (the
// reference's hmc.cpp:121-201, 330-396, 492-645 and the per-site random
// real fields of core.h:1585-1636).
//
// A field-accelerated trajectory carries two momenta per link: gm, which
// moves U_mu(x) from the left (U <- exp(dt gm / m) U), and gm_dual, which
// moves it from the right (U <- U exp(-dt gm_dual / m_dual)), each with its
// own per-link mass field (Field<RealD> of multiplicity 4; an infinite mass
// freezes that link's momentum at zero).  The gauge-transformation part of
// the motion at x is the average ag(x) of the mass-weighted momenta that
// start or end at x; project_gauge_transform subtracts it from both momenta.
//
// Layout and access as in gauge_common.cuh.  One thread per link for the
// link-local kernels (grid.y = mu), one thread per site for the projection's
// site pass and for the reductions, which accumulate in FP64 and reduce in a
// fixed order (per block, then one block over the block sums).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/qlat_b200.h"
#include "gauge_common.cuh"
#include "kernels.h"
#include "rng.cuh"

namespace qgb
{
void set_last_error(const std::string& msg);
void* field_data(const qgb_field* f);
int library_stream(cudaStream_t* st);
int scratch_buffer(size_t bytes, int tag, void** out);
void add_launches(int64_t n);
}  // namespace qgb

namespace
{
using namespace qgb;

constexpr int FA_BS = 256;

__device__ __forceinline__ bool is_pos_inf(double m) { return m == (double)INFINITY; }

__device__ __forceinline__ double ld_mass(const double* mf, long V, int mu, long s)
{
  return __ldg(mf + lay_index<1>(V, mu, 0, s));
}

// fixed-order block sum of one value per thread into partials[blockIdx.x]
__device__ __forceinline__ void block_sum_store(double v, double* partials)
{
  __shared__ double sm[FA_BS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < FA_BS / 32; ++i) t += sm[i];
    partials[blockIdx.x] = t;
  }
}

// set_rand_gauge_momentum(gm, mf, rs) after the unit-sigma draw (hmc.cpp:121-149):
// gm_mu(x) *= sqrt(mf_mu(x)); zero where the mass is infinite.
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_mass_scale(long V, Cx<R>* P, const double* mf)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  const WField<R> Pf{P, V};
  const double m = ld_mass(mf, V, mu, s);
  if (is_pos_inf(m)) Pf.st(s, mu, m3_zero<R>());
  else Pf.st(s, mu, scale((R)sqrt(m), Pf.ld(s, mu)));
}

// gm_hamilton_node(gm, mf) (hmc.cpp:175-201): per site sum_mu (-1/2 tr gm^2) / mf.
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_hamilton_fa(long V, const Cx<R>* P, const double* mf, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (s < V) {
    const CField<R> Pf{P, V};
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) v += neg_half_tr_square(Pf.ld(s, mu)) / ld_mass(mf, V, mu, s);
  }
  block_sum_store(v, partials);
}

// gf_evolve(gf, gm, [mf,] dt) / gf_evolve_dual(gf, gm_dual, [mf_dual,] dt)
// (hmc.cpp:311-396, matrix_evolve / matrix_evolve_dual of matrix-hmc.h:178-200):
//   U <- unitarize(exp(dt_m P) U)      or     U <- unitarize(U exp(-dt_m P)),
// dt_m = dt / mass (dt without a mass field).
template <typename R, bool DUAL>
__global__ void __launch_bounds__(FA_BS) k_evolve_fa(long V, Cx<R>* U, const Cx<R>* P, const double* mf, double dt)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  const WField<R> Uf{U, V};
  const CField<R> Pf{P, V};
  const double dt_m = mf ? dt / ld_mass(mf, V, mu, s) : dt;
  const M3<R> e = exp_ch(scale((R)(DUAL ? -dt_m : dt_m), Pf.ld(s, mu)));
  M3<R> un = DUAL ? mul(Uf.ld(s, mu), e) : mul(e, Uf.ld(s, mu));
  unitarize(un);
  Uf.st(s, mu, un);
}

// set_gm_force_dual (hmc.cpp:492-513): F_dual = -U^+ F U.
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_force_dual(long V, Cx<R>* Fd, const Cx<R>* U, const Cx<R>* F)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  const CField<R> Uf{U, V}, Ff{F, V};
  const M3<R> u = Uf.ld(s, mu);
  const M3<R> r = mul(adj_mul(u, Ff.ld(s, mu)), u);
  Cx<R>* q = Fd + lay_index<9>(V, mu, 0, s);
#pragma unroll
  for (int k = 0; k < 9; ++k) q[32 * k] = cx<R>(-r.e[k].re, -r.e[k].im);
}

// project_gauge_transform, site pass (hmc.cpp:536-567):
//   ag(x) = 1/8 sum_m [ gm_m(x) / sqrt(mf_m(x)) + gm_dual_m(x - m) / sqrt(mf_dual_m(x - m)) ],
// terms with an infinite mass left out; also the per-block sums of qnorm(ag).
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_gt_average(Geo g, const Cx<R>* P, const Cx<R>* Pd, const double* mf,
                                                      const double* mfd, Cx<R>* Ag, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double qn = 0.0;
  if (s < g.V) {
    const CField<R> Pf{P, g.V}, Pdf{Pd, g.V};
    const Coord x = coord_of(g, s);
    M3<R> sum = m3_zero<R>();
    for (int m = 0; m < 4; ++m) {
      const long sm = site_rt(g, x, m, -1, m, 0);
      const double m1 = ld_mass(mf, g.V, m, s);
      const double m2 = ld_mass(mfd, g.V, m, sm);
      if (!is_pos_inf(m1)) add_to(sum, scale((R)(1.0 / sqrt(m1)), Pf.ld(s, m)));
      if (!is_pos_inf(m2)) add_to(sum, scale((R)(1.0 / sqrt(m2)), Pdf.ld(sm, m)));
    }
    const M3<R> ag = scale((R)(1.0 / 8.0), sum);
    const WField<R> Af{Ag, g.V};
    Af.st(s, 0, ag);
#pragma unroll
    for (int k = 0; k < 9; ++k) qn += (double)ag.e[k].re * ag.e[k].re + (double)ag.e[k].im * ag.e[k].im;
  }
  block_sum_store(qn, partials);
}

// project_gauge_transform, link pass (hmc.cpp:569-588):
//   gm_m(x) -= sqrt(mf_m(x)) ag(x);  gm_dual_m(x) -= sqrt(mf_dual_m(x)) ag(x + m),
// links with an infinite mass untouched.
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_gt_subtract(Geo g, Cx<R>* P, Cx<R>* Pd, const double* mf, const double* mfd,
                                                       const Cx<R>* Ag)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int m = blockIdx.y;
  const CField<R> Af{Ag, g.V};
  const double m1 = ld_mass(mf, g.V, m, s);
  const double m2 = ld_mass(mfd, g.V, m, s);
  if (!is_pos_inf(m1)) {
    const WField<R> Pf{P, g.V};
    M3<R> v = Pf.ld(s, m);
    axpy(v, (R)(-sqrt(m1)), Af.ld(s, 0));
    Pf.st(s, m, v);
  }
  if (!is_pos_inf(m2)) {
    const Coord x = coord_of(g, s);
    const WField<R> Pdf{Pd, g.V};
    M3<R> v = Pdf.ld(s, m);
    axpy(v, (R)(-sqrt(m2)), Af.ld(site_rt(g, x, m, 1, m, 0), 0));
    Pdf.st(s, m, v);
  }
}

// set_gauge_transform_momentum (hmc.cpp:591-626): gm_m(x) = gtm(x), gm_dual_m(x) = gtm(x + m).
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_gt_momentum(Geo g, Cx<R>* P, Cx<R>* Pd, const Cx<R>* G)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int m = blockIdx.y;
  const CField<R> Gf{G, g.V};
  const WField<R> Pf{P, g.V}, Pdf{Pd, g.V};
  Pf.st(s, m, Gf.ld(s, 0));
  Pdf.st(s, m, Gf.ld(site_rt(g, coord_of(g, s), m, 1, m, 0), 0));
}

// dot_gauge_momentum (hmc.cpp:628-645): f_m(x) = sum_k Re(a_k) Re(b_k) + Im(a_k) Im(b_k).
template <typename R>
__global__ void __launch_bounds__(FA_BS) k_dot(long V, double* f, const Cx<R>* A, const Cx<R>* B)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int m = blockIdx.y;
  const CField<R> Af{A, V}, Bf{B, V};
  const M3<R> a = Af.ld(s, m), b = Bf.ld(s, m);
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) t += (double)a.e[k].re * b.e[k].re + (double)a.e[k].im * b.e[k].im;
  f[lay_index<1>(V, m, 0, s)] = t;
}

struct RngArg {
  uint32_t v[24];
};

// set_u_rand / set_g_rand of a field (core.h:1585-1636): per site the state
// rs.newtype(gindex), then one draw per real of the site in memory order
// (component, then matrix entry, real before imaginary part).
template <typename R, bool COLOR, bool GAUSS>
__global__ void __launch_bounds__(128) k_rand_field(long V, int mult, RngArg ra, double a, double b, void* out,
                                                    int* ambiguous)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  Rng rs;
  rng_import(rs, ra.v);
  rs.type = (uint64_t)s;  // set_type (rng-state.cpp:38-45)
  rs.cacheAvail = 0;
  rs.gaussianAvail = 0;
  int amb = 0;
  const int n = mult * (COLOR ? 18 : 1);
  for (int i = 0; i < n; ++i) {
    const double v = GAUSS ? rng_g_rand_gen<true>(rs, a, b, &amb) : rng_u_rand_gen(rs, a, b);
    if (COLOR) {
      const int m = i / 18, k = (i % 18) >> 1;
      R* p = reinterpret_cast<R*>((Cx<R>*)out + lay_index<9>(V, m, k, s));
      p[i & 1] = (R)v;
    } else {
      ((R*)out)[lay_index<1>(V, i, 0, s)] = (R)v;
    }
  }
  if (amb) atomicAdd(ambiguous, 1);
}

// f[x, m] = value for all real entries of the sites x < V (set_unit / fill of Field<RealD>)
template <typename R>
__global__ void k_fill_real(long V, int mult, R* f, double value, const uint8_t* mask)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int m = blockIdx.y;
  if (mask && !mask[s * mult + m]) return;
  f[lay_index<1>(V, m, 0, s)] = (R)value;
}

// dst[x, m] = src[x, m] where mask[x * mult + m] (f[sel] = g[sel] with a boolean selection)
template <typename R, int K>
__global__ void k_masked_copy(long V, int mult, R* dst, const R* src, const uint8_t* mask)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int m = blockIdx.y;
  if (!mask[s * mult + m]) return;
  // K reals per entry group: 18 for a color matrix (9 complex), 1 for a real
  constexpr int C = K == 18 ? 9 : 1;
  for (int k = 0; k < C; ++k) {
    const long o = lay_index<C>(V, m, k, s);
    if (K == 18) {
      reinterpret_cast<Cx<R>*>(dst)[o] = reinterpret_cast<const Cx<R>*>(src)[o];
    } else {
      dst[o] = src[o];
    }
  }
}

__global__ void k_sum_partials(const double* partials, int n, double* out)
{
  __shared__ double sm[32];
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sm[i];
    *out = r;
  }
}

// ---- host side ---------------------------------------------------------------

int ffail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

#define FA_CUDA(expr)                                                                                        \
  do {                                                                                                       \
    cudaError_t e_ = (expr);                                                                                 \
    if (e_ != cudaSuccess) return ffail(QGB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define FA_RC(expr)              \
  do {                           \
    int r_ = (expr);             \
    if (r_ != QGB_OK) return r_; \
  } while (0)

struct Meta {
  int32_t ts[4] = {0, 0, 0, 0};
  int32_t mult = 0, kind = -1, prec = 0;
  long V = 0;
  void* d = nullptr;
};

int meta_of(const qgb_field* f, Meta& m, const char* what)
{
  if (!f) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": null field");
  FA_RC(qgb_field_info(f, m.ts, &m.mult, &m.kind, &m.prec));
  m.V = (long)m.ts[0] * m.ts[1] * m.ts[2] * m.ts[3];
  m.d = qgb::field_data(f);
  return QGB_OK;
}

bool same_sites(const Meta& a, const Meta& b)
{
  for (int i = 0; i < 4; ++i)
    if (a.ts[i] != b.ts[i]) return false;
  return true;
}

// color-matrix fields of multiplicity 4 on one lattice in one precision
int check_links(const char* what, std::initializer_list<const Meta*> fs)
{
  const Meta* f0 = *fs.begin();
  for (const Meta* f : fs)
    if (f->kind != QGB_KIND_COLOR_MATRIX || f->mult != 4 || f->prec != f0->prec || !same_sites(*f, *f0))
      return ffail(QGB_ERR_MISMATCH, std::string(what) +
                                         ": gauge fields and momenta must be color-matrix fields of multiplicity 4 "
                                         "on the same lattice in the same precision");
  return QGB_OK;
}

// FP64 real field of multiplicity 4 on the lattice of `ref`
int check_mass(const char* what, const Meta& mf, const Meta& ref)
{
  if (mf.kind != QGB_KIND_REAL || mf.mult != 4 || mf.prec != QGB_F64 || !same_sites(mf, ref))
    return ffail(QGB_ERR_MISMATCH,
                 std::string(what) + ": a mass field must be an FP64 real field of multiplicity 4 on the same lattice");
  return QGB_OK;
}

Geo geo_of(const Meta& m)
{
  Geo g;
  for (int i = 0; i < 4; ++i) g.d[i] = m.ts[i];
  g.V = m.V;
  return g;
}

dim3 link_grid(long V, int mult) { return dim3((unsigned)((V + FA_BS - 1) / FA_BS), (unsigned)mult); }
unsigned site_grid(long V) { return (unsigned)((V + FA_BS - 1) / FA_BS); }

// Scratch tags of this file (distinct from the rest of the library's).
enum { TAG_PARTIALS = 0x7A000, TAG_RESULT, TAG_AG64, TAG_AG32, TAG_MASK, TAG_AMB };

// sum of the per-block partials, copied to the host (synchronises the stream)
int sum_to_host(cudaStream_t st, const double* partials, int n, double* out)
{
  void* r = nullptr;
  FA_RC(qgb::scratch_buffer(sizeof(double), TAG_RESULT, &r));
  k_sum_partials<<<1, 1024, 0, st>>>(partials, n, (double*)r);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  double h = 0.0;
  FA_CUDA(cudaMemcpyAsync(&h, r, sizeof(double), cudaMemcpyDeviceToHost, st));
  FA_CUDA(cudaStreamSynchronize(st));
  *out = h;
  return QGB_OK;
}

int partials_buffer(long V, double** out)
{
  void* p = nullptr;
  FA_RC(qgb::scratch_buffer((size_t)site_grid(V) * sizeof(double), TAG_PARTIALS, &p));
  *out = (double*)p;
  return QGB_OK;
}

// a host boolean selection (one byte per (site, component), site-major) on the device
int upload_mask(cudaStream_t st, const uint8_t* mask, int64_t n, const Meta& f, uint8_t** out)
{
  if (!mask || n != (int64_t)f.V * f.mult)
    return ffail(QGB_ERR_INVALID_ARG, "selection: need one byte per (site, component) of the field");
  void* p = nullptr;
  FA_RC(qgb::scratch_buffer((size_t)n, TAG_MASK, &p));
  FA_CUDA(cudaMemcpyAsync(p, mask, (size_t)n, cudaMemcpyHostToDevice, st));
  *out = (uint8_t*)p;
  return QGB_OK;
}

template <typename R>
int evolve_dispatch(cudaStream_t st, const Meta& gf, const Meta& gm, const double* mf, double dt, bool dual)
{
  const dim3 grid = link_grid(gf.V, 4);
  if (dual) k_evolve_fa<R, true><<<grid, FA_BS, 0, st>>>(gf.V, (Cx<R>*)gf.d, (const Cx<R>*)gm.d, mf, dt);
  else k_evolve_fa<R, false><<<grid, FA_BS, 0, st>>>(gf.V, (Cx<R>*)gf.d, (const Cx<R>*)gm.d, mf, dt);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

int evolve(qgb_field* gf_, const qgb_field* gm_, const qgb_field* mf_, double dt, bool dual, const char* what)
{
  Meta gf, gm, mf;
  FA_RC(meta_of(gf_, gf, what));
  FA_RC(meta_of(gm_, gm, what));
  FA_RC(check_links(what, {&gf, &gm}));
  if (mf_) {
    FA_RC(meta_of(mf_, mf, what));
    FA_RC(check_mass(what, mf, gf));
  }
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  const double* m = mf_ ? (const double*)mf.d : nullptr;
  if (gf.prec == QGB_F64) FA_RC(evolve_dispatch<double>(st, gf, gm, m, dt, dual));
  else FA_RC(evolve_dispatch<float>(st, gf, gm, m, dt, dual));
  return QGB_OK;
}

template <typename R>
int rand_field_dispatch(cudaStream_t st, const Meta& f, const RngArg& ra, double a, double b, bool gauss, int* amb)
{
  const unsigned grid = (unsigned)((f.V + 127) / 128);
  const bool color = f.kind == QGB_KIND_COLOR_MATRIX;
  if (color && gauss) k_rand_field<R, true, true><<<grid, 128, 0, st>>>(f.V, f.mult, ra, a, b, f.d, amb);
  else if (color) k_rand_field<R, true, false><<<grid, 128, 0, st>>>(f.V, f.mult, ra, a, b, f.d, amb);
  else if (gauss) k_rand_field<R, false, true><<<grid, 128, 0, st>>>(f.V, f.mult, ra, a, b, f.d, amb);
  else k_rand_field<R, false, false><<<grid, 128, 0, st>>>(f.V, f.mult, ra, a, b, f.d, amb);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

// The SHA-256 and logarithm tables live in __constant__ memory, one copy per
// translation unit: fill this file's copy once per device before its first
// random-field kernel.
int rng_constants_here()
{
  static std::mutex mu;
  static uint64_t done = 0;  // one bit per device
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  FA_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && ((done >> dev) & 1u)) return QGB_OK;
  FA_CUDA(cudaMemcpyToSymbol(qgb_sha_dev, &qgb_sha_host, sizeof(ShaConst)));
  FA_CUDA(cudaMemcpyToSymbol(qgb_logtab_dev, qgb_logtab_host, sizeof(qgb_logtab_host)));
  if (dev < 64) done |= (uint64_t)1 << dev;
  return QGB_OK;
}

int rand_field(qgb_field* f_, const uint32_t rs[24], double a, double b, bool gauss, const char* what)
{
  Meta f;
  FA_RC(meta_of(f_, f, what));
  if (!rs) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": null RngState");
  // newtype requires an untyped state (rng-state.cpp:40)
  if (rs[10] != 0xffffffffu || rs[11] != 0xffffffffu)
    return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": the RngState already has a type");
  RngArg ra;
  memcpy(ra.v, rs, sizeof(ra.v));
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  FA_RC(rng_constants_here());
  void* amb = nullptr;
  FA_RC(qgb::scratch_buffer(sizeof(int), TAG_AMB, &amb));
  if (f.prec == QGB_F64) FA_RC(rand_field_dispatch<double>(st, f, ra, a, b, gauss, (int*)amb));
  else FA_RC(rand_field_dispatch<float>(st, f, ra, a, b, gauss, (int*)amb));
  if (gauss) {
    // an uncertified rounding of the device logarithm is reported, never hidden
    int h = 0;
    FA_CUDA(cudaMemcpyAsync(&h, amb, sizeof(int), cudaMemcpyDeviceToHost, st));
    FA_CUDA(cudaMemsetAsync(amb, 0, sizeof(int), st));
    FA_CUDA(cudaStreamSynchronize(st));
    if (h) return ffail(QGB_ERR_MISMATCH, std::string(what) + ": a Gaussian draw hit an uncertified log rounding");
  }
  return QGB_OK;
}

}  // namespace

extern "C" {

int qgb_set_rand_gauge_momentum_fa(qgb_field* gm_, const qgb_field* mf_, const uint32_t rs[24])
{
  const char* what = "qgb_set_rand_gauge_momentum_fa";
  Meta gm, mf;
  FA_RC(meta_of(gm_, gm, what));
  FA_RC(meta_of(mf_, mf, what));
  FA_RC(check_links(what, {&gm}));
  FA_RC(check_mass(what, mf, gm));
  FA_RC(qgb_set_rand_gauge_momentum(gm_, 1.0, rs));
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  const dim3 grid = link_grid(gm.V, 4);
  if (gm.prec == QGB_F64) k_mass_scale<double><<<grid, FA_BS, 0, st>>>(gm.V, (Cx<double>*)gm.d, (const double*)mf.d);
  else k_mass_scale<float><<<grid, FA_BS, 0, st>>>(gm.V, (Cx<float>*)gm.d, (const double*)mf.d);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

int qgb_gm_hamilton_node_fa(const qgb_field* gm_, const qgb_field* mf_, double* out)
{
  const char* what = "qgb_gm_hamilton_node_fa";
  Meta gm, mf;
  FA_RC(meta_of(gm_, gm, what));
  FA_RC(meta_of(mf_, mf, what));
  FA_RC(check_links(what, {&gm}));
  FA_RC(check_mass(what, mf, gm));
  if (!out) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": null output");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  double* partials = nullptr;
  FA_RC(partials_buffer(gm.V, &partials));
  if (gm.prec == QGB_F64)
    k_hamilton_fa<double><<<site_grid(gm.V), FA_BS, 0, st>>>(gm.V, (const Cx<double>*)gm.d, (const double*)mf.d,
                                                             partials);
  else
    k_hamilton_fa<float><<<site_grid(gm.V), FA_BS, 0, st>>>(gm.V, (const Cx<float>*)gm.d, (const double*)mf.d,
                                                            partials);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return sum_to_host(st, partials, (int)site_grid(gm.V), out);
}

int qgb_gf_evolve_fa(qgb_field* gf, const qgb_field* gm, const qgb_field* mf, double step_size)
{
  if (!mf) return ffail(QGB_ERR_INVALID_ARG, "qgb_gf_evolve_fa: null mass field");
  return evolve(gf, gm, mf, step_size, false, "qgb_gf_evolve_fa");
}

int qgb_gf_evolve_dual(qgb_field* gf, const qgb_field* gm_dual, double step_size)
{
  return evolve(gf, gm_dual, nullptr, step_size, true, "qgb_gf_evolve_dual");
}

int qgb_gf_evolve_fa_dual(qgb_field* gf, const qgb_field* gm_dual, const qgb_field* mf_dual, double step_size)
{
  if (!mf_dual) return ffail(QGB_ERR_INVALID_ARG, "qgb_gf_evolve_fa_dual: null mass field");
  return evolve(gf, gm_dual, mf_dual, step_size, true, "qgb_gf_evolve_fa_dual");
}

int qgb_set_gm_force_dual(qgb_field* fd_, const qgb_field* gf_, const qgb_field* f_)
{
  const char* what = "qgb_set_gm_force_dual";
  Meta fd, gf, f;
  FA_RC(meta_of(fd_, fd, what));
  FA_RC(meta_of(gf_, gf, what));
  FA_RC(meta_of(f_, f, what));
  FA_RC(check_links(what, {&fd, &gf, &f}));
  if (fd.d == gf.d || fd.d == f.d) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": output aliases an input");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  const dim3 grid = link_grid(gf.V, 4);
  if (gf.prec == QGB_F64)
    k_force_dual<double><<<grid, FA_BS, 0, st>>>(gf.V, (Cx<double>*)fd.d, (const Cx<double>*)gf.d,
                                                 (const Cx<double>*)f.d);
  else
    k_force_dual<float><<<grid, FA_BS, 0, st>>>(gf.V, (Cx<float>*)fd.d, (const Cx<float>*)gf.d,
                                                (const Cx<float>*)f.d);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

int qgb_project_gauge_transform(qgb_field* gm_, qgb_field* gmd_, const qgb_field* mf_, const qgb_field* mfd_,
                                double* change_qnorm)
{
  const char* what = "qgb_project_gauge_transform";
  Meta gm, gmd, mf, mfd;
  FA_RC(meta_of(gm_, gm, what));
  FA_RC(meta_of(gmd_, gmd, what));
  FA_RC(meta_of(mf_, mf, what));
  FA_RC(meta_of(mfd_, mfd, what));
  FA_RC(check_links(what, {&gm, &gmd}));
  FA_RC(check_mass(what, mf, gm));
  FA_RC(check_mass(what, mfd, gm));
  if (gm.d == gmd.d) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": gm and gm_dual are the same field");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  const Geo g = geo_of(gm);
  const size_t creal = gm.prec == QGB_F64 ? sizeof(double) : sizeof(float);
  void* ag = nullptr;
  FA_RC(qgb::scratch_buffer((size_t)padded_sites(g.V) * 18 * creal, gm.prec == QGB_F64 ? TAG_AG64 : TAG_AG32, &ag));
  double* partials = nullptr;
  FA_RC(partials_buffer(g.V, &partials));
  const double *m1 = (const double*)mf.d, *m2 = (const double*)mfd.d;
  if (gm.prec == QGB_F64) {
    k_gt_average<double><<<site_grid(g.V), FA_BS, 0, st>>>(g, (const Cx<double>*)gm.d, (const Cx<double>*)gmd.d, m1,
                                                          m2, (Cx<double>*)ag, partials);
    FA_CUDA(cudaGetLastError());
    qgb::add_launches(1);
    k_gt_subtract<double><<<link_grid(g.V, 4), FA_BS, 0, st>>>(g, (Cx<double>*)gm.d, (Cx<double>*)gmd.d, m1, m2,
                                                              (const Cx<double>*)ag);
  } else {
    k_gt_average<float><<<site_grid(g.V), FA_BS, 0, st>>>(g, (const Cx<float>*)gm.d, (const Cx<float>*)gmd.d, m1, m2,
                                                         (Cx<float>*)ag, partials);
    FA_CUDA(cudaGetLastError());
    qgb::add_launches(1);
    k_gt_subtract<float><<<link_grid(g.V, 4), FA_BS, 0, st>>>(g, (Cx<float>*)gm.d, (Cx<float>*)gmd.d, m1, m2,
                                                             (const Cx<float>*)ag);
  }
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  if (!change_qnorm) return QGB_OK;  // nothing to read back: stay asynchronous
  double qn = 0.0;
  FA_RC(sum_to_host(st, partials, (int)site_grid(g.V), &qn));
  *change_qnorm = qn / (double)g.V;
  return QGB_OK;
}

int qgb_set_gauge_transform_momentum(qgb_field* gm_, qgb_field* gmd_, const qgb_field* gtm_)
{
  const char* what = "qgb_set_gauge_transform_momentum";
  Meta gm, gmd, gtm;
  FA_RC(meta_of(gm_, gm, what));
  FA_RC(meta_of(gmd_, gmd, what));
  FA_RC(meta_of(gtm_, gtm, what));
  FA_RC(check_links(what, {&gm, &gmd}));
  if (gtm.kind != QGB_KIND_COLOR_MATRIX || gtm.mult != 1 || gtm.prec != gm.prec || !same_sites(gtm, gm))
    return ffail(QGB_ERR_MISMATCH, std::string(what) + ": gtm must be a color-matrix field of multiplicity 1 on the "
                                                       "same lattice and in the same precision");
  if (gm.d == gmd.d) return ffail(QGB_ERR_INVALID_ARG, std::string(what) + ": gm and gm_dual are the same field");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  const Geo g = geo_of(gm);
  if (gm.prec == QGB_F64)
    k_gt_momentum<double><<<link_grid(g.V, 4), FA_BS, 0, st>>>(g, (Cx<double>*)gm.d, (Cx<double>*)gmd.d,
                                                              (const Cx<double>*)gtm.d);
  else
    k_gt_momentum<float><<<link_grid(g.V, 4), FA_BS, 0, st>>>(g, (Cx<float>*)gm.d, (Cx<float>*)gmd.d,
                                                             (const Cx<float>*)gtm.d);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

int qgb_dot_gauge_momentum(qgb_field* f_, const qgb_field* a_, const qgb_field* b_)
{
  const char* what = "qgb_dot_gauge_momentum";
  Meta f, a, b;
  FA_RC(meta_of(f_, f, what));
  FA_RC(meta_of(a_, a, what));
  FA_RC(meta_of(b_, b, what));
  FA_RC(check_links(what, {&a, &b}));
  if (f.kind != QGB_KIND_REAL || f.mult != 4 || f.prec != QGB_F64 || !same_sites(f, a))
    return ffail(QGB_ERR_MISMATCH, std::string(what) + ": f must be an FP64 real field of multiplicity 4");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  if (a.prec == QGB_F64)
    k_dot<double><<<link_grid(a.V, 4), FA_BS, 0, st>>>(a.V, (double*)f.d, (const Cx<double>*)a.d,
                                                      (const Cx<double>*)b.d);
  else
    k_dot<float><<<link_grid(a.V, 4), FA_BS, 0, st>>>(a.V, (double*)f.d, (const Cx<float>*)a.d,
                                                     (const Cx<float>*)b.d);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  return QGB_OK;
}

int qgb_field_set_u_rand(qgb_field* f, const uint32_t rs[24], double upper, double lower)
{
  return rand_field(f, rs, upper, lower, false, "qgb_field_set_u_rand");
}

int qgb_field_set_g_rand(qgb_field* f, const uint32_t rs[24], double center, double sigma)
{
  return rand_field(f, rs, center, sigma, true, "qgb_field_set_g_rand");
}

int qgb_field_fill(qgb_field* f_, double value, const uint8_t* mask, int64_t n)
{
  const char* what = "qgb_field_fill";
  Meta f;
  FA_RC(meta_of(f_, f, what));
  if (f.kind != QGB_KIND_REAL) return ffail(QGB_ERR_MISMATCH, std::string(what) + ": needs a real field");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  uint8_t* dm = nullptr;
  if (mask) FA_RC(upload_mask(st, mask, n, f, &dm));
  const dim3 grid = link_grid(f.V, f.mult);
  if (f.prec == QGB_F64) k_fill_real<double><<<grid, FA_BS, 0, st>>>(f.V, f.mult, (double*)f.d, value, dm);
  else k_fill_real<float><<<grid, FA_BS, 0, st>>>(f.V, f.mult, (float*)f.d, value, dm);
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  if (mask) FA_CUDA(cudaStreamSynchronize(st));  // the host mask may be freed on return
  return QGB_OK;
}

int qgb_field_set_selected(qgb_field* dst_, const qgb_field* src_, const uint8_t* mask, int64_t n)
{
  const char* what = "qgb_field_set_selected";
  Meta dst, src;
  FA_RC(meta_of(dst_, dst, what));
  FA_RC(meta_of(src_, src, what));
  if (dst.kind != src.kind || dst.mult != src.mult || dst.prec != src.prec || !same_sites(dst, src))
    return ffail(QGB_ERR_MISMATCH, std::string(what) + ": fields differ in kind, multiplicity, lattice or precision");
  cudaStream_t st;
  FA_RC(qgb::library_stream(&st));
  uint8_t* dm = nullptr;
  FA_RC(upload_mask(st, mask, n, dst, &dm));
  const dim3 grid = link_grid(dst.V, dst.mult);
  const bool color = dst.kind == QGB_KIND_COLOR_MATRIX;
  if (dst.prec == QGB_F64) {
    if (color) k_masked_copy<double, 18><<<grid, FA_BS, 0, st>>>(dst.V, dst.mult, (double*)dst.d, (const double*)src.d, dm);
    else k_masked_copy<double, 1><<<grid, FA_BS, 0, st>>>(dst.V, dst.mult, (double*)dst.d, (const double*)src.d, dm);
  } else {
    if (color) k_masked_copy<float, 18><<<grid, FA_BS, 0, st>>>(dst.V, dst.mult, (float*)dst.d, (const float*)src.d, dm);
    else k_masked_copy<float, 1><<<grid, FA_BS, 0, st>>>(dst.V, dst.mult, (float*)dst.d, (const float*)src.d, dm);
  }
  FA_CUDA(cudaGetLastError());
  qgb::add_launches(1);
  FA_CUDA(cudaStreamSynchronize(st));  // the host mask may be freed on return
  return QGB_OK;
}

}  // extern "C"
