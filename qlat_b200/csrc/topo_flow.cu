// topo_flow.cu -- the flows and site fields of the topology measurement
// (the reference's instanton_map.py:91-224 gf_flow_topo and
// gf_energy_derivative_density_field_topo, wilson-flow.cpp:164-236
// set_plaq_flow_z, qcd.cpp:33-62, 295-341, 391-414 gf_plaq_field and the
// clover plaquette-action densities) and per-timeslice / min / max
// reductions of real fields (glb_sum_tslice, glb_min, glb_max).
//
// The plaquette-weighted flows (Shrink, Freeze, Localize, Preserve) move each
// link along the Wilson-flow force in which every plaquette carries its own
// factor f(p), p = Re tr P / 3 of that plaquette; the step is scaled by 1 /
// norm, norm the largest factor over the lattice, so that the most weighted
// plaquette flows at the nominal rate.  The factors are functions of the
// plaquette field, evaluated in the force kernel with the same IEEE operations
// in the same order as the reference's numpy expressions (no contraction).
//
// Layout as in gauge_common.cuh; a real field with multiplicity m holds
// component k of site s at lay_index<1>(V, k, 0, s).  One thread per site or
// per link; reductions in FP64 in a fixed order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

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
int scratch_buffer(size_t bytes, int tag, void** out);
void add_launches(int64_t n);
}  // namespace qgb

namespace
{
using namespace qgb;

constexpr int TF_BS = 256;

// fixed-order block sum of one value per thread into partials[blockIdx.x]
__device__ __forceinline__ void block_sum_store_tf(double v, double* partials)
{
  __shared__ double sm[TF_BS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < TF_BS / 32; ++i) t += sm[i];
    partials[blockIdx.x] = t;
  }
}

__global__ void k_sum_partials_tf(const double* partials, int n, double* out)
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

// plane index of (mu, nu), mu != nu: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
// (gf_plaq_field_no_comm, qcd.cpp:312-317; the table of wilson-flow.cpp:170-181)
__host__ __device__ __forceinline__ int plane_of(int mu, int nu)
{
  const int a = mu < nu ? mu : nu, b = mu < nu ? nu : mu;
  return a == 0 ? b - 1 : (a == 1 ? b + 1 : 5);
}

// gf_plaq_field (qcd.cpp:295-341): p[m](x) = Re tr(U_a(x) U_b(x+a) (U_b(x) U_a(x+b))^+) / 3
// for the six planes (a, b) in plane_of order.
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_plaq_field(Geo g, const Cx<R>* Up, double* out)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const CField<R> U{Up, g.V};
  const Coord x = coord_of(g, s);
#pragma unroll 1
  for (int p = 0; p < 6; ++p) {
    const int a = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int b = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
    const M3<R> A = mul(U.ld(s, a), U.ld(site_rt(g, x, a, 1, b, 0), b));
    const M3<R> B = mul(U.ld(s, b), U.ld(site_rt(g, x, a, 0, b, 1), a));
    out[lay_index<1>(g.V, p, 0, s)] = (double)re_tr_mul_adj(A, B) / 3.0;
  }
}

// clf_plaq_action_density (qcd.cpp:33-50) from the plaquette field: the clover
// C of plane (a, b) at x averages the four plaquettes with a corner at x, whose
// real traces are those of the plaquettes at x, x-a, x-b, x-a-b; the density
// is sum over the planes (all six, or the spatial (0,1) (0,2) (1,2)) of
// 1 - Re tr C / 3.
__global__ void __launch_bounds__(TF_BS) k_plaq_action_density(Geo g, const double* pf, double* out, int spatial)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const Coord x = coord_of(g, s);
  double sum = 0.0;
  for (int p = 0; p < 6; ++p) {
    if (spatial && (p == 2 || p == 4 || p == 5)) continue;
    const int a = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int b = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
    const double t = pf[lay_index<1>(g.V, p, 0, s)] + pf[lay_index<1>(g.V, p, 0, site_rt(g, x, a, -1, b, 0))] +
                     pf[lay_index<1>(g.V, p, 0, site_rt(g, x, a, 0, b, -1))] +
                     pf[lay_index<1>(g.V, p, 0, site_rt(g, x, a, -1, b, -1))];
    sum += 1.0 - 0.25 * t;
  }
  out[lay_index<1>(g.V, 0, 0, s)] = sum;
}

// plaquette weights of the flows (instanton_map.py:162-188), from p = plaq / 3
enum PlaqKind { PK_FIELD = 0, PK_SHRINK = 1, PK_FREEZE = 2, PK_LOCALIZE = 3, PK_PRESERVE = 4 };

__device__ __forceinline__ double plaq_weight(int kind, double p)
{
  switch (kind) {
    case PK_SHRINK:  // eps / (1 - p + eps) + base, eps = 0.005, base = 0.5
      return __dadd_rn(__ddiv_rn(0.005, __dadd_rn(__dsub_rn(1.0, p), 0.005)), 0.5);
    case PK_FREEZE:  // 1 - p
      return __dsub_rn(1.0, p);
    case PK_LOCALIZE:  // eps / (1 - p + eps) + base (1 - p), eps = 0.002, base = 50
      return __dadd_rn(__ddiv_rn(0.002, __dadd_rn(__dsub_rn(1.0, p), 0.002)), __dmul_rn(50.0, __dsub_rn(1.0, p)));
    case PK_PRESERVE:  // max(1, base (1 - p)), base = 50
      return fmax(1.0, __dmul_rn(50.0, __dsub_rn(1.0, p)));
    default:
      return p;
  }
}

// set_plaq_flow_z (wilson-flow.cpp:164-236): per link
//   S = sum_{nu != mu} f_m(x) U_nu(x) U_mu(x+nu) U_nu(x+mu)^+ + f_m(x-nu) U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu),
//   Z = TA(-U_mu(x) S^+),  m = plane_of(mu, nu),
// f the given factor field (PK_FIELD) or the weight of the plaquette field.
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_plaq_flow_z(Geo g, const Cx<R>* Up, const double* f, int kind, Cx<R>* Z)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const int mu = blockIdx.y;
  const CField<R> U{Up, g.V};
  const Coord x = coord_of(g, s);
  M3<R> acc = m3_zero<R>();
#pragma unroll 1
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    const int m = plane_of(mu, nu);
    const long xn = site_rt(g, x, nu, 1, mu, 0);    // x + nu
    const long xm = site_rt(g, x, mu, 1, nu, 0);    // x + mu
    const long xb = site_rt(g, x, nu, -1, mu, 0);   // x - nu
    const long xbm = site_rt(g, x, nu, -1, mu, 1);  // x - nu + mu
    const double f1 = plaq_weight(kind, __ldg(f + lay_index<1>(g.V, m, 0, s)));
    const double f2 = plaq_weight(kind, __ldg(f + lay_index<1>(g.V, m, 0, xb)));
    const M3<R> w1 = mul_adj(mul(U.ld(s, nu), U.ld(xn, mu)), U.ld(xm, nu));
    const M3<R> w2 = mul(adj_mul(U.ld(xb, nu), U.ld(xb, mu)), U.ld(xbm, nu));
    axpy(acc, (R)f1, w1);
    axpy(acc, (R)f2, w2);
  }
  const M3<R> fz = mul_adj(U.ld(s, mu), acc);
  WField<R>{Z, g.V}.st(s, mu, traceless_antiherm(scale((R)-1, fz)));
}

// gf_energy_density_dir_field (wilson-flow.cpp:53-95): per site and plane
// (a, b) in plane_of order, -Re tr(G G) with G = TA(C), C the clover average
// of the four plaquettes with a corner at the site, each walked from the site
// as in gf_clover_leaf_no_comm (qcd.cpp:10-31).
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_energy_density_dir(Geo g, const Cx<R>* Up, double* out)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const CField<R> U{Up, g.V};
  const Coord x = coord_of(g, s);
#pragma unroll 1
  for (int p = 0; p < 6; ++p) {
    const int a = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int b = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
    const long xa = site_rt(g, x, a, 1, b, 0), xb = site_rt(g, x, a, 0, b, 1);
    const long xma = site_rt(g, x, a, -1, b, 0), xmb = site_rt(g, x, a, 0, b, -1);
    const long xmab = site_rt(g, x, a, -1, b, -1), xmab2 = site_rt(g, x, a, -1, b, 1),
               xamb = site_rt(g, x, a, 1, b, -1);
    // (a, b, -a, -b): U_a(x) U_b(x+a) U_a(x+b)^+ U_b(x)^+
    M3<R> c = mul_adj(mul_adj(mul(U.ld(s, a), U.ld(xa, b)), U.ld(xb, a)), U.ld(s, b));
    // (-a, -b, a, b): U_a(x-a)^+ U_b(x-a-b)^+ U_a(x-a-b) U_b(x-b)
    add_to(c, mul(mul(adj_mul(U.ld(xma, a), adj(U.ld(xmab, b))), U.ld(xmab, a)), U.ld(xmb, b)));
    // (b, -a, -b, a): U_b(x) U_a(x-a+b)^+ U_b(x-a)^+ U_a(x-a)
    add_to(c, mul(mul_adj(mul_adj(U.ld(s, b), U.ld(xmab2, a)), U.ld(xma, b)), U.ld(xma, a)));
    // (-b, a, b, -a): U_b(x-b)^+ U_a(x-b) U_b(x-b+a) U_a(x)^+
    add_to(c, mul_adj(mul(adj_mul(U.ld(xmb, b), U.ld(xmb, a)), U.ld(xamb, b)), U.ld(s, a)));
    const M3<R> G = traceless_antiherm(scale(R(0.25), c));
    out[lay_index<1>(g.V, p, 0, s)] = -(double)re_tr_mul(G, G);
  }
}

// gf_avg_wilson_loop (qcd-utils.cpp:359-400): per site, the sum over the
// spatial directions i of Re tr of the l x t loop from the site: l links along
// +i, t along +3, l along -i, t along -3, multiplied in that order as
// gf_avg_wilson_line walks its path segments.
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_wilson_loop(Geo g, const Cx<R>* Up, int l, int t, double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (s < g.V) {
    const CField<R> U{Up, g.V};
    const Coord x0 = coord_of(g, s);
    for (int i = 0; i < 3; ++i) {
      int c[4] = {x0.c[0], x0.c[1], x0.c[2], x0.c[3]};
      auto site = [&]() {
        return (long)c[0] + (long)g.d[0] * ((long)c[1] + (long)g.d[1] * ((long)c[2] + (long)g.d[2] * (long)c[3]));
      };
      M3<R> m = m3_unit<R>();
      for (int k = 0; k < l; ++k) {
        m = mul(m, U.ld(site(), i));
        c[i] = c[i] + 1 == g.d[i] ? 0 : c[i] + 1;
      }
      for (int k = 0; k < t; ++k) {
        m = mul(m, U.ld(site(), 3));
        c[3] = c[3] + 1 == g.d[3] ? 0 : c[3] + 1;
      }
      for (int k = 0; k < l; ++k) {
        c[i] = c[i] == 0 ? g.d[i] - 1 : c[i] - 1;
        m = mul_adj(m, U.ld(site(), i));
      }
      for (int k = 0; k < t; ++k) {
        c[3] = c[3] == 0 ? g.d[3] - 1 : c[3] - 1;
        m = mul_adj(m, U.ld(site(), 3));
      }
      v += (double)re_tr(m);
    }
  }
  block_sum_store_tf(v, partials);
}

// per-block min and max of each component of a real field (blockDim TF_BS)
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_min_max(long V, int mult, const R* f, double* part)
{
  __shared__ double smin[TF_BS], smax[TF_BS];
  const int m = blockIdx.y;
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const double v = s < V ? (double)f[lay_index<1>(V, m, 0, s)] : 0.0;
  smin[threadIdx.x] = s < V ? v : INFINITY;
  smax[threadIdx.x] = s < V ? v : -INFINITY;
  __syncthreads();
  for (int w = TF_BS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + w]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * ((long)m * gridDim.x + blockIdx.x)] = smin[0];
    part[2 * ((long)m * gridDim.x + blockIdx.x) + 1] = smax[0];
  }
}

__global__ void k_min_max_final(int nblk, int mult, const double* part, double* out)
{
  const int m = threadIdx.x;
  if (m >= mult) return;
  double a = INFINITY, b = -INFINITY;
  for (int i = 0; i < nblk; ++i) {
    a = fmin(a, part[2 * ((long)m * nblk + i)]);
    b = fmax(b, part[2 * ((long)m * nblk + i) + 1]);
  }
  out[2 * m] = a;
  out[2 * m + 1] = b;
}

// glb_sum_tslice (field_base.pyx:750-762): out[t * mult + m] = sum over the
// sites with x[t_dir] = t of component m; one block per (t, m), fixed order.
template <typename R>
__global__ void __launch_bounds__(TF_BS) k_sum_tslice(Geo g, int mult, int t_dir, const R* f, double* out)
{
  __shared__ double sm[TF_BS];
  const int t = blockIdx.x, m = blockIdx.y;
  const long nslice = g.V / g.d[t_dir];
  double acc = 0.0;
  for (long i = threadIdx.x; i < nslice; i += blockDim.x) {
    // the i-th site of slice t: the other three coordinates, x fastest
    long r = i;
    int c[4];
    for (int k = 0; k < 4; ++k) {
      if (k == t_dir) {
        c[k] = t;
        continue;
      }
      c[k] = (int)(r % g.d[k]);
      r /= g.d[k];
    }
    const long s = (long)c[0] + (long)g.d[0] * ((long)c[1] + (long)g.d[1] * ((long)c[2] + (long)g.d[2] * (long)c[3]));
    acc += (double)f[lay_index<1>(g.V, m, 0, s)];
  }
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = TF_BS / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(long)t * mult + m] = sm[0];
}

// |f| elementwise over the sites of a real field (abs_topo_field[:] = np.abs(topo_field[:]))
template <typename R>
__global__ void k_abs(long V, R* f)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const long i = lay_index<1>(V, blockIdx.y, 0, s);
  f[i] = fabs(f[i]);
}

// ---- host side ---------------------------------------------------------------

int tfail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

#define TF_CUDA(expr)                                                                                        \
  do {                                                                                                       \
    cudaError_t e_ = (expr);                                                                                 \
    if (e_ != cudaSuccess) return tfail(QGB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define TF_RC(expr)              \
  do {                           \
    int r_ = (expr);             \
    if (r_ != QGB_OK) return r_; \
  } while (0)
#define TF_LAUNCHED()                 \
  do {                                \
    TF_CUDA(cudaGetLastError());      \
    qgb::add_launches(1);             \
  } while (0)

struct Meta {
  int32_t ts[4] = {0, 0, 0, 0};
  int32_t mult = 0, kind = -1, prec = 0;
  Geo g;
  void* d = nullptr;
};

int meta_of(const qgb_field* f, Meta& m, const char* what)
{
  if (!f) return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": null field");
  TF_RC(qgb_field_info(f, m.ts, &m.mult, &m.kind, &m.prec));
  for (int i = 0; i < 4; ++i) m.g.d[i] = m.ts[i];
  m.g.V = (long)m.ts[0] * m.ts[1] * m.ts[2] * m.ts[3];
  m.d = qgb::field_data(f);
  return QGB_OK;
}

bool same_sites(const Meta& a, const Meta& b)
{
  for (int i = 0; i < 4; ++i)
    if (a.ts[i] != b.ts[i]) return false;
  return true;
}

int check_gauge(const Meta& gf, const char* what)
{
  if (gf.kind != QGB_KIND_COLOR_MATRIX || gf.mult != 4)
    return tfail(QGB_ERR_MISMATCH, std::string(what) + ": need a gauge field (color matrices, multiplicity 4)");
  return QGB_OK;
}

int check_real(const Meta& f, const Meta& gf, int mult, const char* what)
{
  if (f.kind != QGB_KIND_REAL || f.prec != QGB_F64 || (mult > 0 && f.mult != mult) || !same_sites(f, gf))
    return tfail(QGB_ERR_MISMATCH, std::string(what) + ": need an FP64 real field of multiplicity " +
                                       std::to_string(mult) + " on the gauge field's lattice");
  return QGB_OK;
}

enum { TAG_PLAQ = 0x7B000, TAG_Z64, TAG_Z32, TAG_MM_PART, TAG_MM_OUT, TAG_TS_OUT, TAG_WL_PART, TAG_WL_OUT };

unsigned blocks_of(long V) { return (unsigned)((V + TF_BS - 1) / TF_BS); }

int plaq_field_dev(cudaStream_t st, const Meta& gf, double* out)
{
  if (gf.prec == QGB_F64)
    k_plaq_field<double><<<blocks_of(gf.g.V), TF_BS, 0, st>>>(gf.g, (const Cx<double>*)gf.d, out);
  else
    k_plaq_field<float><<<blocks_of(gf.g.V), TF_BS, 0, st>>>(gf.g, (const Cx<float>*)gf.d, out);
  TF_LAUNCHED();
  return QGB_OK;
}

// the plaquette field in a library buffer
int plaq_scratch(cudaStream_t st, const Meta& gf, double** out)
{
  void* p = nullptr;
  TF_RC(qgb::scratch_buffer((size_t)padded_sites(gf.g.V) * 6 * sizeof(double), TAG_PLAQ, &p));
  *out = (double*)p;
  return plaq_field_dev(st, gf, *out);
}

template <typename R>
int min_max_dev(cudaStream_t st, long V, int mult, const R* f, double* host_out)
{
  const unsigned nb = blocks_of(V);
  void *part = nullptr, *out = nullptr;
  TF_RC(qgb::scratch_buffer((size_t)nb * mult * 2 * sizeof(double), TAG_MM_PART, &part));
  TF_RC(qgb::scratch_buffer((size_t)mult * 2 * sizeof(double), TAG_MM_OUT, &out));
  k_min_max<<<dim3(nb, (unsigned)mult), TF_BS, 0, st>>>(V, mult, f, (double*)part);
  TF_LAUNCHED();
  k_min_max_final<<<1, 32 * ((mult + 31) / 32), 0, st>>>((int)nb, mult, (const double*)part, (double*)out);
  TF_LAUNCHED();
  TF_CUDA(cudaMemcpyAsync(host_out, out, (size_t)mult * 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  TF_CUDA(cudaStreamSynchronize(st));
  return QGB_OK;
}

template <typename R>
int plaq_flow_z_dev(cudaStream_t st, const Meta& gf, const double* f, int kind, void* Z)
{
  k_plaq_flow_z<R><<<dim3(blocks_of(gf.g.V), 4), TF_BS, 0, st>>>(gf.g, (const Cx<R>*)gf.d, f, kind, (Cx<R>*)Z);
  TF_LAUNCHED();
  return QGB_OK;
}

// the flow's norm from the lattice's smallest and largest plaquette (instanton_map.py:166-188)
double flow_norm(int kind, double pmin, double pmax)
{
  switch (kind) {
    case PK_SHRINK:
      return 0.005 / (1.0 - pmax + 0.005) + 0.5;
    case PK_FREEZE:
      return 1.0 - pmin;
    case PK_LOCALIZE: {
      const double a = 0.002 / (1.0 - pmax + 0.002) + 50.0 * (1.0 - pmax);
      const double b = 0.002 / (1.0 - pmin + 0.002) + 50.0 * (1.0 - pmin);
      return a > b ? a : b;
    }
    case PK_PRESERVE: {
      const double v = 50.0 * (1.0 - pmin);
      return v > 1.0 ? v : 1.0;
    }
    default:
      return 1.0;
  }
}

}  // namespace

extern "C" {

int qgb_gf_plaq_field(qgb_field* f_plaq, const qgb_field* gf_)
{
  const char* what = "qgb_gf_plaq_field";
  Meta gf, f;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(meta_of(f_plaq, f, what));
  TF_RC(check_gauge(gf, what));
  TF_RC(check_real(f, gf, 6, what));
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  return plaq_field_dev(st, gf, (double*)f.d);
}

int qgb_gf_energy_density_dir_field(qgb_field* fd, const qgb_field* gf_)
{
  const char* what = "qgb_gf_energy_density_dir_field";
  Meta gf, f;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(meta_of(fd, f, what));
  TF_RC(check_gauge(gf, what));
  TF_RC(check_real(f, gf, 6, what));
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  if (gf.prec == QGB_F64)
    k_energy_density_dir<double><<<blocks_of(gf.g.V), TF_BS, 0, st>>>(gf.g, (const Cx<double>*)gf.d, (double*)f.d);
  else
    k_energy_density_dir<float><<<blocks_of(gf.g.V), TF_BS, 0, st>>>(gf.g, (const Cx<float>*)gf.d, (double*)f.d);
  TF_LAUNCHED();
  return QGB_OK;
}

int qgb_topology_charge_5(const qgb_field* gf, double* out) { return qgb_gf_topology(gf, out); }

int qgb_gf_avg_wilson_loop_normalized_tr(const qgb_field* gf_, int32_t l, int32_t t, double* out)
{
  const char* what = "qgb_gf_avg_wilson_loop_normalized_tr";
  Meta gf;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(check_gauge(gf, what));
  if (!out || l < 0 || t < 0) return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": bad argument");
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  const unsigned nb = blocks_of(gf.g.V);
  void *part = nullptr, *res = nullptr;
  TF_RC(qgb::scratch_buffer((size_t)nb * sizeof(double), TAG_WL_PART, &part));
  TF_RC(qgb::scratch_buffer(sizeof(double), TAG_WL_OUT, &res));
  if (gf.prec == QGB_F64)
    k_wilson_loop<double><<<nb, TF_BS, 0, st>>>(gf.g, (const Cx<double>*)gf.d, l, t, (double*)part);
  else
    k_wilson_loop<float><<<nb, TF_BS, 0, st>>>(gf.g, (const Cx<float>*)gf.d, l, t, (double*)part);
  TF_LAUNCHED();
  k_sum_partials_tf<<<1, 1024, 0, st>>>((const double*)part, (int)nb, (double*)res);
  TF_LAUNCHED();
  double h = 0.0;
  TF_CUDA(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, st));
  TF_CUDA(cudaStreamSynchronize(st));
  // average over the sites and the three spatial directions, Re tr / 3
  *out = h / (3.0 * (double)gf.g.V) / 3.0;
  return QGB_OK;
}

int qgb_gf_plaq_action_density_field(qgb_field* paf, const qgb_field* gf_, int32_t spatial)
{
  const char* what = "qgb_gf_plaq_action_density_field";
  Meta gf, f;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(meta_of(paf, f, what));
  TF_RC(check_gauge(gf, what));
  TF_RC(check_real(f, gf, 1, what));
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  double* pf = nullptr;
  TF_RC(plaq_scratch(st, gf, &pf));
  k_plaq_action_density<<<blocks_of(gf.g.V), TF_BS, 0, st>>>(gf.g, pf, (double*)f.d, spatial ? 1 : 0);
  TF_LAUNCHED();
  return QGB_OK;
}

int qgb_set_plaq_flow_z(qgb_field* z_, const qgb_field* gf_, const qgb_field* plaq_factor)
{
  const char* what = "qgb_set_plaq_flow_z";
  Meta gf, z, pf;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(meta_of(z_, z, what));
  TF_RC(meta_of(plaq_factor, pf, what));
  TF_RC(check_gauge(gf, what));
  TF_RC(check_gauge(z, what));
  TF_RC(check_real(pf, gf, 6, what));
  if (z.prec != gf.prec || !same_sites(z, gf)) return tfail(QGB_ERR_MISMATCH, std::string(what) + ": z differs from gf");
  if (z.d == gf.d) return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": z aliases gf");
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  if (gf.prec == QGB_F64) return plaq_flow_z_dev<double>(st, gf, (const double*)pf.d, PK_FIELD, z.d);
  return plaq_flow_z_dev<float>(st, gf, (const double*)pf.d, PK_FIELD, z.d);
}

int qgb_gf_flow_topo(qgb_field* gf_, double step_size, int32_t flow_kind, double c1, int32_t integrator,
                     double* advance)
{
  const char* what = "qgb_gf_flow_topo";
  Meta gf;
  TF_RC(meta_of(gf_, gf, what));
  TF_RC(check_gauge(gf, what));
  if (flow_kind == QGB_FLOW_TOPO_C1) {
    // gf_wilson_flow_step with the action's c1 (instanton_map.py:129-161)
    if (integrator == QGB_FLOW_INTEGRATOR_EULER) TF_RC(qgb_gf_wilson_flow_step_euler(gf_, step_size, c1));
    else if (integrator == QGB_FLOW_INTEGRATOR_RUNGE_KUTTA) TF_RC(qgb_gf_wilson_flow_step(gf_, step_size, c1));
    else return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": unknown integrator");
    if (advance) *advance = step_size;
    return QGB_OK;
  }
  if (flow_kind < QGB_FLOW_TOPO_SHRINK || flow_kind > QGB_FLOW_TOPO_PRESERVE)
    return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": unknown flow kind");
  // plaquette-weighted flows (instanton_map.py:162-190): one Euler step of
  // the weighted force, step_size / norm
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  double* pf = nullptr;
  TF_RC(plaq_scratch(st, gf, &pf));
  std::vector<double> mm(12);
  TF_RC(min_max_dev<double>(st, gf.g.V, 6, pf, mm.data()));
  double pmin = mm[0], pmax = mm[1];
  for (int k = 1; k < 6; ++k) {
    pmin = mm[2 * k] < pmin ? mm[2 * k] : pmin;
    pmax = mm[2 * k + 1] > pmax ? mm[2 * k + 1] : pmax;
  }
  const double norm = flow_norm(flow_kind, pmin, pmax);
  const size_t zbytes = (size_t)padded_sites(gf.g.V) * 4 * 9 * (gf.prec == QGB_F64 ? 16 : 8);
  void* Z = nullptr;
  TF_RC(qgb::scratch_buffer(zbytes, gf.prec == QGB_F64 ? TAG_Z64 : TAG_Z32, &Z));
  if (gf.prec == QGB_F64) {
    TF_RC(plaq_flow_z_dev<double>(st, gf, pf, flow_kind, Z));
    TF_CUDA(launch_evolve<double>(gf.g, gf.d, Z, step_size / norm, 1, 0, st));
  } else {
    TF_RC(plaq_flow_z_dev<float>(st, gf, pf, flow_kind, Z));
    TF_CUDA(launch_evolve<float>(gf.g, gf.d, Z, step_size / norm, 1, 0, st));
  }
  qgb::add_launches(1);
  if (advance) *advance = step_size / norm;
  return QGB_OK;
}

int qgb_field_glb_min_max(const qgb_field* f_, double* mins, double* maxs)
{
  const char* what = "qgb_field_glb_min_max";
  Meta f;
  TF_RC(meta_of(f_, f, what));
  if (f.kind != QGB_KIND_REAL) return tfail(QGB_ERR_MISMATCH, std::string(what) + ": need a real field");
  if (!mins && !maxs) return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": no output");
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  std::vector<double> mm((size_t)2 * f.mult);
  if (f.prec == QGB_F64) TF_RC(min_max_dev<double>(st, f.g.V, f.mult, (const double*)f.d, mm.data()));
  else TF_RC(min_max_dev<float>(st, f.g.V, f.mult, (const float*)f.d, mm.data()));
  for (int m = 0; m < f.mult; ++m) {
    if (mins) mins[m] = mm[2 * m];
    if (maxs) maxs[m] = mm[2 * m + 1];
  }
  return QGB_OK;
}

int qgb_field_glb_sum_tslice(const qgb_field* f_, int32_t t_dir, double* out)
{
  const char* what = "qgb_field_glb_sum_tslice";
  Meta f;
  TF_RC(meta_of(f_, f, what));
  if (f.kind != QGB_KIND_REAL) return tfail(QGB_ERR_MISMATCH, std::string(what) + ": need a real field");
  if (t_dir < 0 || t_dir > 3 || !out) return tfail(QGB_ERR_INVALID_ARG, std::string(what) + ": bad argument");
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  const int nt = f.ts[t_dir];
  const size_t n = (size_t)nt * f.mult;
  void* d = nullptr;
  TF_RC(qgb::scratch_buffer(n * sizeof(double), TAG_TS_OUT, &d));
  const dim3 grid((unsigned)nt, (unsigned)f.mult);
  if (f.prec == QGB_F64)
    k_sum_tslice<double><<<grid, TF_BS, 0, st>>>(f.g, f.mult, t_dir, (const double*)f.d, (double*)d);
  else
    k_sum_tslice<float><<<grid, TF_BS, 0, st>>>(f.g, f.mult, t_dir, (const float*)f.d, (double*)d);
  TF_LAUNCHED();
  TF_CUDA(cudaMemcpyAsync(out, d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  TF_CUDA(cudaStreamSynchronize(st));
  return QGB_OK;
}

int qgb_field_abs(qgb_field* f_)
{
  const char* what = "qgb_field_abs";
  Meta f;
  TF_RC(meta_of(f_, f, what));
  if (f.kind != QGB_KIND_REAL) return tfail(QGB_ERR_MISMATCH, std::string(what) + ": need a real field");
  cudaStream_t st;
  TF_RC(qgb::library_stream(&st));
  const dim3 grid(blocks_of(f.g.V), (unsigned)f.mult);
  if (f.prec == QGB_F64) k_abs<double><<<grid, TF_BS, 0, st>>>(f.g.V, (double*)f.d);
  else k_abs<float><<<grid, TF_BS, 0, st>>>(f.g.V, (float*)f.d);
  TF_LAUNCHED();
  return QGB_OK;
}

}  // extern "C"
