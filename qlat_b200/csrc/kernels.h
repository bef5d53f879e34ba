// kernels.h -- host-side launch interface of the gauge kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qgb
{

// Device layout (gauge_common.cuh): sites in blocks of 32; the number of
// blocks and the padded site count of a field of V sites.
__host__ __device__ inline long site_blocks(long V) { return (V + 31) >> 5; }
__host__ __device__ inline long padded_sites(long V) { return site_blocks(V) << 5; }

struct Geo {
  int d[4];      // X, Y, Z, T
  long V;        // sites of this lattice
  long off = 0;  // index of its first site in a field holding several lattices
  // a sub-lattice of a larger one (time-slab decomposition): the site
  // reductions sum over the sites [r0, r1) only (r1 < 0: all), and the
  // per-site random streams of site s are those of global site s + rng_off
  long r0 = 0, r1 = -1;
  long rng_off = 0;
  // z-slab traversal (slab_order): when zs > 0, the linear work index of a
  // site kernel runs over the x-y planes of zs consecutive z in each time
  // slice before the next slice, slab by slab in z, so that the time slices
  // a running grid reads stay in L2 on large lattices
  int zs = 0;
  // one domain of a lattice decomposed over ranks in up to four directions
  // (qgb_field_set_domain): the field holds the owned box of sites with
  // coordinates [bl_k, bl_k + bn_k) in each direction k and a halo around it.
  // Kernels that only need the owned sites (the force) run over the box,
  // reductions sum over it, and the random streams of local site x are those
  // of global site (x + go) mod gd.  bn[0] == 0: no domain.
  int bl[4] = {0, 0, 0, 0}, bn[4] = {0, 0, 0, 0};
  int gd[4] = {0, 0, 0, 0}, go[4] = {0, 0, 0, 0};
};

__host__ __device__ inline bool has_box(const Geo& g) { return g.bn[0] > 0; }

// sites a site kernel that needs only the owned sites runs over
__host__ __device__ inline long work_sites(const Geo& g)
{
  return has_box(g) ? (long)g.bn[0] * g.bn[1] * g.bn[2] * g.bn[3] : g.V;
}

// local site of the w-th owned site (x fastest) of a domain
__host__ __device__ inline long box_site(const Geo& g, long w)
{
  long c = w;
  const long x0 = c % g.bn[0] + g.bl[0];
  c /= g.bn[0];
  const long x1 = c % g.bn[1] + g.bl[1];
  c /= g.bn[1];
  const long x2 = c % g.bn[2] + g.bl[2];
  const long x3 = c / g.bn[2] + g.bl[3];
  return x0 + (long)g.d[0] * (x1 + (long)g.d[1] * (x2 + (long)g.d[2] * x3));
}

__host__ __device__ inline bool in_box(const Geo& g, long s)
{
  long c = s;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long x = k < 3 ? c % g.d[k] : c;
    if (k < 3) c /= g.d[k];
    if (x < g.bl[k] || x >= g.bl[k] + g.bn[k]) return false;
  }
  return true;
}

__host__ __device__ inline bool in_reduce(const Geo& g, long s)
{
  return s >= g.r0 && (g.r1 < 0 || s < g.r1) && (!has_box(g) || in_box(g, s));
}

// global index of local site s for the per-site random streams
__host__ __device__ inline long rng_index(const Geo& g, long s)
{
  if (g.gd[0] == 0) return s + g.rng_off;
  long c = s, idx = 0, mul = 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long x = k < 3 ? c % g.d[k] : c;
    if (k < 3) c /= g.d[k];
    long y = (x + g.go[k]) % g.gd[k];
    if (y < 0) y += g.gd[k];
    idx += y * mul;
    mul *= g.gd[k];
  }
  return idx;
}

// One chain of a batch: its lattice, offset in the concatenated field and action.
struct ChainInfo {
  int d[4];
  long V;
  long off;
  double beta, c1;
};

// Force kernel output modes (force_impl.cuh).
enum ForceMode {
  FORCE_SET = 0,            // out = F
  FORCE_UPDATE = 1,         // P += dt F
  FORCE_EVOLVE = 2,         // U_out = unitarize(exp(eps F) U)
  FORCE_FLOW = 3,           // Z = a F + b Z_prev; U_out = unitarize(exp(eps Z) U)
  FORCE_UPDATE_EVOLVE = 4,  // P += dt F, then W = exp(ev_eps P) W on a second link field W
};

struct ForceArgs {
  const void* U;    // links in (SoA)
  void* out;        // F (SET) / P (UPDATE, UPDATE_EVOLVE) / U_out (EVOLVE, FLOW)
  const void* zp;   // FLOW: Z_prev (may be null when b == 0)
  void* z;          // FLOW: Z out (may be null)
  double beta, c1;  // gauge action
  double dt;        // UPDATE: P += dt F; EVOLVE/FLOW: exp step
  double a, b;      // FLOW combination
  int unitarize;    // EVOLVE/FLOW: unitarize after exp
  void* ev;         // UPDATE_EVOLVE: W, evolved in place (never read at other links, so W != U)
  double ev_eps;    // UPDATE_EVOLVE: exponential step of W
  int ev_unit;      // UPDATE_EVOLVE: 0 none, 1 unitarize in R, 2 unitarize with FP64 arithmetic
  int ev_from_u;    // UPDATE_EVOLVE: W = exp(ev_eps P) U at the thread's own link (W a second buffer)
                    // instead of evolving W in place
  void* corners;    // site map 5: scratch for the 16 two-link products per site (corner_id), or null
};

// Site map 5 of the force kernel keeps, per site, the 4 double links
// D_a(x) = U_a(x) U_a(x+a) (component a) and the 12 corners
// P_ab(x) = U_a(x) U_b(x+a), a != b (component corner_id(a, b)), as a
// 16-component color-matrix field in the blocked layout.
__host__ __device__ __forceinline__ int corner_id(int a, int b) { return 4 + 3 * a + (b < a ? b : b - 1); }
static const int N_CORNER_FIELDS = 16;

void init_constants();  // SHA-256 and log tables into constant memory (per device)

// `variant` indexes the autotuner's table of launch shapes (force_impl.cuh).
template <typename R>
cudaError_t launch_force(const Geo& g, ForceMode mode, const ForceArgs& a, int variant, cudaStream_t st);
int force_variant_count();
template <typename R>
cudaError_t launch_corners(const Geo& g, const void* U, void* C, cudaStream_t st);
// All chains of a batch in one launch (offs: nchain + 1 ascending offsets on the device).
template <typename R>
cudaError_t launch_force_batch(long Vtot, int nchain, const long* offs, const ChainInfo* chains, bool rect,
                               ForceMode mode, const ForceArgs& a, cudaStream_t st, int variant = 0);
int batch_force_variant_count();
int force_variant_info_c(int variant, int* bs, int* minb, int* split, int* map);

// U = exp(eps P) U (optionally unitarized; exp by Cayley-Hamilton series or the
// reference's order-20 Taylor series).
template <typename R>
cudaError_t launch_evolve(const Geo& g, void* U, const void* P, double eps, int unitarize, int taylor,
                          cudaStream_t st);

// Unitarize all links of a field with multiplicity m; arithmetic in C.
template <typename R, typename C>
cudaError_t launch_unitarize(const Geo& g, int m, void* U, cudaStream_t st);

// Reductions write n_values partial sums per block into `partials`
// (layout [value][block]); finalize sums them into results[slot..].
int reduce_blocks(const Geo& g);
template <typename R>
cudaError_t launch_gm_hamilton(const Geo& g, const void* P, double* partials, cudaStream_t st);
// The same sum (taken on the FP64 one of P and Q) and Q = P converted from RI
// to RO on every stored site, in one pass.
template <typename RI, typename RO>
cudaError_t launch_gm_hamilton_convert(const Geo& g, const void* P, void* Q, double* partials, cudaStream_t st);
// Q = unitarize(P) with FP64 arithmetic, P FP32 and Q FP64 (the conversion and
// k_unitarize<double, double> in one pass).
cudaError_t launch_unitarize_to_f64(const Geo& g, const void* P, void* Q, cudaStream_t st);
// values: 0 = sum(ReTr plaq - 3), 1 = sum(ReTr rect - 3) (if rect)
template <typename R>
cudaError_t launch_action(const Geo& g, const void* U, int rect, double* partials, cudaStream_t st,
                          void* copy_f32 = nullptr);
// values: 0 = energy density sum, 1 = clover topological charge sum; optional fields
template <typename R>
cudaError_t launch_clover(const Geo& g, const void* U, void* e_field, void* q_field, double* partials,
                          cudaStream_t st);
// values 0..4: the five terms of the 5-loop improved charge (qcd.cpp:425-489);
// optional fields: terms (real, multiplicity 5) and their per-site sum (multiplicity 1)
template <typename R>
cudaError_t launch_topology_5li(const Geo& g, const void* U, void* terms, void* total, double* partials,
                                cudaStream_t st);
template <typename R>
cudaError_t launch_qnorm(long n_reals, const void* x, double* partials, int blocks, cudaStream_t st);
cudaError_t launch_finalize(const double* partials, int n_values, int blocks, double* results, int slot,
                            cudaStream_t st);
// results[out] = results[a] + results[b] - results[c] (delta H bookkeeping on the device)
cudaError_t launch_combine(double* results, int out, int a, int b, int c, cudaStream_t st);

// Flow adjoint (adjoint.cu).
template <typename R>
cudaError_t launch_force_vjp(const Geo& g, const void* U, const void* Y, const void* lam_local, void* lam_out,
                             double beta, double c1, double a, cudaStream_t st);
template <typename R>
cudaError_t launch_flow_adj_local(long V, const void* lam, const void* Z, const void* mu_carry, double carry, double eps,
                                  void* mu_out, void* lam_local, cudaStream_t st);
template <typename R>
cudaError_t launch_dexp_adjoint(long V, int m, const void* omega, const void* lam, void* out, cudaStream_t st);
template <typename R>
cudaError_t launch_basis_to_matrix(long V, int m, const void* basis, void* fc, cudaStream_t st);
template <typename R>
cudaError_t launch_matrix_to_basis(long V, int m, const void* fc, void* basis, cudaStream_t st);

// Per-site RNG kernels; rs = 24 x u32 serialised RngState.
template <typename R>
cudaError_t launch_rand_momentum(const Geo& g, void* P, const uint32_t* rs24, double sigma,
                                 int* ambiguous, cudaStream_t st);
template <typename R>
cudaError_t launch_hot_start(const Geo& g, void* U, const uint32_t* rs24, double sigma, int n_step,
                             int* ambiguous, cudaStream_t st);

template <typename R>
cudaError_t launch_set_unit(const Geo& g, int m, void* U, cudaStream_t st);

// Batches of chains concatenated in one field (offs: nchain + 1 offsets, device).
template <typename R>
cudaError_t launch_rand_momentum_batch(long Vtot, int nchain, const long* offs, const uint32_t* rs24, double sigma,
                                       void* P, int* ambiguous, cudaStream_t st);
template <typename R>
cudaError_t launch_hot_start_batch(long Vtot, int nchain, const long* offs, const uint32_t* rs24, double sigma,
                                   int n_step, void* U, int* ambiguous, cudaStream_t st);
template <typename R>
cudaError_t launch_site_values_batch(long Vtot, int nchain, const long* offs, const ChainInfo* chains, int what,
                                     int rect, const void* F, double* vals, cudaStream_t st);
cudaError_t launch_segment_sum(int nchain, const long* offs, const double* vals, double* out, cudaStream_t st);
template <typename R>
cudaError_t launch_accept_batch(long Vtot, int nchain, const long* offs, const int* flags, void* dst, const void* src,
                                cudaStream_t st);
// y = a x + b y over n reals
template <typename R>
cudaError_t launch_axpby(long n, void* y, double a, const void* x, double b, cudaStream_t st);
// Layout conversion: reference image (AoS doubles, [site][m][k]) <-> device
// layout, for sites [off, off + n) of a field of Vf sites (the image holds
// those n sites).  k_per = 18 for color matrices, 1 for real fields.
template <typename R>
cudaError_t launch_aos_to_store(long Vf, long off, long n, int m, int k_per, const double* aos, void* store,
                                cudaStream_t st);
template <typename R>
cudaError_t launch_store_to_aos(long Vf, long off, long n, int m, int k_per, const void* store, double* aos,
                                cudaStream_t st);
// Elementwise conversion over n reals of two fields of the same layout
// (n counts the padded storage).
template <typename RI, typename RO>
cudaError_t launch_convert(long n, const void* in, void* out, cudaStream_t st);
// Copy the sites of the box [lo_k, lo_k + n_k) of every component of a field
// (V sites, m components of K entries of E = the entry type: a complex number
// of a color matrix or a real) into a contiguous buffer, entry (c, w) at
// c * nbox + w for c = component * K + entry and w the box site (x fastest),
// or back (unpack).
template <typename E>
cudaError_t launch_box_copy(const Geo& g, int m, int K, const int lo[4], const int n[4], void* field, void* buf,
                            bool unpack, cudaStream_t st);

}  // namespace qgb

namespace qgb
{
// Host-side RngState operations (same code as the device streams; the
// Gaussian draw uses the C library's log on the host, like the reference).
void rng_host_seed(uint32_t out[24], const char* seed);
bool rng_host_split(uint32_t out[24], const uint32_t rs[24], const char* sindex);
uint64_t rng_host_rand_gen(uint32_t rs[24]);
double rng_host_u_rand_gen(uint32_t rs[24], double upper, double lower);
double rng_host_g_rand_gen(uint32_t rs[24], double center, double sigma);
}  // namespace qgb
