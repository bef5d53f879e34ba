// noalloc.cu -- gauge-action sums for callers that cannot allocate GPU memory.
//
// Some callers of this library cannot call cudaMalloc: a host that has handed
// the device memory to its own pool (a framework's caching allocator, a solver
// with a fixed memory budget set at start-up), or one that cannot afford the
// device-wide synchronisation an allocation or free may cause while its other
// streams are busy.  The regular entry points allocate lazily (the library
// context, reduction scratch, staging), so this file provides one entry point
// that allocates nothing: the sums of (Re tr P - 3) over all plaquettes and
// rectangles (gf_sum_re_tr_plaq_node_no_comm / gf_sum_re_tr_rect_node_no_comm),
// read straight from a caller-owned device buffer in the reference memory
// image.
//
// Its only scratch is the per-block partial-sum array below, a file-scope
// device array that every GPU loading the library holds until the process
// exits.  Its device address is looked up once per device (on the first call
// made on that device) with cudaGetSymbolAddress; in host code the array's
// name is only a host-side stand-in, so the address is always passed to the
// kernels explicitly.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/qlat_b200.h"
#include "gauge_common.cuh"
#include "su3.cuh"

namespace qgb
{

// One double per block and per value (two values: plaquette and rectangle
// sums); blocks have 256 threads, one site per thread.
static const int NOALLOC_BS = 256;
static const long NOALLOC_MAX_BLOCKS = 65536;  // lattices up to 65536 * 256 = 2^24 sites
static __device__ __align__(256) double g_noalloc_partials[2 * NOALLOC_MAX_BLOCKS];  // 1 MiB

// Link (site, mu) of a gauge field in the reference memory image:
// complex128 at [((site * 4 + mu) * 9 + k)], k = 3 * row + col.
struct AosLinks {
  const Cx<double>* __restrict__ p;
  __device__ __forceinline__ M3<double> ld(long site, int mu) const
  {
    M3<double> r;
    const double2* q = reinterpret_cast<const double2*>(p + (site * 4 + mu) * 9);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double2 v = __ldg(q + k);
      r.e[k] = cx<double>(v.x, v.y);
    }
    return r;
  }
};

__global__ void __launch_bounds__(NOALLOC_BS) k_action_aos_noalloc(Geo g, const Cx<double>* links, int rect,
                                                                   double* partials)
{
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double sp = 0.0, sr = 0.0;
  if (s < g.V) {
    const AosLinks U{links};
    const Coord x = coord_of(g, s);
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      const int mu = p < 3 ? 0 : (p < 5 ? 1 : 2);
      const int nu = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
      // plaquette (mu, nu, -mu, -nu) = A B^+, A = U_mu(x) U_nu(x+mu), B = U_nu(x) U_mu(x+nu)
      const M3<double> A = mul(U.ld(s, mu), U.ld(site_rt(g, x, mu, 1, nu, 0), nu));
      const M3<double> B = mul(U.ld(s, nu), U.ld(site_rt(g, x, mu, 0, nu, 1), mu));
      sp += re_tr_mul_adj(A, B) - 3.0;
      if (rect) {
#pragma unroll 1
        for (int o = 0; o < 2; ++o) {
          // (a, a, b, -a, -a, -b) with the long side along a
          const int a = o == 0 ? mu : nu, b = o == 0 ? nu : mu;
          M3<double> A2 = mul(U.ld(s, a), U.ld(site_rt(g, x, a, 1, b, 0), a));
          A2 = mul(A2, U.ld(site_rt(g, x, a, 2, b, 0), b));
          M3<double> B2 = mul(U.ld(s, b), U.ld(site_rt(g, x, a, 0, b, 1), a));
          B2 = mul(B2, U.ld(site_rt(g, x, a, 1, b, 1), a));
          sr += re_tr_mul_adj(A2, B2) - 3.0;
        }
      }
    }
  }
  // fixed-order block reduction: warp shuffles, then the warp sums in order
  __shared__ double sm[2][NOALLOC_BS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sp += __shfl_down_sync(0xffffffffu, sp, o);
    sr += __shfl_down_sync(0xffffffffu, sr, o);
  }
  if (lane == 0) {
    sm[0][w] = sp;
    sm[1][w] = sr;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < NOALLOC_BS / 32; ++i) {
      a += sm[0][i];
      b += sm[1][i];
    }
    partials[blockIdx.x] = a;                 // every block overwrites its own slots,
    partials[gridDim.x + blockIdx.x] = b;     // so nothing needs clearing between calls
  }
}

__global__ void __launch_bounds__(1024) k_finalize_noalloc(const double* partials, int blocks, int rect, double* out)
{
  __shared__ double sm[32];
  for (int k = 0; k < 2; ++k) {
    double t = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) t += partials[(long)k * blocks + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sm[i];
      out[k] = (k == 1 && !rect) ? 0.0 : r;
    }
    __syncthreads();
  }
}

}  // namespace qgb

namespace qgb
{
void set_last_error(const std::string& msg);  // capi.cu: the message qgb_last_error() returns
void add_launches(int64_t n);                 // capi.cu: the count qgb_launch_count() returns
}

namespace
{
std::mutex g_noalloc_mu;
const int NOALLOC_MAX_DEVICES = 64;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

int noalloc_fail(int code, const std::string& msg)
{
  qgb::set_last_error(msg);
  return code;
}
}  // namespace

extern "C" {

int qgb_gf_action_sums_noalloc(const double* links_dev, const int32_t total_site[4], int32_t rect, double* out_dev,
                               void* stream)
{
  if (!links_dev || !total_site || !out_dev)
    return noalloc_fail(QGB_ERR_INVALID_ARG, "qgb_gf_action_sums_noalloc: null argument");
  // the kernels read links as 16-byte complex128 pairs and write doubles
  if ((reinterpret_cast<uintptr_t>(links_dev) & 15) != 0 || (reinterpret_cast<uintptr_t>(out_dev) & 7) != 0)
    return noalloc_fail(QGB_ERR_INVALID_ARG,
                        "qgb_gf_action_sums_noalloc: links_dev must be 16-byte and out_dev 8-byte aligned");
  qgb::Geo g;
  g.V = 1;
  g.off = 0;
  for (int i = 0; i < 4; ++i) {
    if (total_site[i] < 1 || total_site[i] > (1 << 20))
      return noalloc_fail(QGB_ERR_BAD_GEOMETRY, "qgb_gf_action_sums_noalloc: each lattice extent must be in [1, 2^20]");
    g.d[i] = total_site[i];
  }
  // The site count is checked against the scratch limit after every factor:
  // a running product of at most 2^24 sites times an extent of at most 2^20
  // stays below 2^44, so no product can wrap before it is refused.
  const long max_sites = qgb::NOALLOC_MAX_BLOCKS * qgb::NOALLOC_BS;
  for (int i = 0; i < 4; ++i) {
    g.V *= total_site[i];
    if (g.V > max_sites)
      return noalloc_fail(QGB_ERR_INVALID_ARG,
                          "qgb_gf_action_sums_noalloc: lattice " + std::to_string(total_site[0]) + "x" +
                              std::to_string(total_site[1]) + "x" + std::to_string(total_site[2]) + "x" +
                              std::to_string(total_site[3]) + " has more sites than the fixed scratch supports (at most " +
                              std::to_string(max_sites) + " sites)");
  }
  const long blocks = (g.V + qgb::NOALLOC_BS - 1) / qgb::NOALLOC_BS;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(QGB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return noalloc_fail(QGB_ERR_INVALID_ARG, "qgb_gf_action_sums_noalloc: device ordinal out of range");
  double* partials = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, qgb::g_noalloc_partials);
      if (e != cudaSuccess)
        return noalloc_fail(QGB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = static_cast<double*>(ptr);
    }
    partials = g_noalloc_ptr[dev];
  }
  // An error left pending by earlier, unrelated work is reported as such and
  // left in place for its owner, so that an error after the launches below is
  // theirs.
  e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return noalloc_fail(QGB_ERR_CUDA, std::string("qgb_gf_action_sums_noalloc: an earlier CUDA call left an error "
                                                  "pending, nothing launched: ") + cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  qgb::k_action_aos_noalloc<<<(unsigned)blocks, qgb::NOALLOC_BS, 0, st>>>(
      g, reinterpret_cast<const qgb::Cx<double>*>(links_dev), rect ? 1 : 0, partials);
  qgb::k_finalize_noalloc<<<1, 1024, 0, st>>>(partials, (int)blocks, rect ? 1 : 0, out_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(QGB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  qgb::add_launches(2);
  return QGB_OK;
}

}  // extern "C"
