// batch.cu -- many independent pure-gauge HMC chains advanced together.
//
// The chains (each with its own lattice, beta and c1) are concatenated into
// one field of Vtot sites (blocked layout of gauge_common.cuh); every phase of a trajectory --
// momentum refresh, Hamiltonians, forces, exponentials -- is one launch over
// all chains.  The whole trajectory is recorded once as a CUDA graph per
// (n_step, md_time, integrator, precision) and replayed, so a trajectory of
// the batch costs one graph launch plus one read of the per-chain Hamiltonian
// sums.  Every buffer is allocated when the batch is created: the captured
// graph never allocates.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <stdio.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/qlat_b200.h"
#include "kernels.h"

namespace qgb
{
void set_last_error(const std::string& msg);
void add_launches(int64_t n);
}

struct qgb_batch_s {
  int n = 0;
  long Vtot = 0;
  bool rect = false;
  std::vector<qgb::ChainInfo> chains;
  long* d_offs = nullptr;
  qgb::ChainInfo* d_chains = nullptr;
  uint32_t* d_rs = nullptr;
  uint32_t* h_rs = nullptr;
  int* d_flags = nullptr;
  int* h_flags = nullptr;
  double* gf = nullptr;   // chain states (FP64)
  double* gf0 = nullptr;  // trajectory copy (FP64)
  double* gm = nullptr;   // momenta (FP64)
  double* tmp = nullptr;  // FP64 link scratch
  float* gf32 = nullptr;
  float* gm32 = nullptr;
  float* tmp32 = nullptr;
  double* d_vals = nullptr;  // per-site values (2 Vtot)
  double* d_sums = nullptr;  // per-chain sums (8 n)
  double* h_sums = nullptr;  // pinned mirror
  int* d_ambiguous = nullptr;
  double* d_chain_tmp = nullptr;  // one chain's links in the reference image (download / upload)
  long max_chain_reals = 0;
  cudaStream_t stream = nullptr;
  std::map<std::tuple<int, double, int, int, int>, cudaGraphExec_t> graphs;
  int force_variant[2] = {0, 0};  // batched-force launch shape per precision [FP64, FP32] (qgb_batch_autotune)
  int kernels = 0;                 // kernels enqueued by the last enqueue_trajectory
  std::map<std::tuple<int, double, int, int, int>, int> graph_kernels;
};

namespace
{

int bfail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

#define QB_CUDA(expr)                                                                               \
  do {                                                                                              \
    cudaError_t e_ = (expr);                                                                        \
    if (e_ != cudaSuccess) return bfail(QGB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)
// a kernel launch of a trajectory: counted (qgb_launch_count)
#define QB_KERNEL(b, expr) \
  do {                     \
    ++(b)->kernels;        \
    QB_CUDA(expr);         \
  } while (0)
#define QB_RC(expr)              \
  do {                           \
    int r_ = (expr);             \
    if (r_ != QGB_OK) return r_; \
  } while (0)

qgb::ForceArgs bargs(const void* U, void* out, double dt, int unit)
{
  qgb::ForceArgs a;
  memset(&a, 0, sizeof(a));
  a.U = U;
  a.out = out;
  a.dt = dt;
  a.unitarize = unit;
  return a;
}

template <typename R>
int batch_force(qgb_batch_s* b, qgb::ForceMode mode, const qgb::ForceArgs& a)
{
  QB_KERNEL(b, qgb::launch_force_batch<R>(b->Vtot, b->n, b->d_offs, b->d_chains, b->rect, mode, a, b->stream,
                                     b->force_variant[sizeof(R) == 4 ? 1 : 0]));
  return QGB_OK;
}

template <typename R>
int batch_evolve(qgb_batch_s* b, void* U, const void* P, double eps, int unit)
{
  qgb::Geo g;
  g.d[0] = g.d[1] = g.d[2] = g.d[3] = 1;
  g.V = b->Vtot;
  QB_KERNEL(b, qgb::launch_evolve<R>(g, U, P, eps, unit, 0, b->stream));
  return QGB_OK;
}

// Molecular dynamics of all chains (same integrator as the single-lattice
// trajectory: hmc.pyx:169-188 / examples-py/hmc-pure-gauge-fgf.py:57-69).
template <typename R>
int batch_md(qgb_batch_s* b, void* gf, void* gm, void* tmp, int n_step, double md_time, int integrator, int unit_each,
             int reunit_every)
{
  const double dt = md_time / n_step;
  qgb::Geo g;
  g.d[0] = g.d[1] = g.d[2] = g.d[3] = 1;
  g.V = b->Vtot;
  if (integrator == QGB_INTEGRATOR_FORCE_GRADIENT) {
    const double lam = 0.5 * (1.0 - 1.0 / sqrt(3.0));
    const double theta = (2.0 - sqrt(3.0)) / 48.0;
    const double ttheta = theta * dt * dt * dt;
    const double fg_dt = 4.0 * ttheta / dt;
    QB_RC(batch_evolve<R>(b, gf, gm, lam * dt, unit_each));
    for (int i = 0; i < n_step; ++i) {
      const bool reunit = reunit_every > 0 && (i + 1) % reunit_every == 0 && i + 1 < n_step;
      for (int half = 0; half < 2; ++half) {
        QB_RC(batch_force<R>(b, qgb::FORCE_EVOLVE, bargs(gf, tmp, fg_dt, unit_each)));
        // gm += dt/2 F(tmp), then gf = exp(eps gm) gf in the same launch
        qgb::ForceArgs u = bargs(tmp, gm, 0.5 * dt, 1);
        u.ev = gf;
        u.ev_eps = half == 0 ? (1.0 - 2.0 * lam) * dt : (i < n_step - 1 ? 2.0 * lam : lam) * dt;
        u.ev_unit = (half == 1 && reunit) ? 2 : unit_each;
        QB_RC(batch_force<R>(b, qgb::FORCE_UPDATE_EVOLVE, u));
      }
    }
  } else if (integrator == QGB_INTEGRATOR_LEAPFROG && sizeof(R) == 4) {
    // FP32: each step one launch, the two half steps of the link update that
    // meet between force evaluations as one step of dt (the same P), written
    // into the other of two link buffers (gf, tmp) -- as the single-lattice
    // FP32 leapfrog
    QB_RC(batch_evolve<R>(b, gf, gm, 0.5 * dt, unit_each));
    void* cur = gf;
    void* nxt = tmp;
    for (int i = 0; i < n_step; ++i) {
      const bool reunit = reunit_every > 0 && (i + 1) % reunit_every == 0 && i + 1 < n_step;
      qgb::ForceArgs u = bargs(cur, gm, dt, 1);
      u.ev = nxt;
      u.ev_from_u = 1;
      u.ev_eps = i + 1 < n_step ? dt : 0.5 * dt;
      u.ev_unit = reunit ? 2 : unit_each;
      QB_RC(batch_force<R>(b, qgb::FORCE_UPDATE_EVOLVE, u));
      void* t = cur;
      cur = nxt;
      nxt = t;
    }
    if (cur != gf)
      QB_CUDA(cudaMemcpyAsync(gf, cur, (size_t)qgb::padded_sites(b->Vtot) * 72 * sizeof(R), cudaMemcpyDeviceToDevice,
                              b->stream));
  } else if (integrator == QGB_INTEGRATOR_LEAPFROG) {
    for (int i = 0; i < n_step; ++i) {
      QB_RC(batch_evolve<R>(b, gf, gm, 0.5 * dt, unit_each));
      QB_RC(batch_force<R>(b, qgb::FORCE_UPDATE, bargs(gf, gm, dt, 1)));
      QB_RC(batch_evolve<R>(b, gf, gm, 0.5 * dt, unit_each));
      if (reunit_every > 0 && (i + 1) % reunit_every == 0 && i + 1 < n_step)
        QB_KERNEL(b, (qgb::launch_unitarize<R, double>(g, 4, gf, b->stream)));
    }
  } else {
    return bfail(QGB_ERR_INVALID_ARG, "unknown integrator");
  }
  return QGB_OK;
}

// Per-chain Hamiltonian pieces of (gm, gf0) into d_sums[slot * n ...]: gm, plaq, rect.
int batch_hamiltonian(qgb_batch_s* b, int slot)
{
  QB_KERNEL(b, qgb::launch_site_values_batch<double>(b->Vtot, b->n, b->d_offs, b->d_chains, 0, 0, b->gm, b->d_vals,
                                                b->stream));
  QB_KERNEL(b, qgb::launch_segment_sum(b->n, b->d_offs, b->d_vals, b->d_sums + (long)slot * b->n, b->stream));
  QB_KERNEL(b, qgb::launch_site_values_batch<double>(b->Vtot, b->n, b->d_offs, b->d_chains, 1, b->rect ? 1 : 0, b->gf0,
                                                b->d_vals, b->stream));
  QB_KERNEL(b, qgb::launch_segment_sum(b->n, b->d_offs, b->d_vals, b->d_sums + (long)(slot + 1) * b->n, b->stream));
  if (b->rect)
    QB_KERNEL(b, qgb::launch_segment_sum(b->n, b->d_offs, b->d_vals + b->Vtot, b->d_sums + (long)(slot + 2) * b->n,
                                    b->stream));
  else
    QB_CUDA(cudaMemsetAsync(b->d_sums + (long)(slot + 2) * b->n, 0, b->n * sizeof(double), b->stream));
  return QGB_OK;
}

// One trajectory of every chain, enqueued on b->stream (recordable as a graph).
int enqueue_trajectory(qgb_batch_s* b, int n_step, double md_time, int integrator, int mixed, int reunit)
{
  b->kernels = 0;
  const size_t bytes64 = (size_t)qgb::padded_sites(b->Vtot) * 72 * sizeof(double);
  const long n = qgb::padded_sites(b->Vtot) * 72;
  qgb::Geo g;
  g.d[0] = g.d[1] = g.d[2] = g.d[3] = 1;
  g.V = b->Vtot;
  QB_CUDA(cudaMemcpyAsync(b->gf0, b->gf, bytes64, cudaMemcpyDeviceToDevice, b->stream));
  QB_KERNEL(b, qgb::launch_rand_momentum_batch<double>(b->Vtot, b->n, b->d_offs, b->d_rs, 1.0, b->gm, b->d_ambiguous,
                                                  b->stream));
  QB_RC(batch_hamiltonian(b, 0));
  if (mixed) {
    QB_KERNEL(b, (qgb::launch_convert<double, float>(n, b->gf0, b->gf32, b->stream)));
    QB_KERNEL(b, (qgb::launch_convert<double, float>(n, b->gm, b->gm32, b->stream)));
    QB_RC(batch_md<float>(b, b->gf32, b->gm32, b->tmp32, n_step, md_time, integrator, reunit > 0 ? 0 : 1, reunit));
    QB_KERNEL(b, (qgb::launch_convert<float, double>(n, b->gf32, b->gf0, b->stream)));
    QB_KERNEL(b, (qgb::launch_convert<float, double>(n, b->gm32, b->gm, b->stream)));
  } else {
    QB_RC(batch_md<double>(b, b->gf0, b->gm, b->tmp, n_step, md_time, integrator, 1, 0));
  }
  QB_KERNEL(b, (qgb::launch_unitarize<double, double>(g, 4, b->gf0, b->stream)));
  QB_RC(batch_hamiltonian(b, 3));
  QB_CUDA(cudaMemcpyAsync(b->h_sums, b->d_sums, 6 * b->n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  return QGB_OK;
}

double chain_action(const qgb::ChainInfo& c, double sp, double sr)
{
  return -c.beta / 3.0 * ((1.0 - 8.0 * c.c1) * sp + c.c1 * (c.c1 == 0.0 ? 0.0 : sr));
}

}  // namespace

extern "C" {

int qgb_batch_create(qgb_batch** out, int32_t n_chains, const int32_t* total_sites, const double* beta,
                     const double* c1)
{
  if (!out || !total_sites || !beta || !c1 || n_chains < 1)
    return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_create: bad argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bfail(QGB_ERR_NO_DEVICE, "no CUDA device");
  qgb_batch_s* b = new qgb_batch_s;
  b->n = n_chains;
  std::vector<long> offs(n_chains + 1, 0);
  long max_v = 0;
  for (int c = 0; c < n_chains; ++c) {
    qgb::ChainInfo ci;
    long V = 1;
    for (int i = 0; i < 4; ++i) {
      if (total_sites[4 * c + i] < 1 || total_sites[4 * c + i] > (1 << 20)) {
        delete b;
        return bfail(QGB_ERR_BAD_GEOMETRY, "qgb_batch_create: each lattice extent must be in [1, 2^20]");
      }
      ci.d[i] = total_sites[4 * c + i];
      V *= ci.d[i];
      // checked after every factor, so the product cannot wrap before it is refused
      if (V > (1L << 34) || offs[c] + V > (1L << 34)) {
        delete b;
        return bfail(QGB_ERR_BAD_GEOMETRY, "qgb_batch_create: batch too large");
      }
    }
    ci.V = V;
    ci.off = offs[c];
    ci.beta = beta[c];
    ci.c1 = c1[c];
    if (c1[c] != 0.0) b->rect = true;
    offs[c + 1] = offs[c] + V;
    if (V > max_v) max_v = V;
    b->chains.push_back(ci);
  }
  b->Vtot = offs[n_chains];
  b->max_chain_reals = max_v * 72;
  const size_t b64 = (size_t)qgb::padded_sites(b->Vtot) * 72 * sizeof(double), b32 = b64 / 2;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);  // padding sites stay zero
  };
  A((void**)&b->d_offs, (n_chains + 1) * sizeof(long));
  A((void**)&b->d_chains, n_chains * sizeof(qgb::ChainInfo));
  A((void**)&b->d_rs, (size_t)n_chains * 24 * sizeof(uint32_t));
  A((void**)&b->d_flags, n_chains * sizeof(int));
  A((void**)&b->gf, b64);
  A((void**)&b->gf0, b64);
  A((void**)&b->gm, b64);
  A((void**)&b->tmp, b64);
  A((void**)&b->gf32, b32);
  A((void**)&b->gm32, b32);
  A((void**)&b->tmp32, b32);
  A((void**)&b->d_vals, 2 * b->Vtot * sizeof(double));
  A((void**)&b->d_sums, 8 * (size_t)n_chains * sizeof(double));
  A((void**)&b->d_ambiguous, sizeof(int));
  A((void**)&b->d_chain_tmp, b->max_chain_reals * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_rs, (size_t)n_chains * 24 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_flags, n_chains * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_sums, 8 * (size_t)n_chains * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_offs, offs.data(), (n_chains + 1) * sizeof(long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_chains, b->chains.data(), n_chains * sizeof(qgb::ChainInfo), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_ambiguous, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->gf, 0, b64);
  if (e != cudaSuccess) {
    qgb_batch_destroy(b);
    cudaGetLastError();
    return bfail(QGB_ERR_ALLOC, std::string("qgb_batch_create: ") + cudaGetErrorString(e));
  }
  qgb::init_constants();
  *out = b;
  return QGB_OK;
}

int qgb_batch_destroy(qgb_batch* b)
{
  if (!b) return QGB_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  void* dev[] = {b->d_offs, b->d_chains, b->d_rs, b->d_flags, b->gf,     b->gf0,         b->gm,
                 b->tmp,    b->gf32,     b->gm32, b->tmp32,   b->d_vals, b->d_sums,      b->d_ambiguous,
                 b->d_chain_tmp};
  for (void* p : dev)
    if (p) cudaFree(p);
  if (b->h_rs) cudaFreeHost(b->h_rs);
  if (b->h_flags) cudaFreeHost(b->h_flags);
  if (b->h_sums) cudaFreeHost(b->h_sums);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return QGB_OK;
}

int qgb_batch_info(const qgb_batch* b, int32_t* n_chains, int64_t* total_site_count)
{
  if (!b) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_info: null batch");
  if (n_chains) *n_chains = b->n;
  if (total_site_count) *total_site_count = b->Vtot;
  return QGB_OK;
}

int qgb_batch_set_rand(qgb_batch* b, const uint32_t* rs, double sigma, int32_t n_step)
{
  if (!b || !rs) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_set_rand: null argument");
  memcpy(b->h_rs, rs, (size_t)b->n * 24 * sizeof(uint32_t));
  QB_CUDA(cudaMemcpyAsync(b->d_rs, b->h_rs, (size_t)b->n * 24 * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
  QB_CUDA(qgb::launch_hot_start_batch<double>(b->Vtot, b->n, b->d_offs, b->d_rs, sigma, n_step, b->gf,
                                              b->d_ambiguous, b->stream));
  QB_CUDA(cudaStreamSynchronize(b->stream));
  return QGB_OK;
}

int qgb_batch_trajectory(qgb_batch* b, const uint32_t* rs_momentum, int32_t n_step, double md_time,
                         int32_t integrator, int32_t mixed, int32_t reunit_interval, int32_t use_graph,
                         double* delta_h)
{
  if (!b || !rs_momentum || !delta_h || n_step < 1) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_trajectory: bad argument");
  memcpy(b->h_rs, rs_momentum, (size_t)b->n * 24 * sizeof(uint32_t));
  QB_CUDA(cudaMemcpyAsync(b->d_rs, b->h_rs, (size_t)b->n * 24 * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
  const int reunit = mixed ? reunit_interval : 0;
  if (use_graph) {
    auto key = std::make_tuple((int)n_step, md_time, (int)integrator, (int)(mixed != 0), reunit);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t graph = nullptr;
      QB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_trajectory(b, n_step, md_time, integrator, mixed, reunit);
      cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
      if (rc != QGB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (e != cudaSuccess) return bfail(QGB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
      b->graph_kernels[key] = b->kernels;
      cudaGraphExec_t exec = nullptr;
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return bfail(QGB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      it = b->graphs.emplace(key, exec).first;
    }
    QB_CUDA(cudaGraphLaunch(it->second, b->stream));
    qgb::add_launches(b->graph_kernels[key]);
  } else {
    QB_RC(enqueue_trajectory(b, n_step, md_time, integrator, mixed, reunit));
    qgb::add_launches(b->kernels);
  }
  QB_CUDA(cudaStreamSynchronize(b->stream));
  const int n = b->n;
  for (int c = 0; c < n; ++c) {
    const qgb::ChainInfo& ci = b->chains[c];
    const double h0 = b->h_sums[c] + chain_action(ci, b->h_sums[n + c], b->h_sums[2 * n + c]);
    const double h1 = b->h_sums[3 * n + c] + chain_action(ci, b->h_sums[4 * n + c], b->h_sums[5 * n + c]);
    delta_h[c] = h1 - h0;
  }
  return QGB_OK;
}

int qgb_batch_run_hmc(qgb_batch* b, const uint32_t* rs, int32_t traj, int32_t n_step, double md_time,
                      int32_t integrator, int32_t mixed, int32_t reunit_interval, int32_t always_accept,
                      double* delta_h, int32_t* flags)
{
  if (!b || !rs || !delta_h || !flags) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_run_hmc: null argument");
  // run_hmc_pure_gauge (hmc.pyx:190-216) for every chain: rs_c.split(traj), its
  // "set_rand_gauge_momentum" split for the momenta, its "metropolis_accept"
  // split for the Python-API Metropolis draw (hmc.pyx:139-155).
  const int n = b->n;
  std::vector<uint32_t> rs_t(24 * (size_t)n), rs_m(24 * (size_t)n);
  char tbuf[32];
  snprintf(tbuf, sizeof(tbuf), "%d", (int)traj);
  for (int c = 0; c < n; ++c) {
    if (!qgb::rng_host_split(&rs_t[24 * c], rs + 24 * c, tbuf) ||
        !qgb::rng_host_split(&rs_m[24 * c], &rs_t[24 * c], "set_rand_gauge_momentum"))
      return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_run_hmc: RngState split failed");
  }
  QB_RC(qgb_batch_trajectory(b, rs_m.data(), n_step, md_time, integrator, mixed, reunit_interval, 1, delta_h));
  for (int c = 0; c < n; ++c) {
    int flag = 0;
    if (delta_h[c] <= 0.0) {
      flag = 1;
    } else {
      uint32_t ra[24];
      qgb::rng_host_split(ra, &rs_t[24 * c], "metropolis_accept");
      const double u = qgb::rng_host_u_rand_gen(ra, 1.0, 0.0);
      flag = u <= exp(-delta_h[c]) ? 1 : 0;
    }
    flags[c] = flag;
    b->h_flags[c] = (flag || always_accept) ? 1 : 0;
  }
  QB_CUDA(cudaMemcpyAsync(b->d_flags, b->h_flags, b->n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  QB_CUDA(qgb::launch_accept_batch<double>(b->Vtot, b->n, b->d_offs, b->d_flags, b->gf, b->gf0, b->stream));
  qgb::add_launches(1);
  QB_CUDA(cudaStreamSynchronize(b->stream));
  return QGB_OK;
}

int qgb_batch_accept(qgb_batch* b, const int32_t* flags)
{
  if (!b || !flags) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_accept: null argument");
  for (int c = 0; c < b->n; ++c) b->h_flags[c] = flags[c] ? 1 : 0;
  QB_CUDA(cudaMemcpyAsync(b->d_flags, b->h_flags, b->n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  QB_CUDA(qgb::launch_accept_batch<double>(b->Vtot, b->n, b->d_offs, b->d_flags, b->gf, b->gf0, b->stream));
  qgb::add_launches(1);
  QB_CUDA(cudaStreamSynchronize(b->stream));
  return QGB_OK;
}

int qgb_batch_plaq(qgb_batch* b, double* plaq)
{
  if (!b || !plaq) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_plaq: null argument");
  QB_CUDA(qgb::launch_site_values_batch<double>(b->Vtot, b->n, b->d_offs, b->d_chains, 1, 0, b->gf, b->d_vals,
                                                b->stream));
  QB_CUDA(qgb::launch_segment_sum(b->n, b->d_offs, b->d_vals, b->d_sums + 6L * b->n, b->stream));
  QB_CUDA(cudaMemcpyAsync(b->h_sums + 6L * b->n, b->d_sums + 6L * b->n, b->n * sizeof(double), cudaMemcpyDeviceToHost,
                          b->stream));
  QB_CUDA(cudaStreamSynchronize(b->stream));
  for (int c = 0; c < b->n; ++c) plaq[c] = 1.0 + b->h_sums[6L * b->n + c] / (18.0 * (double)b->chains[c].V);
  return QGB_OK;
}

// Chain c's links <-> host buffer in the reference memory image.
int qgb_batch_download_chain(qgb_batch* b, int32_t chain, double* host)
{
  if (!b || !host || chain < 0 || chain >= b->n) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_download_chain: bad argument");
  const qgb::ChainInfo& ci = b->chains[chain];
  double* aos = b->d_chain_tmp;
  QB_CUDA(qgb::launch_store_to_aos<double>(b->Vtot, ci.off, ci.V, 4, 18, b->gf, aos, b->stream));
  QB_CUDA(cudaMemcpyAsync(host, aos, ci.V * 72 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  QB_CUDA(cudaStreamSynchronize(b->stream));
  return QGB_OK;
}

int qgb_batch_upload_chain(qgb_batch* b, int32_t chain, const double* host)
{
  if (!b || !host || chain < 0 || chain >= b->n) return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_upload_chain: bad argument");
  const qgb::ChainInfo& ci = b->chains[chain];
  double* aos = b->d_chain_tmp;
  QB_CUDA(cudaMemcpyAsync(aos, host, ci.V * 72 * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  QB_CUDA(qgb::launch_aos_to_store<double>(b->Vtot, ci.off, ci.V, 4, 18, aos, b->gf, b->stream));
  QB_CUDA(cudaStreamSynchronize(b->stream));
  return QGB_OK;
}


int qgb_batch_autotune(qgb_batch* b, int32_t precision, int32_t reps, int32_t* best, double* best_ms)
{
  if (!b || (precision != QGB_F64 && precision != QGB_F32) || reps < 1)
    return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_autotune: bad argument");
  const bool f32 = precision == QGB_F32;
  const long n = qgb::padded_sites(b->Vtot) * 72;
  // the chains' links in the precision of the force; momenta updated into the scratch buffer
  void* U = f32 ? (void*)b->gf32 : (void*)b->gf;
  void* P = f32 ? (void*)b->tmp32 : (void*)b->tmp;
  if (f32) QB_CUDA((qgb::launch_convert<double, float>(n, b->gf, b->gf32, b->stream)));
  QB_CUDA(cudaMemsetAsync(P, 0, (size_t)n * (f32 ? sizeof(float) : sizeof(double)), b->stream));
  cudaEvent_t e0, e1;
  QB_CUDA(cudaEventCreate(&e0));
  QB_CUDA(cudaEventCreate(&e1));
  int best_v = 0;
  float best_t = 1e30f;
  for (int v = 0; v < qgb::batch_force_variant_count(); ++v) {
    const qgb::ForceArgs a = bargs(U, P, 1e-3, 1);
    auto launch = [&]() {
      return f32 ? qgb::launch_force_batch<float>(b->Vtot, b->n, b->d_offs, b->d_chains, b->rect, qgb::FORCE_UPDATE,
                                                  a, b->stream, v)
                 : qgb::launch_force_batch<double>(b->Vtot, b->n, b->d_offs, b->d_chains, b->rect,
                                                   qgb::FORCE_UPDATE, a, b->stream, v);
    };
    QB_CUDA(launch());
    QB_CUDA(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < reps; ++r) QB_CUDA(launch());
    QB_CUDA(cudaEventRecord(e1, b->stream));
    QB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    QB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    ms /= reps;
    qgb::add_launches(reps + 1);
    if (ms < best_t) {
      best_t = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->force_variant[f32 ? 1 : 0] = best_v;
  // recorded trajectories hold the old launch shape: record them again
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  if (best) *best = best_v;
  if (best_ms) *best_ms = best_t;
  return QGB_OK;
}

int qgb_batch_set_force_variant(qgb_batch* b, int32_t precision, int32_t variant)
{
  if (!b || (precision != QGB_F64 && precision != QGB_F32) || variant < 0 ||
      variant >= qgb::batch_force_variant_count())
    return bfail(QGB_ERR_INVALID_ARG, "qgb_batch_set_force_variant: bad argument");
  b->force_variant[precision == QGB_F32 ? 1 : 0] = variant;
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  return QGB_OK;
}

}  // extern "C"
