/* qlat_b200.hpp -- header-only C++17 layer over the C ABI (qlat_b200.h) with
 * the shapes of Qlattice's C++ API for the pure-gauge path, so drivers written
 * against namespace qlat (examples-cpp/hmc/main.cpp) switch by changing the
 * namespace and the include:
 *
 *   Geometry geo; geo.init(Coordinate(4, 4, 4, 8));        // core.h / geometry.h
 *   GaugeField gf; gf.init(geo); set_unit(gf);            // qcd.h, qcd-utils.cpp
 *   GaugeMomentum gm; gm.init(geo);
 *   set_rand_gauge_momentum(gm, 1.0, rs.split("..."));    // hmc.h:52
 *   set_gm_force(gm_force, gf, ga); gf_evolve(gf, gm, dt); // hmc.h:58-72
 *   gm_force *= dt; gm += gm_force; gf0 = gf; gf0 -= gf;   // field.h operators
 *   metropolis_accept(accept_prob, delta_h, traj, rs);     // hmc.h:100
 *
 * Fields live in GPU memory (one qgb_field each, freed by the destructor);
 * `=` copies on the device.  Errors throw qlat_b200::Error, as the reference's
 * qerr throws.  Link with -lqlat_b200. */
#pragma once

#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "qlat_b200.h"

namespace qlat_b200
{

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc)
{
  if (rc != QGB_OK) throw Error(rc, qgb_last_error());
}

struct Coordinate {
  int32_t x[4] = {0, 0, 0, 0};
  Coordinate() {}
  Coordinate(int32_t a, int32_t b, int32_t c, int32_t d) : x{a, b, c, d} {}
  int32_t& operator[](int i) { return x[i]; }
  int32_t operator[](int i) const { return x[i]; }
};

inline long volume(const Coordinate& c) { return (long)c[0] * c[1] * c[2] * c[3]; }

/* show(Coordinate) of qlat-utils: "XxYxZxT" */
inline std::string show(const Coordinate& c)
{
  return std::to_string(c[0]) + "x" + std::to_string(c[1]) + "x" + std::to_string(c[2]) + "x" + std::to_string(c[3]);
}

struct Geometry {
  Coordinate ts;
  void init(const Coordinate& total_site) { ts = total_site; }
  Coordinate total_site() const { return ts; }
  long total_volume() const { return volume(ts); }
};

/* RngState (rng-state.h:12-99): the 24 x uint32 serialised state. */
struct RngState {
  uint32_t v[24];
  RngState() { check(qgb_rng_seed(v, nullptr)); }
  explicit RngState(const std::string& seed) { check(qgb_rng_seed(v, seed.c_str())); }
  RngState(const RngState& rs, const std::string& sindex) { check(qgb_rng_split(v, rs.v, sindex.c_str())); }
  RngState split(const std::string& sindex) const { return RngState(*this, sindex); }
};

inline uint64_t rand_gen(RngState& rs)
{
  uint64_t r;
  check(qgb_rng_rand_gen(rs.v, &r));
  return r;
}
inline double u_rand_gen(RngState& rs, double upper = 1.0, double lower = 0.0)
{
  double r;
  check(qgb_rng_u_rand_gen(rs.v, upper, lower, &r));
  return r;
}
inline double g_rand_gen(RngState& rs, double center = 0.0, double sigma = 1.0)
{
  double r;
  check(qgb_rng_g_rand_gen(rs.v, center, sigma, &r));
  return r;
}

/* GaugeAction (gauge-action.h:8-28) */
struct GaugeAction {
  double beta = 0.0, c1 = 0.0;
  GaugeAction() {}
  GaugeAction(double b, double c) : beta(b), c1(c) {}
};

/* A field of 3x3 complex matrices (KIND_COLOR_MATRIX) or reals in GPU memory. */
template <int KIND>
class FieldT
{
 public:
  FieldT() {}
  explicit FieldT(const Geometry& geo, int multiplicity = 4, int precision = QGB_F64)
  {
    init(geo, multiplicity, precision);
  }
  FieldT(const FieldT& o) { *this = o; }
  FieldT(FieldT&& o) noexcept : f_(o.f_), geo_(o.geo_), mult_(o.mult_), prec_(o.prec_) { o.f_ = nullptr; }
  ~FieldT() { qgb_field_destroy(f_); }

  void init(const Geometry& geo, int multiplicity = 4, int precision = QGB_F64)
  {
    if (f_ && geo.ts[0] == geo_.ts[0] && geo.ts[1] == geo_.ts[1] && geo.ts[2] == geo_.ts[2] &&
        geo.ts[3] == geo_.ts[3] && multiplicity == mult_ && precision == prec_)
      return;
    qgb_field_destroy(f_);
    f_ = nullptr;
    check(qgb_field_create(&f_, geo.ts.x, multiplicity, KIND, precision));
    geo_ = geo;
    mult_ = multiplicity;
    prec_ = precision;
  }
  bool initialized() const { return f_ != nullptr; }
  const Geometry& geo() const { return geo_; }
  int multiplicity() const { return mult_; }
  qgb_field* handle() { return need(); }
  const qgb_field* handle() const { return need(); }

  FieldT& operator=(const FieldT& o)  // field.h operator=: same geometry, device copy
  {
    if (this == &o) return *this;
    init(o.geo_, o.mult_, prec_ ? prec_ : o.prec_);
    check(qgb_field_copy(f_, o.need()));
    return *this;
  }
  FieldT& operator+=(const FieldT& o)
  {
    check(qgb_field_axpby(need(), 1.0, o.need(), 1.0));
    return *this;
  }
  FieldT& operator-=(const FieldT& o)
  {
    check(qgb_field_axpby(need(), -1.0, o.need(), 1.0));
    return *this;
  }
  FieldT& operator*=(double s)
  {
    check(qgb_field_axpby(need(), 0.0, nullptr, s));
    return *this;
  }
  void set_zero() { check(qgb_field_set_zero(need())); }
  /* The reference memory image ([site][m][...] doubles) to and from the host. */
  std::vector<double> download() const
  {
    std::vector<double> h((size_t)geo_.total_volume() * mult_ * (KIND == QGB_KIND_COLOR_MATRIX ? 18 : 1));
    check(qgb_field_download(need(), h.data()));
    return h;
  }
  void upload(const std::vector<double>& h) { check(qgb_field_upload(need(), h.data())); }

 private:
  qgb_field* need() const
  {
    if (!f_) throw Error(QGB_ERR_INVALID_ARG, "field is not initialised (call init(geo))");
    return f_;
  }
  qgb_field* f_ = nullptr;
  Geometry geo_;
  int mult_ = 0, prec_ = 0;
};

using FieldColorMatrix = FieldT<QGB_KIND_COLOR_MATRIX>;
using FieldRealD = FieldT<QGB_KIND_REAL>;

struct GaugeField : FieldColorMatrix {
  using FieldColorMatrix::FieldColorMatrix;
  using FieldColorMatrix::operator=;
  void init(const Geometry& geo, int precision = QGB_F64) { FieldColorMatrix::init(geo, 4, precision); }
};
struct GaugeMomentum : FieldColorMatrix {
  using FieldColorMatrix::FieldColorMatrix;
  using FieldColorMatrix::operator=;
  void init(const Geometry& geo, int precision = QGB_F64) { FieldColorMatrix::init(geo, 4, precision); }
};

template <int K>
inline double qnorm(const FieldT<K>& f)
{
  double r;
  check(qgb_field_qnorm(f.handle(), &r));
  return r;
}

/* ---- the pure-gauge path (hmc.h, qcd.h, qcd-utils.h, wilson-flow.h) ------- */

inline void set_unit(GaugeField& gf) { check(qgb_set_unit(gf.handle())); }
inline void set_g_rand_color_matrix_field(GaugeField& gf, const RngState& rs, double sigma, int n_step = 1)
{
  check(qgb_gf_set_rand(gf.handle(), rs.v, sigma, n_step));
}
inline void set_rand_gauge_momentum(GaugeMomentum& gm, double sigma, const RngState& rs)
{
  check(qgb_set_rand_gauge_momentum(gm.handle(), sigma, rs.v));
}
inline void set_gm_force(GaugeMomentum& gm_force, const GaugeField& gf, const GaugeAction& ga)
{
  if (!gm_force.initialized()) gm_force.init(gf.geo());
  check(qgb_set_gm_force(gm_force.handle(), gf.handle(), ga.beta, ga.c1));
}
inline void gf_evolve(GaugeField& gf, const GaugeMomentum& gm, double step_size)
{
  check(qgb_gf_evolve(gf.handle(), gm.handle(), step_size));
}
inline void gm_evolve_fg(GaugeMomentum& gm, const GaugeField& gf_init, const GaugeAction& ga, double fg_dt, double dt)
{
  check(qgb_gm_evolve_fg(gm.handle(), gf_init.handle(), ga.beta, ga.c1, fg_dt, dt));
}
inline double gm_hamilton_node(const GaugeMomentum& gm)
{
  double r;
  check(qgb_gm_hamilton_node(gm.handle(), &r));
  return r;
}
inline double gf_hamilton_node(const GaugeField& gf, const GaugeAction& ga)
{
  double r;
  check(qgb_gf_hamilton_node(gf.handle(), ga.beta, ga.c1, &r));
  return r;
}
inline void unitarize(GaugeField& gf) { check(qgb_unitarize(gf.handle())); }
inline double gf_avg_plaq(const GaugeField& gf)
{
  double r;
  check(qgb_gf_avg_plaq(gf.handle(), &r));
  return r;
}
/* One rank: the node sums are the global sums (glb_sum is the identity). */
inline void glb_sum(double&) {}
/* hmc.cpp:77-105 (the C++ draw, u_rand_gen(rs, 0.0, 1.0)) */
inline bool metropolis_accept(double& accept_prob, double delta_h, int traj, const RngState& rs)
{
  int32_t flag = 0;
  check(qgb_metropolis_accept(delta_h, traj, rs.v, &accept_prob, &flag));
  return flag != 0;
}
/* One whole trajectory on the GPU (the integrator of hmc.pyx:169-188 /
 * examples-cpp/hmc/main.cpp:run_hmc_evolve); returns delta_h. */
inline double run_hmc_evolve(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, int n_step,
                             double md_time = 1.0, int integrator = QGB_INTEGRATOR_FORCE_GRADIENT)
{
  double dh;
  check(qgb_run_hmc_evolve(gm.handle(), gf.handle(), ga.beta, ga.c1, n_step, md_time, integrator, &dh));
  return dh;
}
/* The same trajectory in the mixed form: FP32 molecular dynamics on copies of
 * the FP64 fields, FP64 re-unitarisation every reunit_interval steps, FP64
 * Hamiltonians; returns delta_h. */
inline double run_hmc_evolve_mixed(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, int n_step,
                                   double md_time = 1.0, int integrator = QGB_INTEGRATOR_FORCE_GRADIENT,
                                   int reunit_interval = 4)
{
  double dh;
  check(qgb_run_hmc_evolve_mixed(gm.handle(), gf.handle(), ga.beta, ga.c1, n_step, md_time, integrator,
                                 reunit_interval, &dh));
  return dh;
}
inline void gf_wilson_flow_step(GaugeField& gf, double epsilon, double c1 = 0.0)
{
  check(qgb_gf_wilson_flow_step(gf.handle(), epsilon, c1));
}
inline double gf_energy_density(const GaugeField& gf)
{
  double r;
  check(qgb_gf_energy_density(gf.handle(), &r));
  return r;
}
inline std::vector<double> gf_wilson_flow(GaugeField& gf, double flow_time, int steps, double c1 = 0.0)
{
  std::vector<double> e(steps);
  check(qgb_gf_wilson_flow(gf.handle(), flow_time, steps, c1, e.data()));
  return e;
}
inline double gf_topology_clf(const GaugeField& gf)
{
  double r;
  check(qgb_gf_topology_clf(gf.handle(), &r));
  return r;
}
inline double gf_topology(const GaugeField& gf)
{
  double r;
  check(qgb_gf_topology(gf.handle(), &r));
  return r;
}
/* qcd.h:146-250 (NERSC files) */
inline long save_gauge_field(const GaugeField& gf, const std::string& path)
{
  int64_t n = 0;
  check(qgb_save_gauge_field(gf.handle(), path.c_str(), nullptr, nullptr, nullptr, 0.0, 0, &n));
  return (long)n;
}
inline long load_gauge_field(GaugeField& gf, const std::string& path)
{
  Geometry geo;
  check(qgb_nersc_read_header(path.c_str(), geo.ts.x, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  gf.init(geo);
  int32_t checks = 0;
  int64_t n = 0;
  check(qgb_load_gauge_field(gf.handle(), path.c_str(), &checks, &n));
  return (long)n;
}

/* ---- field-accelerated HMC (hmc.h:20-80): per-link masses, dual momenta --- */

inline void set_rand_gauge_momentum(GaugeMomentum& gm, const FieldRealD& mf, const RngState& rs)
{
  if (!gm.initialized()) gm.init(mf.geo());
  check(qgb_set_rand_gauge_momentum_fa(gm.handle(), mf.handle(), rs.v));
}
inline double gm_hamilton_node(const GaugeMomentum& gm, const FieldRealD& mf)
{
  double r;
  check(qgb_gm_hamilton_node_fa(gm.handle(), mf.handle(), &r));
  return r;
}
inline void gf_evolve(GaugeField& gf, const GaugeMomentum& gm, const FieldRealD& mf, double step_size)
{
  check(qgb_gf_evolve_fa(gf.handle(), gm.handle(), mf.handle(), step_size));
}
inline void gf_evolve_dual(GaugeField& gf, const GaugeMomentum& gm_dual, double step_size)
{
  check(qgb_gf_evolve_dual(gf.handle(), gm_dual.handle(), step_size));
}
inline void gf_evolve_dual(GaugeField& gf, const GaugeMomentum& gm_dual, const FieldRealD& mf_dual, double step_size)
{
  check(qgb_gf_evolve_fa_dual(gf.handle(), gm_dual.handle(), mf_dual.handle(), step_size));
}
inline void set_gm_force_dual(GaugeMomentum& gm_force_dual, const GaugeField& gf, const GaugeMomentum& gm_force)
{
  if (!gm_force_dual.initialized()) gm_force_dual.init(gf.geo());
  check(qgb_set_gm_force_dual(gm_force_dual.handle(), gf.handle(), gm_force.handle()));
}
inline double project_gauge_transform(GaugeMomentum& gm, GaugeMomentum& gm_dual, const FieldRealD& mf,
                                      const FieldRealD& mf_dual)
{
  double r;
  check(qgb_project_gauge_transform(gm.handle(), gm_dual.handle(), mf.handle(), mf_dual.handle(), &r));
  return r;
}
inline void set_gauge_transform_momentum(GaugeMomentum& gm, GaugeMomentum& gm_dual, const FieldColorMatrix& gtm)
{
  if (!gm.initialized()) gm.init(gtm.geo());
  if (!gm_dual.initialized()) gm_dual.init(gtm.geo());
  check(qgb_set_gauge_transform_momentum(gm.handle(), gm_dual.handle(), gtm.handle()));
}
inline void dot_gauge_momentum(FieldRealD& f, const GaugeMomentum& gm1, const GaugeMomentum& gm2)
{
  f.init(gm1.geo(), 4);
  check(qgb_dot_gauge_momentum(f.handle(), gm1.handle(), gm2.handle()));
}
/* set_u_rand / set_g_rand of a real field (core.h:1585-1636) */
inline void set_u_rand(FieldRealD& f, const RngState& rs, double upper = 1.0, double lower = -1.0)
{
  check(qgb_field_set_u_rand(f.handle(), rs.v, upper, lower));
}
inline void set_g_rand(FieldRealD& f, const RngState& rs, double center = 0.0, double sigma = 1.0)
{
  check(qgb_field_set_g_rand(f.handle(), rs.v, center, sigma));
}

/* ---- fields of the flow and the topology (qcd.h, wilson-flow.h, qcd-topology.h) */

inline void gf_plaq_field(FieldRealD& f_plaq, const GaugeField& gf)
{
  f_plaq.init(gf.geo(), 6);
  check(qgb_gf_plaq_field(f_plaq.handle(), gf.handle()));
}
inline void gf_energy_density_field(FieldRealD& fd, const GaugeField& gf)
{
  fd.init(gf.geo(), 1);
  check(qgb_gf_energy_density_field(fd.handle(), gf.handle()));
}
inline void gf_energy_density_dir_field(FieldRealD& fd, const GaugeField& gf)
{
  fd.init(gf.geo(), 6);
  check(qgb_gf_energy_density_dir_field(fd.handle(), gf.handle()));
}
inline void set_wilson_flow_z(GaugeMomentum& z, const GaugeField& gf, double c1)
{
  if (!z.initialized()) z.init(gf.geo());
  check(qgb_set_wilson_flow_z(z.handle(), gf.handle(), c1));
}
inline void set_plaq_flow_z(GaugeMomentum& z, const GaugeField& gf, const FieldRealD& plaq_factor)
{
  if (!z.initialized()) z.init(gf.geo());
  check(qgb_set_plaq_flow_z(z.handle(), gf.handle(), plaq_factor.handle()));
}
inline void gf_wilson_flow_step_euler(GaugeField& gf, double epsilon, double c1 = 0.0)
{
  check(qgb_gf_wilson_flow_step_euler(gf.handle(), epsilon, c1));
}
inline void clf_plaq_action_density_field(FieldRealD& paf, const GaugeField& gf)
{
  paf.init(gf.geo(), 1);
  check(qgb_gf_plaq_action_density_field(paf.handle(), gf.handle(), 0));
}
inline void clf_spatial_plaq_action_density_field(FieldRealD& paf, const GaugeField& gf)
{
  paf.init(gf.geo(), 1);
  check(qgb_gf_plaq_action_density_field(paf.handle(), gf.handle(), 1));
}
inline void clf_topology_field(FieldRealD& topf, const GaugeField& gf)
{
  topf.init(gf.geo(), 1);
  check(qgb_clf_topology_field(topf.handle(), gf.handle()));
}
inline void clf_topology_field_5(FieldRealD& topf, const GaugeField& gf)
{
  topf.init(gf.geo(), 1);
  check(qgb_clf_topology_field_5(topf.handle(), gf.handle()));
}
inline double topology_charge_5(const GaugeField& gf)
{
  double r;
  check(qgb_topology_charge_5(gf.handle(), &r));
  return r;
}

/* ---- flowed HMC with masked invertible flows (flowed-hmc.h) ----------------- */

/* FlowStepInfo (flowed-hmc.h:26-41) */
struct FlowStepInfo {
  int mask = 0, mu = 0;
  double epsilon = 0.0;
  int flow_size = 1;
};
/* FlowInfo (flowed-hmc.h:43-46) */
struct FlowInfo {
  std::vector<FlowStepInfo> v;
};

inline std::vector<qgb_flow_step> flow_steps(const FlowInfo& fi)
{
  std::vector<qgb_flow_step> s(fi.v.size());
  for (size_t i = 0; i < s.size(); ++i) {
    s[i].mask = fi.v[i].mask;
    s[i].mu = fi.v[i].mu;
    s[i].epsilon = fi.v[i].epsilon;
    s[i].flow_size = fi.v[i].flow_size;
  }
  return s;
}

/* show(FlowInfo) (flowed-hmc.h:48-62): one line per step */
inline std::string show(const FlowInfo& fi)
{
  std::string out;
  char buf[128];
  for (size_t i = 0; i < fi.v.size(); ++i) {
    const FlowStepInfo& f = fi.v[i];
    std::snprintf(buf, sizeof(buf), "flow step %d: mask=%d mu=%d epsilon=%.17g flow_size=%d\n", (int)i, f.mask,
                  f.mu, f.epsilon, f.flow_size);
    out += buf;
  }
  return out;
}

/* mk_flow_info_step(rs, epsilon) and (rs, epsilon, epsilon2) (flowed-hmc.cpp:21-69) */
inline FlowInfo mk_flow_info_step(const RngState& rs, double epsilon)
{
  qgb_flow_step s[16];
  int32_t n = 0;
  check(qgb_flow_info_step(rs.v, epsilon, 0.0, 0, s, &n));
  FlowInfo fi;
  for (int i = 0; i < n; ++i) fi.v.push_back(FlowStepInfo{s[i].mask, s[i].mu, s[i].epsilon, s[i].flow_size});
  return fi;
}
inline FlowInfo mk_flow_info_step(const RngState& rs, double epsilon, double epsilon2)
{
  qgb_flow_step s[16];
  int32_t n = 0;
  check(qgb_flow_info_step(rs.v, epsilon, epsilon2, 1, s, &n));
  FlowInfo fi;
  for (int i = 0; i < n; ++i) fi.v.push_back(FlowStepInfo{s[i].mask, s[i].mu, s[i].epsilon, s[i].flow_size});
  return fi;
}

/* vector_append (qlat-utils vector.h) */
template <class T>
inline void vector_append(std::vector<T>& v, const std::vector<T>& w)
{
  v.insert(v.end(), w.begin(), w.end());
}

/* gf_flow / gf_flow_inv (flowed-hmc.cpp:540-594) */
inline void gf_flow(GaugeField& gf, const GaugeField& gf0, const FlowInfo& fi)
{
  if (!gf.initialized()) gf.init(gf0.geo());
  const std::vector<qgb_flow_step> s = flow_steps(fi);
  check(qgb_gf_flow(gf.handle(), gf0.handle(), s.data(), (int32_t)s.size()));
}
inline void gf_flow_inv(GaugeField& gf, const GaugeField& gf1, const FlowInfo& fi)
{
  if (!gf.initialized()) gf.init(gf1.geo());
  const std::vector<qgb_flow_step> s = flow_steps(fi);
  check(qgb_gf_flow_inv(gf.handle(), gf1.handle(), s.data(), (int32_t)s.size()));
}
/* gf_hamilton_flowed_node (flowed-hmc.cpp:1301-1321): the action of the flowed
 * field minus the log-determinant of the flow */
inline double gf_hamilton_flowed_node(const GaugeField& gf0, const GaugeAction& ga, const FlowInfo& fi)
{
  const std::vector<qgb_flow_step> s = flow_steps(fi);
  double act = 0.0, ln_det = 0.0;
  check(qgb_gf_hamilton_flowed_node(gf0.handle(), ga.beta, ga.c1, s.data(), (int32_t)s.size(), &act, &ln_det));
  return act - ln_det;
}
/* set_gm_force_flowed (flowed-hmc.cpp:1500-1509) */
inline void set_gm_force_flowed(GaugeMomentum& gm_force, const GaugeField& gf0, const GaugeAction& ga,
                                const FlowInfo& fi)
{
  if (!gm_force.initialized()) gm_force.init(gf0.geo());
  const std::vector<qgb_flow_step> s = flow_steps(fi);
  check(qgb_set_gm_force_flowed(gm_force.handle(), gf0.handle(), ga.beta, ga.c1, s.data(), (int32_t)s.size(), 1));
}

}  // namespace qlat_b200
