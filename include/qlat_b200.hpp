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

}  // namespace qlat_b200
