// The reference's flowed-HMC C++ driver (examples-cpp/flowed-hmc/main.cpp) on
// the GPU library, through include/qlat_b200.hpp: the same flow
// (mk_flow_info_step(rs, 0.1, -0.01)), the same force-gradient integrator on
// the flowed action written out of set_gm_force_flowed / gf_evolve / field
// arithmetic, the same RNG splits, inverse-flow and reversibility checks,
// C++ Metropolis step (always accepted up to trajectory 20), and the same
// CHECK lines (examples-cpp/flowed-hmc/log).  The driver's diagnostic files
// (force magnitudes, Wilson-flow tables, saved configurations) are left out.
#include <cmath>
#include <cstdio>

#include "qlat_b200.hpp"

using namespace qlat_b200;

static void gm_evolve_fg(GaugeMomentum& gm, const GaugeField& gf_init, const GaugeAction& ga, const FlowInfo& fi,
                         double fg_dt, double dt)
{
  GaugeField gf;
  gf = gf_init;
  GaugeMomentum gm_force;
  set_gm_force_flowed(gm_force, gf, ga, fi);
  gf_evolve(gf, gm_force, fg_dt);
  set_gm_force_flowed(gm_force, gf, ga, fi);
  gm_force *= dt;
  gm += gm_force;
}

static double run_hmc_evolve_flowed(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, const FlowInfo& fi,
                                    int steps, double md_time)
{
  const double energy = gm_hamilton_node(gm) + gf_hamilton_flowed_node(gf, ga, fi);
  const double dt = md_time / steps;
  const double lambda = 0.5 * (1.0 - 1.0 / std::sqrt(3.0));
  const double theta = (2.0 - std::sqrt(3.0)) / 48.0;
  const double ttheta = theta * dt * dt * dt;
  gf_evolve(gf, gm, lambda * dt);
  for (int i = 0; i < steps; i++) {
    gm_evolve_fg(gm, gf, ga, fi, 4.0 * ttheta / dt, 0.5 * dt);
    gf_evolve(gf, gm, (1.0 - 2.0 * lambda) * dt);
    gm_evolve_fg(gm, gf, ga, fi, 4.0 * ttheta / dt, 0.5 * dt);
    gf_evolve(gf, gm, (i < steps - 1 ? 2.0 * lambda : lambda) * dt);
  }
  unitarize(gf);
  double delta_h = gm_hamilton_node(gm) + gf_hamilton_flowed_node(gf, ga, fi) - energy;
  glb_sum(delta_h);
  return delta_h;
}

static FlowInfo mk_flow_info(const RngState& rs)
{
  FlowInfo fi;
  vector_append(fi.v, mk_flow_info_step(rs, 0.1, -0.01).v);
  return fi;
}

static void run_hmc(GaugeField& gf, const GaugeAction& ga, int traj, const RngState& rs)
{
  const Geometry& geo = gf.geo();
  const bool is_reverse_test = traj < 3;
  const FlowInfo fi = mk_flow_info(rs.split("mk_flow_info"));
  std::printf("%s", show(fi).c_str());
  GaugeField gf0;
  gf_flow_inv(gf0, gf, fi);
  if (is_reverse_test) {
    GaugeField gf_r;
    gf_flow(gf_r, gf0, fi);
    gf_r -= gf;
    std::printf("gf_flow_inv gf_diff: %24.17E / %24.17E\n", qnorm(gf_r), qnorm(gf));
  }
  GaugeField gf0_init;
  if (is_reverse_test) gf0_init = gf0;
  GaugeMomentum gm;
  gm.init(geo);
  set_rand_gauge_momentum(gm, 1.0, rs.split("set_rand_gauge_momentum"));
  const int steps = 6;
  const double md_time = 1.0;
  const double delta_h = run_hmc_evolve_flowed(gm, gf0, ga, fi, steps, md_time);
  const double plaq_avg = gf_avg_plaq(gf0);
  std::printf("run_hmc: U_0: traj=%d ; plaq_avg=%24.17E ; plaq_sum=%24.17E .\n", traj, plaq_avg,
              volume(geo.total_site()) * 6 * (1.0 - plaq_avg));
  if (is_reverse_test) {
    GaugeMomentum gm_r;
    gm_r = gm;
    GaugeField gf0_r;
    gf0_r = gf0;
    const double delta_h_rev = run_hmc_evolve_flowed(gm_r, gf0_r, ga, fi, steps, -md_time);
    gf0_r -= gf0_init;
    std::printf("run_hmc_evolve_flowed reversed delta_diff: %24.17E / %24.17E\n", delta_h + delta_h_rev, delta_h);
    std::printf("run_hmc_evolve_flowed reversed gf_diff: %24.17E / %24.17E\n", qnorm(gf0_r), qnorm(gf0));
  }
  double accept_prob;
  const bool flag = metropolis_accept(accept_prob, delta_h, traj, rs.split("metropolis_accept"));
  if (flag || traj <= 20) {
    std::printf("run_hmc: update gf (traj=%d).\n", traj);
    gf_flow(gf, gf0, fi);
  }
}

int main()
{
  const Coordinate total_site(4, 4, 4, 8);
  const int traj_max = 3;
  Geometry geo;
  geo.init(total_site);
  const GaugeAction ga(2.31, -0.331);
  const RngState rs("test_hmc-" + show(total_site));
  GaugeField gf;
  gf.init(geo);
  set_unit(gf);
  set_g_rand_color_matrix_field(gf, RngState(), 1.0);
  for (int traj = 1; traj <= traj_max; ++traj) {
    run_hmc(gf, ga, traj, rs.split("hmc-" + std::to_string(traj)));
    const double plaq_avg = gf_avg_plaq(gf);
    const double plaq_sum = volume(total_site) * 6 * (1.0 - plaq_avg);
    std::printf("CHECK: test_hmc: traj=%d ; plaq_avg=%24.12E ; plaq_sum=%24.12E.\n", traj, plaq_avg, plaq_sum);
  }
  std::printf("CHECK: finished successfully.\n");
  return 0;
}
