// The reference's C++ HMC driver (examples-cpp/hmc/main.cpp) on the GPU
// library, through include/qlat_b200.hpp: the same force-gradient integrator
// written out of gf_evolve / set_gm_force / field arithmetic, the same RNG
// splits, reversibility check and C++ Metropolis step, and the same CHECK
// lines (examples-cpp/hmc/log).
#include <cmath>
#include <cstdio>

#include "qlat_b200.hpp"

using namespace qlat_b200;

static void gm_evolve_fg_cpp(GaugeMomentum& gm, const GaugeField& gf_init, const GaugeAction& ga, double fg_dt,
                             double dt)
{
  GaugeField gf;
  gf = gf_init;
  GaugeMomentum gm_force;
  set_gm_force(gm_force, gf, ga);
  gf_evolve(gf, gm_force, fg_dt);
  set_gm_force(gm_force, gf, ga);
  gm_force *= dt;
  gm += gm_force;
}

static double run_hmc_evolve_cpp(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, int steps, double md_time)
{
  const double energy = gm_hamilton_node(gm) + gf_hamilton_node(gf, ga);
  const double dt = md_time / steps;
  const double lambda = 0.5 * (1.0 - 1.0 / std::sqrt(3.0));
  const double theta = (2.0 - std::sqrt(3.0)) / 48.0;
  const double ttheta = theta * dt * dt * dt;
  gf_evolve(gf, gm, lambda * dt);
  for (int i = 0; i < steps; i++) {
    gm_evolve_fg_cpp(gm, gf, ga, 4.0 * ttheta / dt, 0.5 * dt);
    gf_evolve(gf, gm, (1.0 - 2.0 * lambda) * dt);
    gm_evolve_fg_cpp(gm, gf, ga, 4.0 * ttheta / dt, 0.5 * dt);
    gf_evolve(gf, gm, (i < steps - 1 ? 2.0 * lambda : lambda) * dt);
  }
  unitarize(gf);
  double delta_h = gm_hamilton_node(gm) + gf_hamilton_node(gf, ga) - energy;
  glb_sum(delta_h);
  return delta_h;
}

static void run_hmc(GaugeField& gf, const GaugeAction& ga, int traj, const RngState& rs)
{
  const Geometry& geo = gf.geo();
  const bool is_reverse_test = traj < 3;
  GaugeField gf0;
  gf0 = gf;
  GaugeMomentum gm;
  gm.init(geo);
  set_rand_gauge_momentum(gm, 1.0, rs.split("set_rand_gauge_momentum"));
  const int steps = 6;
  const double md_time = 1.0;
  const double delta_h = run_hmc_evolve_cpp(gm, gf0, ga, steps, md_time);
  if (is_reverse_test) {
    GaugeMomentum gm_r;
    gm_r = gm;
    GaugeField gf0_r;
    gf0_r = gf0;
    const double delta_h_rev = run_hmc_evolve_cpp(gm_r, gf0_r, ga, steps, -md_time);
    gf0_r -= gf;
    printf("run_hmc_evolve reversed delta_diff: %24.17E / %24.17E\n", delta_h + delta_h_rev, delta_h);
    printf("run_hmc_evolve reversed gf_diff: %24.17E / %24.17E\n", qnorm(gf0_r), qnorm(gf0));
  }
  double accept_prob;
  const bool flag = metropolis_accept(accept_prob, delta_h, traj, rs.split("metropolis_accept"));
  if (flag or traj <= 20) gf = gf0;
}

static void test_hmc(const Coordinate& total_site, const GaugeAction& ga)
{
  Geometry geo;
  geo.init(total_site);
  const RngState rs = RngState("test_hmc-" + show(total_site));
  GaugeField gf;
  gf.init(geo);
  set_unit(gf);
  for (int traj = 1; traj <= 4; ++traj) {
    run_hmc(gf, ga, traj, rs.split("hmc-" + std::to_string(traj)));
    const double plaq_avg = gf_avg_plaq(gf);
    const double plaq_sum = volume(total_site) * 6 * (1.0 - plaq_avg);
    printf("CHECK: test_hmc: traj=%d ; plaq_avg=%24.12E ; plaq_sum=%24.12E.\n", traj, plaq_avg, plaq_sum);
  }
}

int main()
{
  const Coordinate total_site(4, 4, 4, 8);
  test_hmc(total_site, GaugeAction(2.13, -0.331));
  test_hmc(total_site, GaugeAction(5.5, 0.0));
  printf("CHECK: finished successfully.\n");
  return 0;
}
