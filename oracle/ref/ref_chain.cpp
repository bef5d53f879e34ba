// ref_chain.cpp -- runs an HMC chain with the reference Qlattice CPU library
// (OpenMP on the host cores): the chain of the Python driver
// run_hmc_pure_gauge (hmc.pyx:190-216), each trajectory's molecular dynamics
// through the reference library's own set_gm_force / gf_evolve /
// gm_hamilton_node / gf_hamilton_node / unitarize, and the Python form of
// metropolis_accept (hmc.pyx:139-155).  Test infrastructure: it only calls the
// reference library's own functions, to record golden chains and to time whole
// trajectories for the CPU baseline.
//
//   ref_chain X Y Z T beta c1 fg|leapfrog n_step md_time seed start n_traj n_always
//
// start: "unit" (set_unit) or "hot:<sigma>:<n_step>" (GaugeField.set_rand(
// RngState(seed).split("gf-init"), sigma, n_step), qcd-utils.cpp:71-92).
// The chain's RngState is RngState(seed).split("hmc"), split per trajectory
// exactly as run_hmc_pure_gauge does; trajectories 1..n_always are accepted
// whatever Metropolis says (is_always_accept).
//
// force-gradient: run_hmc_evolve_pure_gauge (hmc.pyx:169-188) with
// gm_evolve_fg_pure_gauge (hmc.pyx:157-167).  leapfrog: the composition of
// examples-py/hmc-pure-gauge-fgf.py:57-69 (gf_evolve dt/2, gm += dt F,
// gf_evolve dt/2), then unitarize, as the FG driver ends.
//
// Prints one JSON line per trajectory: traj, flag, delta_h, plaq (after the
// accept step), seconds of the trajectory (momenta, molecular dynamics, both
// Hamiltonians, Metropolis).
#include <qlat/qlat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

using namespace qlat;

static double now()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// hmc.pyx:157-167
static void gm_evolve_fg(GaugeMomentum& gm, const GaugeField& gf_init, const GaugeAction& ga, const RealD fg_dt,
                         const RealD dt)
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

static RealD hamiltonian(const GaugeMomentum& gm, const GaugeField& gf, const GaugeAction& ga)
{
  return gm_hamilton_node(gm) + gf_hamilton_node(gf, ga);
}

// hmc.pyx:169-188
static RealD run_hmc_evolve_fg(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, const int n_step,
                               const RealD md_time)
{
  const RealD energy = hamiltonian(gm, gf, ga);
  const RealD dt = md_time / n_step;
  const RealD lam = 0.5 * (1.0 - 1.0 / std::sqrt(3.0));
  const RealD theta = (2.0 - std::sqrt(3.0)) / 48.0;
  const RealD ttheta = theta * dt * dt * dt;
  gf_evolve(gf, gm, lam * dt);
  for (int i = 0; i < n_step; ++i) {
    gm_evolve_fg(gm, gf, ga, 4.0 * ttheta / dt, 0.5 * dt);
    gf_evolve(gf, gm, (1.0 - 2.0 * lam) * dt);
    gm_evolve_fg(gm, gf, ga, 4.0 * ttheta / dt, 0.5 * dt);
    if (i < n_step - 1) {
      gf_evolve(gf, gm, 2.0 * lam * dt);
    } else {
      gf_evolve(gf, gm, lam * dt);
    }
  }
  unitarize(gf);
  return hamiltonian(gm, gf, ga) - energy;
}

// examples-py/hmc-pure-gauge-fgf.py:57-69 (qq_evolve = gf_evolve, pp_evolve = gm += dt F)
static RealD run_hmc_evolve_leapfrog(GaugeMomentum& gm, GaugeField& gf, const GaugeAction& ga, const int n_step,
                                     const RealD md_time)
{
  const RealD energy = hamiltonian(gm, gf, ga);
  const RealD dt = md_time / n_step;
  GaugeMomentum gm_force;
  for (int i = 0; i < n_step; ++i) {
    gf_evolve(gf, gm, 0.5 * dt);
    set_gm_force(gm_force, gf, ga);
    gm_force *= dt;
    gm += gm_force;
    gf_evolve(gf, gm, 0.5 * dt);
  }
  unitarize(gf);
  return hamiltonian(gm, gf, ga) - energy;
}

int main(int argc, char* argv[])
{
  if (argc < 14) {
    fprintf(stderr,
            "usage: ref_chain X Y Z T beta c1 fg|leapfrog n_step md_time seed start n_traj n_always\n"
            "       start = unit | hot:<sigma>:<n_step>\n");
    return 2;
  }
  const Coordinate total_site(atoi(argv[1]), atoi(argv[2]), atoi(argv[3]), atoi(argv[4]));
  const GaugeAction ga(atof(argv[5]), atof(argv[6]));
  const bool fg = strcmp(argv[7], "fg") == 0;
  if (!fg && strcmp(argv[7], "leapfrog") != 0) {
    fprintf(stderr, "integrator must be fg or leapfrog\n");
    return 2;
  }
  const int n_step = atoi(argv[8]);
  const RealD md_time = atof(argv[9]);
  const std::string seed = argv[10];
  const std::string start = argv[11];
  const int n_traj = atoi(argv[12]), n_always = atoi(argv[13]);
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  Geometry geo;
  geo.init(total_site);
  const RngState rs0(seed);
  GaugeField gf;
  gf.init(geo);
  if (start == "unit") {
    set_unit(gf);
  } else {
    double sigma = 0.0;
    int hot_steps = 0;
    if (sscanf(start.c_str(), "hot:%lf:%d", &sigma, &hot_steps) != 2) {
      fprintf(stderr, "bad start %s\n", start.c_str());
      return 2;
    }
    set_g_rand_color_matrix_field(gf, rs0.split("gf-init"), sigma, hot_steps);
  }
  const RngState rs_chain = rs0.split("hmc");
  printf("{\"threads\": %d, \"sites\": %ld, \"plaq0\": %.17g}\n", omp_get_max_threads(), (long)geo.total_volume(),
         gf_avg_plaq(gf));
  fflush(stdout);
  for (int traj = 1; traj <= n_traj; ++traj) {
    const double t0 = now();
    // hmc.pyx:190-216
    const RngState rs = rs_chain.split(std::to_string(traj));
    GaugeField gf0;
    gf0 = gf;
    GaugeMomentum gm;
    gm.init(geo);
    set_rand_gauge_momentum(gm, 1.0, rs.split("set_rand_gauge_momentum"));
    const RealD delta_h = fg ? run_hmc_evolve_fg(gm, gf0, ga, n_step, md_time)
                             : run_hmc_evolve_leapfrog(gm, gf0, ga, n_step, md_time);
    // hmc.pyx:139-155, Python form: u = u_rand_gen(rs, 1.0, 0.0)
    bool flag = true;
    RealD accept_prob = 1.0;
    if (delta_h > 0.0) {
      accept_prob = std::exp(-delta_h);
      RngState rsm = rs.split("metropolis_accept");
      const RealD rand_num = u_rand_gen(rsm, 1.0, 0.0);
      flag = rand_num <= accept_prob;
    }
    if (flag || traj <= n_always) gf = gf0;
    const double t = now() - t0;
    printf("{\"traj\": %d, \"flag\": %d, \"delta_h\": %.17g, \"accept_prob\": %.17g, \"plaq\": %.17g, "
           "\"seconds\": %.6f}\n",
           traj, flag ? 1 : 0, delta_h, accept_prob, gf_avg_plaq(gf), t);
    fflush(stdout);
  }
  end();
  return 0;
}
