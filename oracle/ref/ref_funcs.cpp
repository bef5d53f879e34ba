// ref_funcs.cpp -- times single hot-path functions of the reference Qlattice
// CPU implementation (OpenMP on the host cores), for the per-function CPU
// baseline.  Test infrastructure: it only calls the reference library's own
// functions.
//
//   ref_funcs hmc  X Y Z T beta c1 sigma reps
//       set_gm_force, gf_evolve, gm_hamilton_node, gf_hamilton_node,
//       set_rand_gauge_momentum, unitarize, gf_avg_plaq (hmc.h, qcd.h)
//   ref_funcs flow X Y Z T eps  c1 sigma reps
//       gf_wilson_flow_step (RK3), gf_energy_density (wilson-flow.h),
//       clf_topology_field + its sum, topology_charge_5 (qcd-topology.h)
//
// The field is the hot start GaugeField.set_rand(RngState(name).split("gf-init"),
// sigma, 1) of qcd-utils.cpp:71-92.  Prints one JSON line: seconds per call.
#include <qlat/qlat.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>

using namespace qlat;

static double now()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static double per_call(int reps, const std::function<void()>& f)
{
  f();  // warm-up: first-touch allocations and caches
  const double t0 = now();
  for (int i = 0; i < reps; ++i) f();
  return (now() - t0) / reps;
}

int main(int argc, char* argv[])
{
  if (argc < 10 || (strcmp(argv[1], "hmc") != 0 && strcmp(argv[1], "flow") != 0)) {
    fprintf(stderr, "usage: ref_funcs hmc|flow X Y Z T beta|eps c1 sigma reps\n");
    return 2;
  }
  const bool hmc = strcmp(argv[1], "hmc") == 0;
  const Coordinate total_site(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]));
  const double p = atof(argv[6]), c1 = atof(argv[7]), sigma = atof(argv[8]);
  const int reps = atoi(argv[9]);
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  Geometry geo;
  geo.init(total_site);
  const RngState rs(hmc ? "b200-c2-24x64-iwasaki" : "b200-c3-32x32-flow");
  GaugeField gf;
  gf.init(geo);
  set_g_rand_color_matrix_field(gf, rs.split("gf-init"), sigma, 1);
  std::string out = "{\"threads\": " + std::to_string(omp_get_max_threads()) +
                    ", \"sites\": " + std::to_string((long)geo.total_volume()) + ", \"reps\": " +
                    std::to_string(reps);
  auto add = [&](const char* name, double t) {
    char buf[128];
    snprintf(buf, sizeof(buf), ", \"%s\": %.6e", name, t);
    out += buf;
  };
  double sink = 0.0;
  if (hmc) {
    const GaugeAction ga(p, c1);
    GaugeMomentum gm, gf_force;
    gm.init(geo);
    gf_force.init(geo);
    set_rand_gauge_momentum(gm, 1.0, rs.split("1").split("set_rand_gauge_momentum"));
    add("set_gm_force", per_call(reps, [&]() { set_gm_force(gf_force, gf, ga); }));
    add("gf_evolve", per_call(reps, [&]() { gf_evolve(gf, gm, 1e-3); }));
    add("gm_hamilton_node", per_call(reps, [&]() { sink += gm_hamilton_node(gm); }));
    add("gf_hamilton_node", per_call(reps, [&]() { sink += gf_hamilton_node(gf, ga); }));
    add("set_rand_gauge_momentum",
        per_call(reps, [&]() { set_rand_gauge_momentum(gm, 1.0, rs.split("2").split("set_rand_gauge_momentum")); }));
    add("unitarize", per_call(reps, [&]() { unitarize(gf); }));
    add("gf_avg_plaq", per_call(reps, [&]() { sink += gf_avg_plaq(gf); }));
  } else {
    add("gf_wilson_flow_step", per_call(reps, [&]() { gf_wilson_flow_step(gf, p, c1); }));
    add("gf_energy_density", per_call(reps, [&]() { sink += gf_energy_density(gf); }));
    FieldM<RealD, 1> topf;
    add("clf_topology_sum", per_call(reps, [&]() {
          clf_topology_field(topf, gf);
          sink += field_glb_sum(topf)[0];
        }));
    add("topology_charge_5", per_call(reps, [&]() { sink += topology_charge_5(gf); }));
  }
  char buf[64];
  snprintf(buf, sizeof(buf), ", \"check\": %.6e}", sink);
  out += buf;
  printf("%s\n", out.c_str());
  end();
  return 0;
}
