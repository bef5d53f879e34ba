// ref_bench.cpp -- times the reference Qlattice CPU implementation of the
// pure-gauge hot path (OpenMP on the host cores), for the CPU baseline.
// Test infrastructure: it only calls the reference library's own functions.
//
//   ref_bench X Y Z T beta c1 sigma n_samples
//
// Builds a hot start with GaugeField.set_rand's C++ (qcd-utils.cpp:71-92),
// then times (a) the per-trajectory ends: set_rand_gauge_momentum,
// 2 x (gm_hamilton_node + gf_hamilton_node) and unitarize; and (b) n_samples
// samples of one set_gm_force + one gf_evolve, the pair a force-gradient
// trajectory repeats 32 times at n_step = 8 (hmc.pyx:169-188).  Prints one
// JSON line.
#include <qlat/qlat.h>

#include <chrono>
#include <cstdio>

using namespace qlat;

static double now()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char* argv[])
{
  if (argc < 9) {
    fprintf(stderr, "usage: ref_bench X Y Z T beta c1 sigma n_samples\n");
    return 2;
  }
  const Coordinate total_site(atoi(argv[1]), atoi(argv[2]), atoi(argv[3]), atoi(argv[4]));
  const GaugeAction ga(atof(argv[5]), atof(argv[6]));
  const double sigma = atof(argv[7]);
  const int n = atoi(argv[8]);
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  Geometry geo;
  geo.init(total_site);
  const RngState rs("b200-c2-24x64-iwasaki");
  GaugeField gf;
  gf.init(geo);
  double t0 = now();
  set_g_rand_color_matrix_field(gf, rs.split("gf-init"), sigma, 1);
  const double t_hot = now() - t0;
  GaugeMomentum gm, gf_force;
  gm.init(geo);
  gf_force.init(geo);
  t0 = now();
  set_rand_gauge_momentum(gm, 1.0, rs.split("1").split("set_rand_gauge_momentum"));
  double h = gm_hamilton_node(gm) + gf_hamilton_node(gf, ga);
  h += gm_hamilton_node(gm) + gf_hamilton_node(gf, ga);
  unitarize(gf);
  const double t_ends = now() - t0;
  double t_pair = 0;
  for (int i = 0; i < n; ++i) {
    t0 = now();
    set_gm_force(gf_force, gf, ga);
    gf_evolve(gf, gf_force, 1e-3);
    t_pair += now() - t0;
  }
  const double per_pair = t_pair / n;
  printf("{\"threads\": %d, \"sites\": %ld, \"t_hot_start\": %.6f, \"t_ends\": %.6f, \"t_force_evolve\": %.6f, "
         "\"samples\": %d, \"check\": %.6e}\n",
         omp_get_max_threads(), (long)geo.total_volume(), t_hot, t_ends, per_pair, n, h);
  end();
  return 0;
}
