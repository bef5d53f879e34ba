// Every function of include/qlat_b200.hpp beyond the HMC drivers, on a seeded
// 4^3 x 8 configuration; prints one "name value" line per result for the test
// to compare with the Python API on the same seeds.
#include <cmath>
#include <cstdio>

#include "qlat_b200.hpp"

using namespace qlat_b200;

static double sum(const FieldRealD& f)
{
  double s = 0.0;
  for (double v : f.download()) s += v;
  return s;
}

int main()
{
  Geometry geo;
  geo.init(Coordinate(4, 4, 4, 8));
  const RngState rs("api-surface");
  GaugeField gf;
  gf.init(geo);
  set_g_rand_color_matrix_field(gf, rs.split("gf"), 0.3, 2);
  // field-accelerated HMC
  FieldRealD mf(geo, 4), mfd(geo, 4);
  set_u_rand(mf, rs.split("mf"), 4.0, 1.0);
  set_u_rand(mfd, rs.split("mfd"), 4.0, 1.0);
  GaugeMomentum gm, gmd;
  set_rand_gauge_momentum(gm, mf, rs.split("gm"));
  set_rand_gauge_momentum(gmd, mfd, rs.split("gmd"));
  std::printf("gm_hamilton_fa %.17g\n", gm_hamilton_node(gm, mf));
  std::printf("project %.17g\n", project_gauge_transform(gm, gmd, mf, mfd));
  GaugeField g1;
  g1 = gf;
  gf_evolve(g1, gm, mf, 0.1);
  gf_evolve_dual(g1, gmd, mfd, 0.1);
  gf_evolve_dual(g1, gmd, 0.05);
  std::printf("plaq_fa %.17g\n", gf_avg_plaq(g1));
  GaugeMomentum F, Fd;
  set_gm_force(F, gf, GaugeAction(2.13, -0.331));
  set_gm_force_dual(Fd, gf, F);
  std::printf("qnorm_force_dual %.17g\n", qnorm(Fd));
  FieldRealD dot;
  dot_gauge_momentum(dot, gm, gmd);
  std::printf("dot %.17g\n", sum(dot));
  FieldRealD gr(geo, 3);
  set_g_rand(gr, rs.split("g"), 0.5, 2.0);
  std::printf("g_rand %.17g\n", sum(gr));
  // flow and topology fields
  FieldRealD fp, ed, edd, paf, spaf, q1, q5;
  gf_plaq_field(fp, gf);
  gf_energy_density_field(ed, gf);
  gf_energy_density_dir_field(edd, gf);
  clf_plaq_action_density_field(paf, gf);
  clf_spatial_plaq_action_density_field(spaf, gf);
  clf_topology_field(q1, gf);
  clf_topology_field_5(q5, gf);
  std::printf("plaq_field %.17g\nenergy %.17g\nenergy_dir %.17g\npaf %.17g\nspaf %.17g\n", sum(fp), sum(ed),
              sum(edd), sum(paf), sum(spaf));
  std::printf("topo_clf %.17g\ntopo_5 %.17g\ntopology_charge_5 %.17g\n", sum(q1), sum(q5), topology_charge_5(gf));
  GaugeMomentum z, zp;
  set_wilson_flow_z(z, gf, -0.331);
  set_plaq_flow_z(zp, gf, fp);
  std::printf("z %.17g\nzp %.17g\n", qnorm(z), qnorm(zp));
  GaugeField g2;
  g2 = gf;
  gf_wilson_flow_step_euler(g2, 0.05, -0.331);
  std::printf("plaq_euler %.17g\n", gf_avg_plaq(g2));
  // flowed HMC pieces
  const FlowInfo fi = mk_flow_info_step(rs.split("fi"), 0.1);
  GaugeField gfl, gfi;
  gf_flow(gfl, gf, fi);
  gf_flow_inv(gfi, gfl, fi);
  gfi -= gf;
  std::printf("flow_steps %d\nflow_round_trip %.17g\nflowed_action %.17g\n", (int)fi.v.size(), qnorm(gfi),
              gf_hamilton_flowed_node(gf, GaugeAction(2.31, -0.331), fi));
  // the mixed trajectory
  GaugeField g3;
  g3 = gf;
  GaugeMomentum m3;
  m3.init(geo);
  set_rand_gauge_momentum(m3, 1.0, rs.split("mom"));
  std::printf("delta_h_mixed %.17g\n", run_hmc_evolve_mixed(m3, g3, GaugeAction(2.13, -0.331), 6));
  std::printf("plaq_mixed %.17g\n", gf_avg_plaq(g3));
  return 0;
}
