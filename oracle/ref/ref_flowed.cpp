// ref_flowed.cpp -- the reference library's flowed HMC (flowed-hmc.cpp) on a
// seeded configuration, stage by stage, for pinning the GPU library's
// implementation.  Test infrastructure: it only calls the reference's
// functions.
//
//   ref_flowed DIR X Y Z T sigma fi_seed eps eps2 beta c1
//     gf0 = set_g_rand_color_matrix_field(RngState("flowed-test").split("gf-init"), sigma, 1)
//     fi  = mk_flow_info_step(RngState(fi_seed), eps, eps2)
//   writes into DIR (reference memory image, native doubles):
//     gf0.bin, flow.bin (gf_flow), flow_inv.bin (gf_flow_inv),
//     force.bin (set_gm_force_flowed), force_no_det.bin
//     (set_gm_force_flowed_no_det of set_gm_force of the flowed field)
//   and prints one JSON line: the flow steps, flowed action and ln det.
#include <qlat/flowed-hmc.h>
#include <qlat/qlat.h>

#include <cstdio>

using namespace qlat;

static void dump(const std::string& path, const Field<ColorMatrix>& f)
{
  FILE* fp = fopen(path.c_str(), "wb");
  const Geometry& geo = f.geo();
  for (Long i = 0; i < geo.local_volume(); ++i) {
    const Vector<ColorMatrix> v = f.get_elems_const(i);
    fwrite(v.data(), sizeof(ColorMatrix), v.size(), fp);
  }
  fclose(fp);
}

int main(int argc, char* argv[])
{
  if (argc < 12) {
    fprintf(stderr, "usage: ref_flowed DIR X Y Z T sigma fi_seed eps eps2 beta c1\n");
    return 2;
  }
  const std::string dir = argv[1];
  const Coordinate total_site(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]));
  const double sigma = atof(argv[6]);
  const FlowInfo fi = mk_flow_info_step(RngState(argv[7]), atof(argv[8]), atof(argv[9]));
  const GaugeAction ga(atof(argv[10]), atof(argv[11]));
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  Geometry geo;
  geo.init(total_site);
  GaugeField gf0;
  gf0.init(geo);
  set_g_rand_color_matrix_field(gf0, RngState("flowed-test").split("gf-init"), sigma, 1);
  dump(dir + "/gf0.bin", gf0);
  GaugeField gf1, gf2;
  gf_flow(gf1, gf0, fi);
  dump(dir + "/flow.bin", gf1);
  gf_flow_inv(gf2, gf0, fi);
  dump(dir + "/flow_inv.bin", gf2);
  GaugeField gf3;
  const double ln_det = gf_flow_and_ln_det_node(gf3, gf0, fi);  // one rank: node = global
  const double flowed_action = gf_hamilton_node(gf3, ga);
  GaugeMomentum gm_force;
  set_gm_force_flowed(gm_force, gf0, ga, fi);
  dump(dir + "/force.bin", gm_force);
  GaugeMomentum f_phys, f_no_det;
  set_gm_force(f_phys, gf1, ga);
  set_gm_force_flowed_no_det(f_no_det, f_phys, gf0, fi);
  dump(dir + "/force_no_det.bin", f_no_det);
  printf("{\"steps\": [");
  for (size_t i = 0; i < fi.v.size(); ++i)
    printf("%s[%d, %d, %.17g, %d]", i ? ", " : "", fi.v[i].mask, fi.v[i].mu, fi.v[i].epsilon, fi.v[i].flow_size);
  printf("], \"flowed_action\": %.17g, \"ln_det\": %.17g}\n", flowed_action, ln_det);
  end();
  return 0;
}
