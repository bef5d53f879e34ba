// ref_fa.cpp -- the reference library's field-accelerated HMC primitives
// (hmc.cpp:121-201, 330-396, 492-645; set_u_rand / set_g_rand of core.h) on
// seeded inputs, for pinning the oracle and the GPU library.  Test
// infrastructure: it only calls the reference's functions.
//
//   ref_fa DIR X Y Z T seed dt beta c1
//     rs  = RngState(seed)
//     gf0 = set_g_rand_color_matrix_field(rs.split("gf"), 0.3, 2)
//     mf, mf_dual = set_u_rand(rs.split("mf"|"mfd"), 4.0, 1.0), then +inf on
//                   every link with (site + 2 mu) % 7 == 3 (mf) or == 5 (mf_dual)
//     gm, gm_dual = set_rand_gauge_momentum(mf|mf_dual, rs.split("gm"|"gmd"))
//   writes into DIR (reference memory image, native doubles):
//     gf0, mf, mfd, gm, gmd, gm_proj, gmd_proj (project_gauge_transform),
//     evolve_fa (gf_evolve with mf), evolve_fa_dual (gf_evolve_dual with
//     mf_dual), evolve_dual (gf_evolve_dual without masses), force,
//     force_dual (set_gm_force_dual of set_gm_force), gtm
//     (set_g_rand_anti_hermitian_matrix_field(rs.split("gtm"), 1.0), one per
//     site), gt_gm, gt_gmd (set_gauge_transform_momentum), dot
//     (dot_gauge_momentum(gm, gmd)), grand (set_g_rand(rs.split("g"), 0.5,
//     2.0) of a real field of multiplicity 3)
//   and prints one JSON line with gm_hamilton_node(gm, mf),
//   gm_hamilton_node(gm_dual, mf_dual) and the projection's change_qnorm.
#include <qlat/qlat.h>

#include <cstdio>
#include <limits>

using namespace qlat;

template <class M>
static void dump(const std::string& path, const Field<M>& f)
{
  FILE* fp = fopen(path.c_str(), "wb");
  const Geometry& geo = f.geo();
  for (Long i = 0; i < geo.local_volume(); ++i) {
    const Vector<M> v = f.get_elems_const(i);
    fwrite(v.data(), sizeof(M), v.size(), fp);
  }
  fclose(fp);
}

static void set_inf(Field<RealD>& mf, const Int r)
{
  const RealD inf = std::numeric_limits<RealD>::infinity();
  const Geometry& geo = mf.geo();
  for (Long i = 0; i < geo.local_volume(); ++i) {
    Vector<RealD> v = mf.get_elems(i);
    for (Int mu = 0; mu < 4; ++mu)
      if ((i + 2 * mu) % 7 == r) v[mu] = inf;
  }
}

int main(int argc, char* argv[])
{
  if (argc < 10) {
    fprintf(stderr, "usage: ref_fa DIR X Y Z T seed dt beta c1\n");
    return 2;
  }
  const std::string dir = argv[1];
  const Coordinate total_site(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]));
  const RngState rs(argv[6]);
  const RealD dt = atof(argv[7]);
  const GaugeAction ga(atof(argv[8]), atof(argv[9]));
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  Geometry geo;
  geo.init(total_site);
  GaugeField gf0;
  gf0.init(geo);
  set_g_rand_color_matrix_field(gf0, rs.split("gf"), 0.3, 2);
  dump(dir + "/gf0.bin", gf0);
  Field<RealD> mf, mfd;
  mf.init(geo, 4);
  mfd.init(geo, 4);
  set_u_rand(mf, rs.split("mf"), 4.0, 1.0);
  set_u_rand(mfd, rs.split("mfd"), 4.0, 1.0);
  set_inf(mf, 3);
  set_inf(mfd, 5);
  dump(dir + "/mf.bin", mf);
  dump(dir + "/mfd.bin", mfd);
  GaugeMomentum gm, gmd;
  gm.init(geo);
  gmd.init(geo);
  set_rand_gauge_momentum(gm, mf, rs.split("gm"));
  set_rand_gauge_momentum(gmd, mfd, rs.split("gmd"));
  dump(dir + "/gm.bin", gm);
  dump(dir + "/gmd.bin", gmd);
  const RealD h1 = gm_hamilton_node(gm, mf);
  const RealD h2 = gm_hamilton_node(gmd, mfd);
  GaugeMomentum gmp, gmdp;
  gmp = gm;
  gmdp = gmd;
  const RealD change = project_gauge_transform(gmp, gmdp, mf, mfd);
  dump(dir + "/gm_proj.bin", gmp);
  dump(dir + "/gmd_proj.bin", gmdp);
  GaugeField gf;
  gf = gf0;
  gf_evolve(gf, gm, mf, dt);
  dump(dir + "/evolve_fa.bin", gf);
  gf = gf0;
  gf_evolve_dual(gf, gmd, mfd, dt);
  dump(dir + "/evolve_fa_dual.bin", gf);
  gf = gf0;
  gf_evolve_dual(gf, gmd, dt);
  dump(dir + "/evolve_dual.bin", gf);
  GaugeMomentum force, force_dual;
  set_gm_force(force, gf0, ga);
  set_gm_force_dual(force_dual, gf0, force);
  dump(dir + "/force.bin", force);
  dump(dir + "/force_dual.bin", force_dual);
  FieldM<ColorMatrix, 1> gtm;
  gtm.init(geo);
  set_g_rand_anti_hermitian_matrix_field(gtm, rs.split("gtm"), 1.0);
  dump(dir + "/gtm.bin", gtm);
  GaugeMomentum gt_gm, gt_gmd;
  set_gauge_transform_momentum(gt_gm, gt_gmd, gtm);
  dump(dir + "/gt_gm.bin", gt_gm);
  dump(dir + "/gt_gmd.bin", gt_gmd);
  Field<RealD> dot;
  dot_gauge_momentum(dot, gm, gmd);
  dump(dir + "/dot.bin", dot);
  Field<RealD> grand;
  grand.init(geo, 3);
  set_g_rand(grand, rs.split("g"), 0.5, 2.0);
  dump(dir + "/grand.bin", grand);
  printf("{\"h_gm\": %.17g, \"h_gmd\": %.17g, \"change_qnorm\": %.17g}\n", h1, h2, change);
  fflush(stdout);
  end();
  return 0;
}
