// ref_nersc.cpp -- the reference library's own NERSC gauge-file writer and
// reader (save_gauge_field / load_gauge_field, qcd.h:146-250), driven from
// the command line so the tests can pin the GPU library's files against them.
// Test infrastructure: it only calls the reference library's functions.
//
//   ref_nersc save PATH X Y Z T sigma n_step seed
//       hot start set_g_rand_color_matrix_field(RngState(seed).split("gf-init"),
//       sigma, n_step) saved with the default GaugeFieldInfo; prints one JSON
//       line with the plaquette and link trace
//   ref_nersc load PATH OUT
//       load_gauge_field, then writes the links to OUT in the reference memory
//       image (native doubles, [site][mu][3][3] complex) and prints one JSON line
#include <qlat/qlat.h>

#include <cstdio>

using namespace qlat;

int main(int argc, char* argv[])
{
  if (argc < 4) {
    fprintf(stderr, "usage: ref_nersc save PATH X Y Z T sigma n_step seed | ref_nersc load PATH OUT\n");
    return 2;
  }
  const std::string mode = argv[1], path = argv[2];
  int argc0 = 1;
  char** argv0 = argv;
  begin(&argc0, &argv0);
  if (mode == "save" && argc >= 10) {
    const Coordinate total_site(atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]));
    Geometry geo;
    geo.init(total_site);
    GaugeField gf;
    gf.init(geo);
    set_g_rand_color_matrix_field(gf, RngState(argv[9]).split("gf-init"), atof(argv[7]), atoi(argv[8]));
    const Long n = save_gauge_field(gf, path);
    printf("{\"bytes\": %ld, \"plaq\": %.17g, \"link_trace\": %.17g}\n", (long)n, gf_avg_plaq(gf),
           gf_avg_link_trace(gf));
  } else if (mode == "load") {
    GaugeField gf;
    const Long n = load_gauge_field(gf, path);
    const Geometry& geo = gf.geo();
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 1;
    for (Long i = 0; i < geo.local_volume(); ++i) {
      const Vector<ColorMatrix> v = gf.get_elems_const(i);
      fwrite(v.data(), sizeof(ColorMatrix), v.size(), f);
    }
    fclose(f);
    printf("{\"bytes\": %ld, \"plaq\": %.17g}\n", (long)n, gf_avg_plaq(gf));
  } else {
    fprintf(stderr, "bad arguments\n");
    return 2;
  }
  end();
  return 0;
}
