// Host check of the su(3) exponential (su3.cuh: exp_su3) in FP32 and FP64
// against the general Cayley-Hamilton exponential in FP64 (exp_ch<double>, all
// 20 terms of the reference's Taylor polynomial) on random su(3) matrices with
// Frobenius norms from 1e-5 to 3.4.  Prints the largest entry error per norm
// and exits non-zero when either precision exceeds its bound (argv[1] FP32,
// argv[2] FP64).
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <random>

#include "su3.cuh"

using namespace qgb;

int main(int argc, char** argv)
{
  const double bound = argc > 1 ? atof(argv[1]) : 1e-6;
  const double bound64 = argc > 2 ? atof(argv[2]) : 1e-14;
  double worst64 = 0;
  std::mt19937_64 gen(12345);
  std::normal_distribution<double> nd(0.0, 1.0);
  double worst = 0;
  const double norms[] = {1e-5, 1e-4, 1e-3, 1e-2, 0.1, 0.3, 0.5, 1.0, 2.0, 3.4};
  for (double target : norms) {
    double err = 0, err64 = 0;
    for (int trial = 0; trial < 2000; ++trial) {
      // a = X - X^+ made traceless, scaled to the target norm
      double xr[9], xi[9];
      for (int k = 0; k < 9; ++k) { xr[k] = nd(gen); xi[k] = nd(gen); }
      M3<double> a;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          a.e[3 * i + j] = cx<double>(0.5 * (xr[3 * i + j] - xr[3 * j + i]), 0.5 * (xi[3 * i + j] + xi[3 * j + i]));
      const double tr = (a.e[0].im + a.e[4].im + a.e[8].im) / 3;
      for (int i = 0; i < 3; ++i) a.e[4 * i].im -= tr;
      double nrm = 0;
      for (int k = 0; k < 9; ++k) nrm += a.e[k].re * a.e[k].re + a.e[k].im * a.e[k].im;
      nrm = sqrt(nrm);
      M3<float> af;
      for (int k = 0; k < 9; ++k) {
        a.e[k].re *= target / nrm;
        a.e[k].im *= target / nrm;
        af.e[k] = cx<float>((float)a.e[k].re, (float)a.e[k].im);
      }
      // FP32: against the FP64 reference on the same (FP32-rounded) input
      M3<double> ad;
      for (int k = 0; k < 9; ++k) ad.e[k] = cx<double>(af.e[k].re, af.e[k].im);
      const M3<double> e64 = exp_ch(ad);
      const M3<float> e32 = exp_su3(af);
      // FP64: on the FP64 matrix itself (su(3) to FP64 rounding; the FP32-rounded
      // one is not traceless to FP64 resolution)
      const M3<double> r64 = exp_ch(a);
      const M3<double> s64 = exp_su3(a);
      for (int k = 0; k < 9; ++k) {
        err = fmax(err, fmax(fabs(e32.e[k].re - e64.e[k].re), fabs(e32.e[k].im - e64.e[k].im)));
        err64 = fmax(err64, fmax(fabs(s64.e[k].re - r64.e[k].re), fabs(s64.e[k].im - r64.e[k].im)));
      }
    }
    printf("norm %-8g max entry error FP32 %.3e FP64 %.3e\n", target, err, err64);
    worst = fmax(worst, err);
    worst64 = fmax(worst64, err64);
  }
  printf("worst FP32 %.3e (bound %.3e), FP64 %.3e (bound %.3e)\n", worst, bound, worst64, bound64);
  return worst <= bound && worst64 <= bound64 ? 0 : 1;
}
