// A time-slab caller written against the C ABI alone: one rank holding the
// whole 4^3 x 16 lattice as an expanded field with 2 halo slices on each side
// (the reference's expansion for the rectangle action, field-expand.h), its
// halo refreshed by a C hook that the library calls before every force
// evaluation, as refresh_expanded precedes each force in hmc.cpp:466-490.
// The slab trajectory (FP32 molecular dynamics on FP32 copies, FP64
// Hamiltonians over the owned sites) must reproduce the trajectory of the
// plain field: the same delta_h and the same links on every owned site.
// Prints "CHECK: slab hook ok" and exits 0 on success.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "qlat_b200.h"

#define CK(x)                                                                   \
  do {                                                                          \
    const int rc_ = (x);                                                        \
    if (rc_ != QGB_OK) {                                                        \
      std::fprintf(stderr, "%s:%d: %s -> %d: %s\n", __FILE__, __LINE__, #x, rc_, \
                   qgb_last_error());                                           \
      return 1;                                                                 \
    }                                                                           \
  } while (0)

struct Slab {
  int nt, h;           // owned slices, halo slices on each side
  void* buf[2] = {nullptr, nullptr};
  size_t cap = 0;
  int calls = 0;
};

// One rank: the bottom halo is a copy of the top owned slices and the top
// halo a copy of the bottom owned slices (the periodic ring of one slab).
static int refresh_halo(qgb_field* f, void* user)
{
  Slab* sl = static_cast<Slab*>(user);
  int64_t n = 0;
  if (qgb_field_tslice_bytes(f, sl->h, &n) != QGB_OK) return 1;
  if ((size_t)n > sl->cap) {
    for (void*& b : sl->buf) {
      if (b) cudaFree(b);
      if (cudaMalloc(&b, (size_t)n) != cudaSuccess) return 2;
    }
    sl->cap = (size_t)n;
  }
  if (qgb_field_pack_tslices(f, sl->nt, sl->h, sl->buf[0]) != QGB_OK) return 3;  // top owned slices
  if (qgb_field_pack_tslices(f, sl->h, sl->h, sl->buf[1]) != QGB_OK) return 3;   // bottom owned slices
  if (qgb_field_unpack_tslices(f, 0, sl->h, sl->buf[0]) != QGB_OK) return 4;
  if (qgb_field_unpack_tslices(f, sl->nt + sl->h, sl->h, sl->buf[1]) != QGB_OK) return 4;
  sl->calls++;
  return 0;
}

int main()
{
  const int X = 4, Y = 4, Z = 4, T = 16, H = 2, N_STEP = 4, REUNIT = 2;
  const double beta = 2.13, c1 = -0.331, sigma = 0.3;
  const int32_t ts[4] = {X, Y, Z, T}, tl[4] = {X, Y, Z, T + 2 * H};
  const long V3 = (long)X * Y * Z, V = V3 * T, VL = V3 * (T + 2 * H);
  const int64_t s0 = H * V3, s1 = (H + T) * V3;  // owned sites of the slab
  uint32_t rs[24], r_init[24], r_mom[24];
  CK(qgb_rng_seed(rs, "slab-hook"));
  CK(qgb_rng_split(r_init, rs, "gf-init"));
  CK(qgb_rng_split(r_mom, rs, "mom"));

  qgb_field *gf = nullptr, *gm = nullptr, *sgf = nullptr, *sgm = nullptr;
  qgb_field *gf32 = nullptr, *gm32 = nullptr, *sgf32 = nullptr, *sgm32 = nullptr;
  CK(qgb_field_create(&gf, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
  CK(qgb_field_create(&gm, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
  CK(qgb_field_create(&gf32, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F32));
  CK(qgb_field_create(&gm32, ts, 4, QGB_KIND_COLOR_MATRIX, QGB_F32));
  CK(qgb_field_create(&sgf, tl, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
  CK(qgb_field_create(&sgm, tl, 4, QGB_KIND_COLOR_MATRIX, QGB_F64));
  CK(qgb_field_create(&sgf32, tl, 4, QGB_KIND_COLOR_MATRIX, QGB_F32));
  CK(qgb_field_create(&sgm32, tl, 4, QGB_KIND_COLOR_MATRIX, QGB_F32));

  // the same hot start and momenta on the plain field and on the slab's
  // owned sites (the slab's site s is global site s - H V3)
  CK(qgb_gf_set_rand(gf, r_init, sigma, 1));
  CK(qgb_set_rand_gauge_momentum(gm, 1.0, r_mom));
  CK(qgb_gf_set_rand_sites(sgf, r_init, sigma, 1, -s0));
  CK(qgb_set_rand_gauge_momentum_sites(sgm, 1.0, r_mom, -s0));
  Slab sl;
  sl.nt = T;
  sl.h = H;
  if (refresh_halo(sgf, &sl)) return 1;

  // plain trajectory: H0, FP32 molecular dynamics, back to FP64, H1
  double k0, a0, k1, a1;
  CK(qgb_gm_hamilton_node(gm, &k0));
  CK(qgb_gf_hamilton_node(gf, beta, c1, &a0));
  CK(qgb_field_copy(gf32, gf));
  CK(qgb_field_copy(gm32, gm));
  CK(qgb_run_md_hooked(gm32, gf32, beta, c1, N_STEP, 1.0, QGB_INTEGRATOR_FORCE_GRADIENT, REUNIT, 0, nullptr,
                       nullptr));
  CK(qgb_field_copy(gf, gf32));
  CK(qgb_field_copy(gm, gm32));
  CK(qgb_unitarize(gf));
  CK(qgb_gm_hamilton_node(gm, &k1));
  CK(qgb_gf_hamilton_node(gf, beta, c1, &a1));
  const double dh = (k1 + a1) - (k0 + a0);

  // slab trajectory: the same steps, owned-site sums, a halo refresh before
  // every force (refresh_shifted = 1: the 2-slice halo is the force's reach)
  double sk0, sa0, sk1, sa1;
  CK(qgb_gm_hamilton_node_sites(sgm, s0, s1, &sk0));
  CK(qgb_gf_hamilton_node_sites(sgf, beta, c1, s0, s1, &sa0));
  CK(qgb_field_copy(sgf32, sgf));
  CK(qgb_field_copy(sgm32, sgm));
  CK(qgb_run_md_hooked(sgm32, sgf32, beta, c1, N_STEP, 1.0, QGB_INTEGRATOR_FORCE_GRADIENT, REUNIT, 1,
                       refresh_halo, &sl));
  CK(qgb_field_copy(sgf, sgf32));
  CK(qgb_field_copy(sgm, sgm32));
  CK(qgb_unitarize(sgf));
  if (refresh_halo(sgf, &sl)) return 1;
  CK(qgb_gm_hamilton_node_sites(sgm, s0, s1, &sk1));
  CK(qgb_gf_hamilton_node_sites(sgf, beta, c1, s0, s1, &sa1));
  const double sdh = (sk1 + sa1) - (sk0 + sa0);

  std::vector<double> a((size_t)V * 4 * 18), b((size_t)VL * 4 * 18);
  CK(qgb_field_download(gf, a.data()));
  CK(qgb_field_download(sgf, b.data()));
  double dmax = 0.0;
  for (long s = 0; s < V; ++s)
    for (int k = 0; k < 4 * 18; ++k)
      dmax = std::fmax(dmax, std::fabs(a[(size_t)s * 72 + k] - b[(size_t)(s + s0) * 72 + k]));
  const int expected_calls = 2 + 4 * N_STEP;  // 2 direct, 2 per force-gradient update
  std::printf("delta_h plain %.15e slab %.15e ; max link difference %.3e ; hook calls %d\n", dh, sdh, dmax,
              sl.calls);
  const bool ok = std::fabs(dh - sdh) < 1e-9 && dmax < 1e-12 && sl.calls == expected_calls;
  for (qgb_field* f : {gf, gm, gf32, gm32, sgf, sgm, sgf32, sgm32}) qgb_field_destroy(f);
  for (void* p : sl.buf)
    if (p) cudaFree(p);
  if (!ok) {
    std::printf("CHECK: slab hook MISMATCH\n");
    return 1;
  }
  std::printf("CHECK: slab hook ok\n");
  return 0;
}
