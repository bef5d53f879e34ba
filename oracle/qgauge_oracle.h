/* qgauge_oracle.h -- CPU restatement of Qlattice's pure-gauge SU(3) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it.  No
 * product code path links, loads or calls it.
 *
 * Fields are in the reference layout (Qlattice core.h:191-197,753-861): site
 * major, sites ordered with x fastest (coordinate.h:182-188), then the
 * multiplicity (4 links per site for gauge fields and momenta), then a
 * row-major 3x3 complex matrix stored as (re, im) pairs: 18 doubles per
 * matrix, 72 doubles per site.  dims[] = {X, Y, Z, T}.
 *
 * Parity is pinned two ways: against the golden logs shipped with the
 * reference (examples-cpp/hmc/log, examples-py/*.log.json) and against the
 * reference library itself compiled from source (oracle/ref/). */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of the reference RngState (qlat-utils rng-state.h:38-99). */
typedef struct {
  uint64_t numBytes;
  uint32_t hash[8];
  uint64_t type;
  uint64_t index;
  uint64_t cache[3];
  double gaussian;
  int32_t cacheAvail;
  int32_t gaussianAvail;
} or_rng;

/* log used inside the Gaussian draw: 0 = the C library's log (what the
 * reference calls, rng-state.cpp:276), 1 = a correctly rounded log computed
 * through binary128 (libquadmath) and rounded once to double. */
void or_set_log_mode(int mode);

void or_sha256_block(uint32_t out[8], const uint32_t in[8], const uint8_t data[64]);
void or_sha256_final(uint32_t out[8], const uint32_t in[8], uint64_t num_bytes,
                     const uint8_t* input, uint64_t input_size);
void or_sha256_initial(uint32_t h[8]);

void or_rng_reset(or_rng* rs);
void or_rng_seed(or_rng* rs, const char* seed);
void or_rng_split(or_rng* out, const or_rng* rs0, const char* sindex);
void or_rng_split_long(or_rng* out, const or_rng* rs0, int64_t sindex);
uint64_t or_rand_gen(or_rng* rs);
double or_u_rand_gen(or_rng* rs, double upper, double lower);
double or_g_rand_gen(or_rng* rs, double center, double sigma);
void or_rng_export(uint32_t v[24], const or_rng* rs);
void or_rng_import(or_rng* rs, const uint32_t v[24]);

/* Field-level operations (single node, periodic). */
void or_set_unit(double* gf, const int dims[4]);
void or_set_rand_gauge_momentum(double* gm, const int dims[4], const or_rng* rs, double sigma);
void or_set_g_rand_color_matrix_field(double* gf, const int dims[4], const or_rng* rs, double sigma,
                                      int n_step);
double or_gf_avg_plaq(const double* gf, const int dims[4]);
double or_gm_hamilton_node(const double* gm, const int dims[4]);
double or_gf_sum_re_tr_plaq(const double* gf, const int dims[4]);
double or_gf_sum_re_tr_rect(const double* gf, const int dims[4]);
double or_gf_hamilton_node(const double* gf, const int dims[4], double beta, double c1);
void or_set_gm_force(double* gm_force, const double* gf, const int dims[4], double beta, double c1);
void or_gf_evolve(double* gf, const double* gm, const int dims[4], double step_size);
void or_unitarize_field(double* gf, const int dims[4]);
void or_gf_wilson_flow_step(double* gf, const int dims[4], double epsilon, double c1);
void or_gf_wilson_flow_step_euler(double* gf, const int dims[4], double epsilon, double c1);
void or_gf_energy_density_field(double* fd, const double* gf, const int dims[4]);
double or_gf_energy_density(const double* gf, const int dims[4]);
void or_clf_topology_field(double* topf, const double* gf, const int dims[4]);
double or_gf_topology_clf(const double* gf, const int dims[4]);
/* qcd.cpp:425-489: the five terms of the improved (5-loop) charge density, topf[5 * site + k] */
void or_clf_topology_field_5_terms(double* topf, const double* gf, const int dims[4]);
/* topology.pyx:98-108: the improved charge, summed over the lattice */
double or_gf_topology(const double* gf, const int dims[4]);
/* Omelyan force-gradient trajectory (hmc.pyx:170-188); returns delta_h. */
double or_run_hmc_evolve_fg(double* gm, double* gf, const int dims[4], double beta, double c1,
                            int n_step, double md_time);
/* Leapfrog composition of the same primitives (examples-py/hmc-pure-gauge-fgf.py:57-69):
 * per step gf_evolve(dt/2), gm += dt F, gf_evolve(dt/2); returns delta_h. */
double or_run_hmc_evolve_leapfrog(double* gm, double* gf, const int dims[4], double beta, double c1,
                                  int n_step, double md_time);
/* Field-accelerated HMC (hmc.cpp:121-201, 330-396, 492-645).  A mass field mf
 * holds 4 doubles per site (one per link), +inf freezing a link. */
/* set_u_rand / set_g_rand of a field (core.h:1585-1636): per site
 * rs.newtype(site index), n_per_site draws in memory order. */
void or_field_set_u_rand(double* f, const int dims[4], int n_per_site, const or_rng* rs, double upper, double lower);
void or_field_set_g_rand(double* f, const int dims[4], int n_per_site, const or_rng* rs, double center, double sigma);
void or_set_rand_gauge_momentum_fa(double* gm, const double* mf, const int dims[4], const or_rng* rs);
double or_gm_hamilton_node_fa(const double* gm, const double* mf, const int dims[4]);
/* dual = 0: U = unitarize(exp(dt/m P) U); dual = 1: U = unitarize(U exp(-dt/m P));
 * mf NULL: m = 1 (the overloads without a mass field). */
void or_gf_evolve_fa(double* gf, const double* gm, const double* mf, const int dims[4], double step_size, int dual);
void or_set_gm_force_dual(double* fd, const double* gf, const double* f, const int dims[4]);
double or_project_gauge_transform(double* gm, double* gmd, const double* mf, const double* mfd, const int dims[4]);
void or_set_gauge_transform_momentum(double* gm, double* gmd, const double* gtm, const int dims[4]);
void or_dot_gauge_momentum(double* f, const double* gm1, const double* gm2, const int dims[4]);
/* Topology-measurement flows (qcd.cpp:33-62, 295-341; wilson-flow.cpp:164-236;
 * instanton_map.py:91-191).  Plaquette fields hold 6 doubles per site, planes
 * (0,1) (0,2) (0,3) (1,2) (1,3) (2,3). */
void or_gf_plaq_field(double* f_plaq, const double* gf, const int dims[4]);
/* qcd-utils.cpp:359-400: Re tr / 3 of the l x t Wilson loop averaged over sites and spatial directions */
double or_gf_avg_wilson_loop_normalized_tr(const double* gf, const int dims[4], int l, int t);
/* wilson-flow.cpp:53-95: per site and plane -Re tr(G G), G = TA(clover); 6 per site */
void or_gf_energy_density_dir_field(double* fd, const double* gf, const int dims[4]);
void or_clf_plaq_action_density_field(double* paf, const double* gf, const int dims[4], int spatial);
void or_set_plaq_flow_z(double* z, const double* gf, const double* plaq_factor, const int dims[4]);
/* one step of a plaquette-weighted flow: kind 1 Shrink, 2 Freeze, 3 Localize,
 * 4 Preserve; returns step_size / norm */
double or_gf_flow_topo_plaq(double* gf, const int dims[4], double step_size, int kind);
/* Single-matrix helpers used by the tests. */
void or_make_matrix_exp(double out[18], const double a[18], int max_order);
void or_unitarize(double m[18]);
void or_make_tr_less_anti_herm(double out[18], const double m[18]);

#ifdef __cplusplus
}
#endif
