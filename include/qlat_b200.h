/* qlat_b200.h -- C ABI of the B200-native pure-gauge SU(3) hot path.
 *
 * This is the drop-in boundary for Qlattice's pure-gauge HMC and gradient-flow
 * path.  Every entry point below replaces one C++ function that Qlattice's
 * Cython layer binds (qlat/qlat/everything.pxd) or that the C++ drivers call
 * (examples-cpp/hmc/main.cpp); the reference declaration is cited beside it.
 * Paths are inside the Qlattice project.
 *
 * Conventions
 *  - Every function returns an int status: QGB_OK (0) or one of the QGB_ERR_*
 *    codes; qgb_last_error() gives a message for the calling thread.  This
 *    replaces the reference's `qerr` C++ exceptions, which Cython turns into
 *    RuntimeError (`except +`).
 *  - A qgb_field is an opaque handle to a lattice field resident in GPU
 *    memory: a GaugeField (multiplicity 4, color matrices), a GaugeMomentum
 *    (same shape), or a Field<RealD> (real numbers, any multiplicity).  It is
 *    stored in FP64 or FP32 (QGB_F64 / QGB_F32).
 *  - Host buffers passed to upload/download use the reference memory image
 *    (core.h:753-861): site-major, x fastest (coordinate.h:182-188), then the
 *    multiplicity index, then a row-major 3x3 complex matrix of (re, im)
 *    doubles -- i.e. exactly what np.asarray(qlat.GaugeField) exposes.
 *  - RngState crosses the boundary in its 24 x uint32 serialised form
 *    (rng-state.cpp:61-81, exportRngState / importRngState).
 *  - Work is queued on the library's current CUDA stream (qgb_set_stream);
 *    functions that return host scalars synchronise that stream.
 *  - Single GPU, single node: the `_node` functions are whole-lattice sums.
 */
#ifndef QLAT_B200_H
#define QLAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QGB_OK 0
#define QGB_ERR_INVALID_ARG 1
#define QGB_ERR_BAD_GEOMETRY 2
#define QGB_ERR_ALLOC 3
#define QGB_ERR_CUDA 4
#define QGB_ERR_NAN 5
#define QGB_ERR_TIMEOUT 6
#define QGB_ERR_MISMATCH 7
#define QGB_ERR_NO_DEVICE 8
#define QGB_ERR_IO 9 /* file missing, unreadable, short or not in the expected format */
#define QGB_ERR_HOOK 10 /* a caller-supplied hook returned non-zero */

#define QGB_F64 64
#define QGB_F32 32

#define QGB_KIND_COLOR_MATRIX 0
#define QGB_KIND_REAL 1

#define QGB_INTEGRATOR_FORCE_GRADIENT 0
#define QGB_INTEGRATOR_LEAPFROG 1

typedef struct qgb_field_s qgb_field;
typedef struct qgb_batch_s qgb_batch;

/* ---- library state ---------------------------------------------------- */

/* Message of the last failing call on this thread ("" if none). */
const char* qgb_last_error(void);
/* Library version as an integer (major*10000 + minor*100 + patch). */
int qgb_version(void);
/* Select the CUDA device used by subsequent calls of this thread. */
int qgb_set_device(int32_t device);
/* Use `stream` (a cudaStream_t, may be NULL for the legacy default stream)
 * for all subsequent work; the library otherwise creates its own stream. */
int qgb_set_stream(void* stream);
int qgb_synchronize(void);

/* ---- fields (Field<M> / GaugeField / GaugeMomentum: core.h:753-969) ------ */

/* Geometry(total_site) + Field::init(geo, multiplicity) (core.h:92-359,
 * 753-781); kind is QGB_KIND_COLOR_MATRIX or QGB_KIND_REAL. */
int qgb_field_create(qgb_field** out, const int32_t total_site[4], int32_t multiplicity, int32_t kind,
                     int32_t precision);
/* Releases the field; its device storage is kept in a pool keyed by size and
 * reused by the next qgb_field_create of that size (the reference's
 * run_hmc_pure_gauge, hmc.pyx:190-216, builds a link copy and a momentum field
 * every trajectory). */
int qgb_field_destroy(qgb_field* f);
/* Frees the pooled storage of destroyed fields (qgb_field_create also does
 * this by itself when cudaMalloc runs out of memory); writes the bytes freed
 * when released is not NULL. */
int qgb_field_pool_release(int64_t* released);
int qgb_field_info(const qgb_field* f, int32_t total_site[4], int32_t* multiplicity, int32_t* kind,
                   int32_t* precision);
/* Copy a host buffer in the reference memory image into the field (and back).
 * Color-matrix fields take complex128 (double pairs); real fields take double. */
int qgb_field_upload(qgb_field* f, const double* host);
int qgb_field_download(const qgb_field* f, double* host);
/* Stream a sequence of host configurations into f, overlapping each copy with
 * the work queued after it: copy host_now into f (from the library's staging
 * copy if an earlier call prefetched it, else now), then start the
 * host-to-device copy of host_next (may be NULL) on a library copy stream, to
 * be committed by the next call with host_now = host_next.  The prefetch reads
 * host_next when the copy engine reaches it: keep that buffer unchanged until
 * the next call.  Overlap needs pinned host memory. */
int qgb_field_upload_pipelined(qgb_field* f, const double* host_now, const double* host_next);
/* Queue a copy of f, in the reference memory image, into `host` behind the
 * work queued so far, without waiting: the field is converted into one of two
 * library staging slots on the library stream and copied to the host on a
 * library download stream, so the copy overlaps the work queued after it
 * (pinned host memory).  `host` holds the data once qgb_synchronize (or
 * qgb_field_download_join followed by a synchronisation of the library
 * stream) has returned; keep it unread and unchanged until then.  A third
 * download waits for the first's copy to leave its slot. */
int qgb_field_download_async(const qgb_field* f, double* host);
/* Orders the library stream after every queued download (qgb_synchronize does
 * this itself). */
int qgb_field_download_join(void);
/* Same, from / into a device buffer in the reference memory image. */
int qgb_field_upload_device(qgb_field* f, const double* dev);
int qgb_field_download_device(const qgb_field* f, double* dev);
/* f1 @= f2 (field_types.pyx.in:92 `@=`); converts between FP64 and FP32. */
int qgb_field_copy(qgb_field* dst, const qgb_field* src);
int qgb_field_set_zero(qgb_field* f);
/* y = a*x + b*y: covers `f *= s` (x = y or a = 0), `f += g`, `f -= g`
 * (field.h operators used by hmc.pyx:166-167 and wilson-flow.cpp:36-46). */
int qgb_field_axpby(qgb_field* y, double a, const qgb_field* x, double b);
/* qnorm(field) = sum of |element|^2 (field.h, qnorm). */
int qgb_field_qnorm(const qgb_field* f, double* out);

/* ---- RngState (rng-state.h:12-99, lib/rng-state.cpp:150-281) ------------ */

/* RngState(seed): reset(rs, seed); seed NULL: RngState(), reset(rs)
 * (rng-state.cpp:150-164). */
int qgb_rng_seed(uint32_t out[24], const char* seed);
/* rs.split(sindex) (split_rng_state, rng-state.cpp:173-201). */
int qgb_rng_split(uint32_t out[24], const uint32_t rs[24], const char* sindex);
/* rand_gen / u_rand_gen / g_rand_gen (rng-state.cpp:203-281); update rs. */
int qgb_rng_rand_gen(uint32_t rs[24], uint64_t* out);
int qgb_rng_u_rand_gen(uint32_t rs[24], double upper, double lower, double* out);
int qgb_rng_g_rand_gen(uint32_t rs[24], double center, double sigma, double* out);

/* ---- hot path: gauge field set-up (qcd-utils.cpp:47-92, qcd.pyx:69) ----- */

/* set_unit(gf) (field.h set_unit, everything.pxd:187). */
int qgb_set_unit(qgb_field* gf);
/* GaugeField.set_rand(rs, sigma, n_step) -> set_g_rand_color_matrix_field
 * (qcd-utils.cpp:71-92): per site RngState(rs, gindex), n_step products of
 * exp(X) (order-20 Taylor, then unitarize) with X from 8 Gaussians of std
 * sigma/sqrt(2). */
int qgb_gf_set_rand(qgb_field* gf, const uint32_t rs[24], double sigma, int32_t n_step);

/* ---- hot path: HMC (hmc.h:20-114, everything.pxd:437-456) --------------- */

/* set_rand_gauge_momentum(gm, sigma, rs) (hmc.cpp:107-119). */
int qgb_set_rand_gauge_momentum(qgb_field* gm, double sigma, const uint32_t rs[24]);
/* gm_hamilton_node(gm) (hmc.cpp:151-173). */
int qgb_gm_hamilton_node(const qgb_field* gm, double* out);
/* gf_hamilton_node(gf, ga) (hmc.cpp:254-298). */
int qgb_gf_hamilton_node(const qgb_field* gf, double beta, double c1, double* out);
/* gf_sum_re_tr_plaq_node_no_comm / gf_sum_re_tr_rect_node_no_comm (hmc.cpp:203-252). */
int qgb_gf_sum_re_tr_plaq_node(const qgb_field* gf, double* out);
int qgb_gf_sum_re_tr_rect_node(const qgb_field* gf, double* out);
/* gf_avg_plaq(gf) (qcd.cpp:94-142). */
int qgb_gf_avg_plaq(const qgb_field* gf, double* out);
/* set_gm_force(gm_force, gf, GaugeAction(beta, c1)) (hmc.cpp:466-490). */
int qgb_set_gm_force(qgb_field* gm_force, const qgb_field* gf, double beta, double c1);
/* gf_evolve(gf, gm, step_size) (hmc.cpp:311-328). */
int qgb_gf_evolve(qgb_field* gf, const qgb_field* gm, double step_size);
/* gm_evolve_fg_pure_gauge(gm, gf_init, ga, fg_dt, dt) (hmc.pyx:157-167). */
int qgb_gm_evolve_fg(qgb_field* gm, const qgb_field* gf_init, double beta, double c1, double fg_dt,
                     double dt);
/* unitarize(gf) (qcd.cpp:346-359). */
int qgb_unitarize(qgb_field* gf);
/* metropolis_accept(accept_prob, delta_h, traj, rs) (hmc.cpp:77-105). */
int qgb_metropolis_accept(double delta_h, int32_t traj, const uint32_t rs[24], double* accept_prob,
                          int32_t* flag);
/* run_hmc_evolve_pure_gauge(gm, gf, ga, rs, n_step, md_time) (hmc.pyx:169-188),
 * force-gradient or leapfrog (examples-py/hmc-pure-gauge-fgf.py:57-69), all
 * in the fields' precision (FP64 for the plain form); writes delta_h. */
int qgb_run_hmc_evolve(qgb_field* gm, qgb_field* gf, double beta, double c1, int32_t n_step,
                       double md_time, int32_t integrator, double* delta_h);
/* Mixed form of the same trajectory: gm and gf are FP64; molecular dynamics
 * runs on FP32 copies, links are re-unitarised in FP64 arithmetic every
 * `reunit_interval` steps, and both Hamiltonians are FP64 sums on FP64 fields. */
int qgb_run_hmc_evolve_mixed(qgb_field* gm, qgb_field* gf, double beta, double c1, int32_t n_step,
                             double md_time, int32_t integrator, int32_t reunit_interval,
                             double* delta_h);
/* The two entry points above replay their kernels as a CUDA graph (no
 * counterpart in the reference): the first call with given fields, geometry,
 * parameters and force-kernel shapes launches directly, the second records
 * the launches and replays them, later calls replay -- the same kernels with
 * the same arguments, one graph launch instead of 40 or more kernel launches.
 * Direct launches are used while per-kernel timing is on, while the caller
 * captures the stream and on the legacy default stream.  enable = 0 switches
 * graphs off (and frees the recorded ones); qgb_trajectory_graph_count gives
 * the number held (at most 16, least recently used dropped first). */
int qgb_set_trajectory_graphs(int32_t enable);
int qgb_trajectory_graph_count(int32_t* n);

/* Halo hook of a domain-decomposed trajectory: called with a link field
 * before a force evaluation reads it, after the kernels before it have been
 * enqueued on the library stream; it must leave the field's halo sites fresh
 * copies of the neighbouring domains' links and return 0 (any other value
 * aborts the trajectory with QGB_ERR_HOOK). */
typedef int (*qgb_halo_hook)(qgb_field* gf, void* user);
/* The molecular dynamics of run_hmc_evolve_pure_gauge (hmc.pyx:169-188)
 * without the Hamiltonians, in the fields' precision (gm, gf both FP64 or both
 * FP32), on the reference's refresh-before-force schedule (hmc.cpp:466-490
 * refreshes the expanded field before each force).  When hook is not NULL,
 * hook(gf, user) runs before each force evaluation on gf, and with
 * refresh_shifted != 0 also hook(shifted, user) before the force at the
 * force-gradient shift U' = exp(eps F(U)) U (shifted: a library-owned field of
 * gf's shape; a halo thinner than twice the force's reach needs it).  The
 * kernel sequence is the one qgb_run_hmc_evolve (reunit_interval = 0:
 * unitarise after every exponential) and qgb_run_hmc_evolve_mixed
 * (reunit_interval > 0, on FP32 fields: FP64 re-unitarisation every that many
 * steps) run. */
int qgb_run_md_hooked(qgb_field* gm, qgb_field* gf, double beta, double c1, int32_t n_step, double md_time,
                      int32_t integrator, int32_t reunit_interval, int32_t refresh_shifted, qgb_halo_hook hook,
                      void* user);

/* ---- hot path: gradient flow (wilson-flow.h:9-43, everything.pxd:514-521) --- */

/* set_wilson_flow_z(z, gf, c1) = set_gm_force with beta = 3 (wilson-flow.cpp:12-17). */
int qgb_set_wilson_flow_z(qgb_field* z, const qgb_field* gf, double c1);
/* gf_wilson_flow_step(gf, epsilon, c1): Luescher RK3 (wilson-flow.cpp:29-50). */
int qgb_gf_wilson_flow_step(qgb_field* gf, double epsilon, double c1);
/* gf_wilson_flow_step_euler(gf, epsilon, c1) (wilson-flow.cpp:19-27). */
int qgb_gf_wilson_flow_step_euler(qgb_field* gf, double epsilon, double c1);
/* gf_energy_density_field(fd, gf) (wilson-flow.cpp:99-129); fd: real, multiplicity 1. */
int qgb_gf_energy_density_field(qgb_field* fd, const qgb_field* gf);
/* gf_energy_density(gf) (wilson-flow.cpp:131-141). */
int qgb_gf_energy_density(const qgb_field* gf, double* out);
/* gf_wilson_flow(gf, existing_flow_time, flow_time, steps, c1) (wilson-flow.cpp:144-162);
 * energy_list receives `steps` energy densities. */
int qgb_gf_wilson_flow(qgb_field* gf, double flow_time, int32_t steps, double c1, double* energy_list);

/* ---- flow adjoint (no counterpart in the reference) ---------------------- */

/* Tangents and gradients are su(3) fields acting by left multiplication,
 * U -> exp(s X) U; the gradient of L is sum_a (dL/domega_a) T_a in the basis of
 * matrix-hmc.h:76-106 (tr T_a T_b = -2 delta_ab).  With this convention the
 * gradient of the gauge action is -2 x set_gm_force.
 *
 * Vector-Jacobian product of `steps` RK3 flow steps of size epsilon
 * (gf_wilson_flow_step, wilson-flow.cpp:29-50, with the flow force of
 * GaugeAction(3, c1), set_wilson_flow_z at wilson-flow.cpp:12-17: Wilson,
 * Iwasaki, DBW2 or any c1): given the cotangent at the flowed field, writes
 * the cotangent at gf.  Forward states are checkpointed every
 * `checkpoint_every` steps and recomputed. */
int qgb_gf_wilson_flow_vjp(const qgb_field* gf, double epsilon, int32_t steps, double c1, int32_t checkpoint_every,
                           const qgb_field* cotangent, qgb_field* grad);
/* L = gf_hamilton_node(V_t, GaugeAction(beta, c1_loss)) of the flowed field
 * V_t (steps RK3 steps of epsilon) and its gradient with respect to gf. */
int qgb_gf_flow_action_grad(const qgb_field* gf, double epsilon, int32_t steps, double c1, int32_t checkpoint_every,
                            double beta, double c1_loss, qgb_field* grad, double* loss);
/* set_anti_hermitian_matrix_from_basis / set_basis_from_anti_hermitian_matrix
 * (hmc.h:108-113, hmc.cpp:647-697): fc[x, m] = sum_a T_a basis[x, 8 m + a]. */
int qgb_set_anti_hermitian_matrix_from_basis(qgb_field* fc, const qgb_field* basis);
int qgb_set_basis_from_anti_hermitian_matrix(qgb_field* basis, const qgb_field* fc);
/* out = dexp_{-omega}(lam) per link: the gradient with respect to omega of a
 * function of exp(omega) U whose gradient at exp(omega) U is lam. */
int qgb_su3_dexp_adjoint(qgb_field* out, const qgb_field* omega, const qgb_field* lam);

/* ---- hot path: topology (qcd-topology.h, everything.pxd:531-535) --------- */

/* clf_topology_field(topf, gf) (qcd.cpp:416-423, 608-619); topf: real, multiplicity 1. */
int qgb_clf_topology_field(qgb_field* topf, const qgb_field* gf);
/* gf_topology_clf(gf) = glb_sum of clf_topology_field (topology.pyx:89-96). */
int qgb_gf_topology_clf(const qgb_field* gf, double* out);

/* The 5-loop improved topological charge (hep-lat/9701012 Eq. 2-7): the five
 * terms c_k / (m n)^2 q_{m x n} of the m x n clover-leaf densities, (m, n) =
 * (1,1), (2,2), (1,2), (1,3), (3,3), the 1 x 2 and 1 x 3 leaves averaged with
 * their transposes.
 * Replaces clf_topology_field_5_terms (qcd.cpp:425-489; topology.pyx:121-140,
 * gf_topology_terms_field / gf_topology_terms): topf real, multiplicity 5, the
 * links' precision. */
int qgb_clf_topology_field_5_terms(qgb_field* topf, const qgb_field* gf);
/* Replaces clf_topology_field_5 (qcd.cpp:491-509; topology.pyx:98-108,
 * gf_topology_field): per-site sum of the five terms, topf multiplicity 1. */
int qgb_clf_topology_field_5(qgb_field* topf, const qgb_field* gf);
/* The five terms summed over the lattice (topology.pyx:130-140, gf_topology_terms). */
int qgb_gf_topology_terms(const qgb_field* gf, double out[5]);
/* Their sum, the improved charge (topology.pyx:110-118, gf_topology). */
int qgb_gf_topology(const qgb_field* gf, double* out);

/* ---- instrumentation (timer.h:48-414 TIMER / Timer::display) ------------ */

/* Per-kernel-class device timing with CUDA events on the library stream. */
int qgb_prof_enable(int32_t on);
int qgb_prof_reset(void);
/* name: "force", "force_update", "force_evolve", "evolve", "reduce", "rng",
 * "unitarize", "convert", "clover", "flow_stage"; totals since the last reset. */
int qgb_prof_get(const char* name, double* total_ms, int64_t* launches);
/* ---- batches of independent chains (no counterpart in the reference) ---- */

/* Many independent pure-gauge HMC chains of different lattice sizes, betas and
 * c1 advanced together: every phase of a trajectory is one launch over all
 * chains, and the trajectory is recorded once as a CUDA graph per
 * (n_step, md_time, integrator, precision) and replayed.  Chain c has lattice
 * total_sites[4c .. 4c+3], beta[c], c1[c]; RngStates are 24 x uint32 per chain,
 * concatenated.  Each chain follows run_hmc_evolve_pure_gauge (hmc.pyx:169-188)
 * with the per-site RngState(rs_c, gindex) momenta of set_rand_gauge_momentum
 * (hmc.cpp:107-119); accept/reject is the caller's (qgb_batch_accept). */
int qgb_batch_create(qgb_batch** out, int32_t n_chains, const int32_t* total_sites, const double* beta,
                     const double* c1);
int qgb_batch_destroy(qgb_batch* b);
int qgb_batch_info(const qgb_batch* b, int32_t* n_chains, int64_t* total_site_count);
/* Hot start of every chain: GaugeField.set_rand(rs_c, sigma, n_step) (qcd-utils.cpp:71-92). */
int qgb_batch_set_rand(qgb_batch* b, const uint32_t* rs, double sigma, int32_t n_step);
/* One trajectory of every chain from its current state: momenta from rs_momentum
 * (sigma 1), molecular dynamics in FP64 (mixed = 0) or FP32 (mixed = 1, FP64
 * re-unitarisation every reunit_interval steps), FP64 Hamiltonians; writes the
 * n_chains values of delta_h and keeps the proposals until qgb_batch_accept.
 * use_graph != 0 records / replays the trajectory as a CUDA graph. */
int qgb_batch_trajectory(qgb_batch* b, const uint32_t* rs_momentum, int32_t n_step, double md_time,
                         int32_t integrator, int32_t mixed, int32_t reunit_interval, int32_t use_graph,
                         double* delta_h);
/* run_hmc_pure_gauge (hmc.pyx:190-216) for every chain at once: rs holds each
 * chain's RngState, split by `traj`, by "set_rand_gauge_momentum" for the
 * momenta and by "metropolis_accept" for the Metropolis draw (Python-API
 * semantics, hmc.pyx:139-155); writes delta_h and the accept flags, and
 * updates every accepted chain (every chain if always_accept). */
int qgb_batch_run_hmc(qgb_batch* b, const uint32_t* rs, int32_t traj, int32_t n_step, double md_time,
                      int32_t integrator, int32_t mixed, int32_t reunit_interval, int32_t always_accept,
                      double* delta_h, int32_t* flags);
/* Replace the state of every chain whose flag is non-zero by its proposal. */
int qgb_batch_accept(qgb_batch* b, const int32_t* flags);
/* gf_avg_plaq of every chain. */
int qgb_batch_plaq(qgb_batch* b, double* plaq);
/* The batch's own force-kernel autotuner (no counterpart in the reference):
 * times the launch shapes of the batched force (block size and register
 * budget; 4 shapes) on the batch's current links in `precision` (QGB_F64 for
 * the FP64 form, QGB_F32 for the mixed form's molecular dynamics), `reps`
 * launches each, and keeps the fastest for that precision; returns it and
 * its time per launch.  qgb_batch_set_force_variant picks one by hand. */
int qgb_batch_autotune(qgb_batch* b, int32_t precision, int32_t reps, int32_t* best, double* best_ms);
int qgb_batch_set_force_variant(qgb_batch* b, int32_t precision, int32_t variant);
/* One chain's links in the reference memory image. */
int qgb_batch_download_chain(qgb_batch* b, int32_t chain, double* host);
int qgb_batch_upload_chain(qgb_batch* b, int32_t chain, const double* host);

/* ---- NERSC gauge-configuration files ------------------------------------ */

/* The format of save_gauge_field / load_gauge_field (qcd.h:66-250): ASCII
 * header, then the links as IEEE doubles in the reference site order, first two
 * rows of each link ("4D_SU3_GAUGE"; "4D_SU3_GAUGE_3x3" is also read),
 * big-endian ("IEEE64BIG"; "IEEE64LITTLE" is also read), with the simple
 * checksum (sum of 32-bit words, field-io.h:11-25) and the CRC-32
 * (field-io.h:84-88) in the header.  The *_host functions need no GPU and use
 * host buffers in the reference memory image ([site][mu][3][3] complex128).
 * Null strings take the reference's defaults (GaugeFieldInfo, qcd.h:34-58):
 * ensemble_id "42", ensemble_label "default-ensemble", creator "Qlat", date =
 * now (ctime). */
int qgb_nersc_write_host(const char* path, const double* links, const int32_t total_site[4], double plaq,
                         double link_trace, const char* ensemble_id, const char* ensemble_label, const char* creator,
                         const char* date, double beta, int64_t sequence_num, int64_t* file_size);
/* read_gauge_field_header (qcd.h:94-144).  n_rows: 2, 3, or 0 for an unknown
 * DATATYPE; big_endian: 1, 0, or -1 for an unknown FLOATING_POINT. */
int qgb_nersc_read_header(const char* path, int32_t total_site[4], int32_t* n_rows, int32_t* big_endian, double* plaq,
                          double* link_trace, uint32_t* simple_checksum, uint32_t* crc32);
/* The links of the file (whose lattice must be total_site).  Two-row files
 * leave row 3 zero: unitarize rebuilds it.  checks: bit 0 CRC-32 matches, bit 1
 * simple checksum matches, bit 2 two-row file.  A mismatch is reported, not an
 * error (the reference warns). */
int qgb_nersc_read_host(const char* path, double* links, const int32_t total_site[4], int32_t* checks,
                        int64_t* file_size);
/* Replace save_gauge_field (qcd.h:146-181; GaugeField.save, qcd.pyx:55-60): the
 * header's plaquette and link trace are computed from gf. */
int qgb_save_gauge_field(const qgb_field* gf, const char* path, const char* ensemble_id, const char* ensemble_label,
                         const char* creator, double beta, int64_t sequence_num, int64_t* file_size);
/* Replace load_gauge_field (qcd.h:183-250; GaugeField.load, qcd.pyx:62-67): gf
 * must have the file's lattice (qgb_nersc_read_header gives it); two-row links
 * are unitarized on the GPU. */
int qgb_load_gauge_field(qgb_field* gf, const char* path, int32_t* checks, int64_t* file_size);

/* ---- flowed HMC with masked invertible flows (flowed-hmc.h) --------------- */

/* FlowStepInfo (flowed-hmc.h:26-41): flow the links U_mu(x) of the sites of
 * mask 1 or 2 (even/odd sites for flow_size 1; even/odd 2^4 blocks for
 * flow_size 2) with step epsilon, by the plaquette staple (flow_size 1) or the
 * staple of the rectangles whose short edge is the link (flow_size 2).  Lattice
 * extents must be multiples of 2 * flow_size.  FP64 fields only. */
typedef struct {
  int32_t mask;
  int32_t mu;
  double epsilon;
  int32_t flow_size;
} qgb_flow_step;
/* mk_flow_info_step(rs, epsilon) (two_eps = 0) or mk_flow_info_step(rs,
 * epsilon, epsilon2) (two_eps = 1) (flowed-hmc.cpp:21-69): the steps in the
 * reference's order, including its random_permute; out holds up to 16. */
int qgb_flow_info_step(const uint32_t rs[24], double epsilon, double epsilon2, int32_t two_eps, qgb_flow_step* out,
                       int32_t* n_out);
/* gf_flow(gf, gf0, fi) / gf_flow_inv(gf, gf1, fi) (flowed-hmc.cpp:540-594). */
int qgb_gf_flow(qgb_field* gf, const qgb_field* gf0, const qgb_flow_step* steps, int32_t n);
int qgb_gf_flow_inv(qgb_field* gf, const qgb_field* gf1, const qgb_flow_step* steps, int32_t n);
/* gf_flow_and_ln_det_node (flowed-hmc.cpp:1257-1299): gf = flowed gf0, ln_det
 * = sum of ln det of the flow's Jacobian. */
int qgb_gf_flow_and_ln_det_node(qgb_field* gf, const qgb_field* gf0, const qgb_flow_step* steps, int32_t n,
                                double* ln_det);
/* gf_hamilton_flowed (flowed-hmc.cpp:1301-1321): the gauge action of the flowed
 * field and ln det; the flowed-HMC action is flowed_action - ln_det. */
int qgb_gf_hamilton_flowed_node(const qgb_field* gf0, double beta, double c1, const qgb_flow_step* steps, int32_t n,
                                double* flowed_action, double* ln_det);
/* set_gm_force_flowed (with_det = 1, flowed-hmc.cpp:1500-1509), or the force of
 * the flowed field propagated without the determinant term (with_det = 0,
 * set_gm_force_flowed_no_det of set_gm_force of the flowed field). */
int qgb_set_gm_force_flowed(qgb_field* gm_force, const qgb_field* gf0, double beta, double c1,
                            const qgb_flow_step* steps, int32_t n, int32_t with_det);
/* set_gm_force_flowed_no_det (flowed-hmc.cpp:1511-1520): gm_force_pre, a force
 * on the flowed field, propagated back through the steps to gf0 without the
 * determinant term. */
int qgb_set_gm_force_flowed_no_det(qgb_field* gm_force, const qgb_field* gm_force_pre, const qgb_field* gf0,
                                   const qgb_flow_step* steps, int32_t n);

/* ---- topology measurement: flows and site fields (instanton_map.py,
 * qcd.cpp:33-62, 295-341, 391-414, wilson-flow.cpp:164-236) ----------------- */

#define QGB_FLOW_TOPO_C1 0       /* gf_wilson_flow_step with the action's c1 (Wilson 0, Iwasaki -0.331, DBW2 -1.4008) */
#define QGB_FLOW_TOPO_SHRINK 1   /* plaquette weight 0.005 / (1 - p + 0.005) + 0.5 */
#define QGB_FLOW_TOPO_FREEZE 2   /* 1 - p */
#define QGB_FLOW_TOPO_LOCALIZE 3 /* 0.002 / (1 - p + 0.002) + 50 (1 - p) */
#define QGB_FLOW_TOPO_PRESERVE 4 /* max(1, 50 (1 - p)) */
#define QGB_FLOW_INTEGRATOR_EULER 0
#define QGB_FLOW_INTEGRATOR_RUNGE_KUTTA 1

/* gf_plaq_field (qcd.cpp:295-341; qcd.pyx:209-213): f_plaq, an FP64 real field
 * of multiplicity 6, gets Re tr P / 3 of the plaquettes at each site in the
 * planes (0,1) (0,2) (0,3) (1,2) (1,3) (2,3). */
int qgb_gf_plaq_field(qgb_field* f_plaq, const qgb_field* gf);
/* gf_energy_density_dir_field (wilson-flow.cpp:53-95; wilson_flow.pyx:49-63):
 * per site and plane (planes as in qgb_gf_plaq_field) -Re tr(G G), G the
 * traceless anti-Hermitian part of the clover; the six sum to
 * gf_energy_density_field.  fd: FP64 real, multiplicity 6. */
int qgb_gf_energy_density_dir_field(qgb_field* fd, const qgb_field* gf);
/* gf_avg_wilson_loop_normalized_tr(gf, l, t) (qcd-utils.cpp:359-400; qcd.pyx:250-254):
 * Re tr / 3 of the l x t Wilson loop (l links along a spatial direction, t along
 * direction 3), averaged over the sites and the three spatial directions. */
int qgb_gf_avg_wilson_loop_normalized_tr(const qgb_field* gf, int32_t l, int32_t t, double* out);
/* topology_charge_5 (qcd.cpp:376-389): the lattice sum of the 5-loop improved
 * charge density (same as qgb_gf_topology). */
int qgb_topology_charge_5(const qgb_field* gf, double* out);
/* clf_plaq_action_density_field (spatial = 0) / clf_spatial_plaq_action_density_field
 * (spatial = 1) (qcd.cpp:33-62, 391-414; topology.pyx:26-75): per site, sum over
 * the planes (spatial: (0,1) (0,2) (1,2)) of 1 - Re tr C / 3, C the clover
 * average of the four plaquettes with a corner at the site; paf: FP64 real,
 * multiplicity 1. */
int qgb_gf_plaq_action_density_field(qgb_field* paf, const qgb_field* gf, int32_t spatial);
/* set_plaq_flow_z (wilson-flow.cpp:164-236; gf_plaq_flow_force, wilson_flow.pyx:65-75):
 * the Wilson-flow force with each plaquette weighted by plaq_factor (FP64 real,
 * multiplicity 6, planes as in qgb_gf_plaq_field). */
int qgb_set_plaq_flow_z(qgb_field* z, const qgb_field* gf, const qgb_field* plaq_factor);
/* gf_flow_topo(gf, step_size, flow_type, integrator) (instanton_map.py:91-191):
 * QGB_FLOW_TOPO_C1 takes one gf_wilson_flow_step with c1 and the integrator;
 * the plaquette-weighted kinds take one Euler step of step_size / norm along the
 * weighted force, norm the weight's extreme over the lattice.  advance (may be
 * NULL) = the flow time taken, step_size / norm. */
int qgb_gf_flow_topo(qgb_field* gf, double step_size, int32_t flow_kind, double c1, int32_t integrator,
                     double* advance);
/* glb_min / glb_max of each component of a real field (either output may be
 * NULL; each holds multiplicity values). */
int qgb_field_glb_min_max(const qgb_field* f, double* mins, double* maxs);
/* glb_sum_tslice (field_base.pyx:750-762): out[t * multiplicity + m] = sum over
 * the sites with coordinate t in direction t_dir of component m (real field). */
int qgb_field_glb_sum_tslice(const qgb_field* f, int32_t t_dir, double* out);
/* f = |f| entrywise (real field). */
int qgb_field_abs(qgb_field* f);

/* ---- field-accelerated HMC: per-link masses and dual momenta (hmc.h:20-80) */

/* A mass field is an FP64 real field of multiplicity 4 (Field<RealD>, one mass
 * per link); +inf freezes a link's momentum at zero.  gm moves a link from the
 * left, gm_dual from the right; momenta and gauge fields share one lattice and
 * precision. */
/* set_rand_gauge_momentum(gm, mf, rs) (hmc.cpp:121-149; GaugeMomentum.set_rand_fa,
 * hmc.pyx:51-63): unit-sigma draw, then gm_mu(x) *= sqrt(mf_mu(x)), zero where
 * the mass is +inf. */
int qgb_set_rand_gauge_momentum_fa(qgb_field* gm, const qgb_field* mf, const uint32_t rs[24]);
/* gm_hamilton_node(gm, mf) (hmc.cpp:175-201; gm_hamilton_node_fa, hmc.pyx:65-66):
 * sum of (-1/2 tr gm^2) / mf over the links. */
int qgb_gm_hamilton_node_fa(const qgb_field* gm, const qgb_field* mf, double* out);
/* gf_evolve(gf, gm, mf, dt) (hmc.cpp:350-372; gf_evolve_fa, hmc.pyx:77-78):
 * U = unitarize(exp(dt / mf P) U). */
int qgb_gf_evolve_fa(qgb_field* gf, const qgb_field* gm, const qgb_field* mf, double step_size);
/* gf_evolve_dual(gf, gm_dual, dt) (hmc.cpp:330-348; hmc.pyx:74-75):
 * U = unitarize(U exp(-dt P)). */
int qgb_gf_evolve_dual(qgb_field* gf, const qgb_field* gm_dual, double step_size);
/* gf_evolve_dual(gf, gm_dual, mf_dual, dt) (hmc.cpp:374-396; gf_evolve_fa_dual,
 * hmc.pyx:80-81): U = unitarize(U exp(-dt / mf_dual P)). */
int qgb_gf_evolve_fa_dual(qgb_field* gf, const qgb_field* gm_dual, const qgb_field* mf_dual, double step_size);
/* set_gm_force_dual (hmc.cpp:492-513): gm_force_dual = -U^+ gm_force U
 * (output distinct from both inputs). */
int qgb_set_gm_force_dual(qgb_field* gm_force_dual, const qgb_field* gf, const qgb_field* gm_force);
/* project_gauge_transform (hmc.cpp:515-589): subtract the gauge-transformation
 * motion from gm and gm_dual; change_qnorm = qnorm of the per-site average it
 * removed / total volume (NULL: not computed, and the call does not
 * synchronise). */
int qgb_project_gauge_transform(qgb_field* gm, qgb_field* gm_dual, const qgb_field* mf, const qgb_field* mf_dual,
                                double* change_qnorm);
/* set_gauge_transform_momentum (hmc.cpp:591-626): gm_mu(x) = gtm(x),
 * gm_dual_mu(x) = gtm(x + mu); gtm a color-matrix field of multiplicity 1. */
int qgb_set_gauge_transform_momentum(qgb_field* gm, qgb_field* gm_dual, const qgb_field* gtm);
/* dot_gauge_momentum (hmc.cpp:628-645): f_mu(x) = Re tr(gm1_mu(x)^+ gm2_mu(x)),
 * f an FP64 real field of multiplicity 4. */
int qgb_dot_gauge_momentum(qgb_field* f, const qgb_field* gm1, const qgb_field* gm2);
/* set_u_rand / set_g_rand (core.h:1585-1636; FieldRealD.set_rand / set_rand_g,
 * field_types.pyx.in:194-200): per site the state rs.newtype(site index), one
 * draw per real of the site in memory order.  rs must be untyped. */
int qgb_field_set_u_rand(qgb_field* f, const uint32_t rs[24], double upper, double lower);
int qgb_field_set_g_rand(qgb_field* f, const uint32_t rs[24], double center, double sigma);
/* Real field: every entry = value (set_unit(f, value) of a Field<RealD>); with a
 * selection (n = sites * multiplicity bytes, site-major, nonzero = selected)
 * only the selected entries: `f[sel] = value`. */
int qgb_field_fill(qgb_field* f, double value, const uint8_t* mask, int64_t n);
/* `dst[sel] = src[sel]` with a boolean selection of the (site, component)
 * entries as above; fields of one kind, multiplicity, lattice and precision. */
int qgb_field_set_selected(qgb_field* dst, const qgb_field* src, const uint8_t* mask, int64_t n);

/* ---- time-slab decomposition (the reference's domain decomposition,
 * field-expand.h / hmc.cpp:466-490 refresh_expanded, restricted to the time
 * direction) ------------------------------------------------------------- */

/* A rank holds the slab of T / R time slices it owns plus h halo slices on each
 * side as an ordinary field of extent T / R + 2 h in direction 3.  The halo
 * slices are copied from the neighbouring ranks (pack / unpack below, sent by
 * the caller's communication library); the owned sites are the contiguous
 * local site range [h X Y Z, (h + T / R) X Y Z). */
/* Sums over the local sites [s0, s1) only: gm_hamilton_node, the plaquette and
 * rectangle sums of gf_sum_re_tr_*_node (out[1] = 0 unless rect), and
 * gf_hamilton_node. */
int qgb_gm_hamilton_node_sites(const qgb_field* gm, int64_t s0, int64_t s1, double* out);
int qgb_gf_action_sums_sites(const qgb_field* gf, int32_t rect, int64_t s0, int64_t s1, double out[2]);
int qgb_gf_hamilton_node_sites(const qgb_field* gf, double beta, double c1, int64_t s0, int64_t s1, double* out);
/* set_rand_gauge_momentum / set_g_rand_color_matrix_field with the per-site
 * streams of global site (local site + site_offset). */
int qgb_set_rand_gauge_momentum_sites(qgb_field* gm, double sigma, const uint32_t rs[24], int64_t site_offset);
int qgb_gf_set_rand_sites(qgb_field* gf, const uint32_t rs[24], double sigma, int32_t n_step, int64_t site_offset);
/* Copy the time slices [t0, t0 + nt) of every component of f into a device
 * buffer of qgb_field_tslice_bytes(f, nt) bytes, or back; X Y Z must be a
 * multiple of 32.  Asynchronous on the library stream. */
int qgb_field_tslice_bytes(const qgb_field* f, int32_t nt, int64_t* bytes);
int qgb_field_pack_tslices(const qgb_field* f, int32_t t0, int32_t nt, void* dev);
int qgb_field_unpack_tslices(qgb_field* f, int32_t t0, int32_t nt, const void* dev);

/* ---- four-dimensional domain decomposition (Geometry's node partition and
 * expanded fields: core.h:17-110 GeometryNode / node_site / expansion_left,
 * field-expand.h:116-200 refresh_expanded, hmc.cpp:466-490) --------------- */

/* Make f the domain of one rank of a decomposed lattice of global extents
 * global_site: the rank owns the sites with global coordinates
 * [origin_k, origin_k + dims_k - 2 halo_k) and f holds them with halo_k sites
 * of the neighbouring domains on either side in each direction k (the
 * reference's node_site with expansion_left = expansion_right = halo).  A
 * direction with halo_k = 0 is not cut: f holds all of it (dims_k =
 * global_site_k, origin_k = 0) and wraps periodically.  Then, on f:
 *  - the force (qgb_set_gm_force, the fused kernels of qgb_run_md_hooked) is
 *    evaluated on the owned sites only, reading the halo, which the caller
 *    refreshes before each force (the hook of qgb_run_md_hooked);
 *  - the _node sums (gm_hamilton_node, gf_hamilton_node, the _sites action
 *    sums) are over the owned sites, as the reference's node sums are over
 *    its node's sites;
 *  - the per-site random streams are those of each local site's global
 *    index, so the owned sites draw what a single field of the whole lattice
 *    draws: set_rand draws every local site (the halo sites what their owners
 *    draw), set_rand_gauge_momentum the owned sites only (halo momenta are set
 *    to zero: no force or sum reads them);
 *  - element-wise operations run on every local site;
 *  - qgb_run_md_hooked with the force-gradient integrator needs
 *    refresh_shifted = 1 (the shifted field, too, is evaluated on the owned
 *    sites only);
 *  - qgb_run_hmc_evolve[_mixed], the gradient flow, the clover and 5-loop
 *    charges and gf_avg_plaq refuse it (QGB_ERR_INVALID_ARG).
 * qgb_field_copy copies the domain with the data. */
int qgb_field_set_domain(qgb_field* f, const int32_t global_site[4], const int32_t origin[4],
                         const int32_t halo[4]);
int qgb_field_domain(const qgb_field* f, int32_t* has_domain, int32_t global_site[4], int32_t origin[4],
                     int32_t halo[4]);
/* Copy the local sites [lo_k, lo_k + n_k) of every component of f into a
 * device buffer of qgb_field_box_bytes(f, n) bytes (entry-major: for each
 * component and matrix entry, the box's sites with x fastest), or back: the
 * faces a halo exchange sends.  Asynchronous on the library stream. */
int qgb_field_box_bytes(const qgb_field* f, const int32_t n[4], int64_t* bytes);
int qgb_field_pack_box(const qgb_field* f, const int32_t lo[4], const int32_t n[4], void* dev);
int qgb_field_unpack_box(qgb_field* f, const int32_t lo[4], const int32_t n[4], const void* dev);

/* ---- force-kernel autotuner (no counterpart in the reference) ---------- */

/* The force kernels (set_gm_force and its fused HMC / flow consumers) exist
 * in several launch shapes: threads per block, a register cap through the
 * minimum resident blocks per SM, one or two threads per link, and the site
 * mapping and staple evaluation (0: consecutive sites, one mu per block; 1:
 * each block takes the four links of a compact 4-d tile; 2: as 0 with
 * per-thread neighbour offsets and sign-specialised staple directions; 3: as 2
 * with SU(3) link chains carried as two rows, FP32 only -- FP64 runs 2).  The
 * shape is chosen per (precision, rect): by hand, or by timing them all on a
 * given gauge field. */
int qgb_force_variant_count(int32_t* n);
int qgb_force_variant_info(int32_t variant, int32_t* block_size, int32_t* min_blocks, int32_t* threads_per_link,
                           int32_t* site_map);
int qgb_force_set_variant(int32_t precision, int32_t rect, int32_t variant);
int qgb_force_get_variant(int32_t precision, int32_t rect, int32_t* variant);
/* Time every variant on gf with action coefficient c1 -- `reps` steps of the
 * force-gradient integrator's two force launches (force + link shift, then
 * force + momentum update + link update), each with the variant's own
 * passes -- and select the fastest for gf's precision and (c1 != 0), keeping
 * the current shape unless another is faster by more than 2%; returns the
 * selection and its time per force launch.  Shapes with site map 5 (a precomputed
 * field of two-link products, 16 color matrices per site of scratch) are not
 * timed; qgb_force_set_variant selects them. */
int qgb_autotune_force(const qgb_field* gf, double c1, int32_t reps, int32_t* best, double* best_ms);
/* Time one variant without selecting it. */
int qgb_force_time_variant(const qgb_field* gf, double c1, int32_t variant, int32_t reps, double* ms_per_launch);

/* ---- allocation-free action sums (no counterpart in the reference) ------ */

/* For callers that cannot allocate GPU memory: a host whose device memory
 * belongs to its own pool (a framework's caching allocator, a solver with a
 * fixed memory budget set at start-up), or one that cannot afford the
 * device-wide synchronisation that cudaMalloc / cudaFree may cause while its
 * other streams are busy.  Every other entry point may allocate (the library
 * context, reduction scratch, staging); this one calls no cudaMalloc, cudaFree
 * or allocating library routine.
 *
 * Computes the gauge-action sums of gf_sum_re_tr_plaq_node_no_comm and
 * gf_sum_re_tr_rect_node_no_comm (hmc.cpp:203-252): out_dev[0] = sum over
 * plaquettes of (Re tr P - 3), out_dev[1] = sum over rectangles of
 * (Re tr R - 3) when rect != 0, else 0.  links_dev is a caller-owned device
 * buffer holding the FP64 gauge field in the reference memory image
 * ([site][mu][3][3] complex128, x fastest), 16-byte aligned; out_dev is
 * caller-owned device memory for two doubles, 8-byte aligned.  Work is queued
 * on `stream` (a cudaStream_t; NULL for the legacy default stream) and nothing
 * is synchronised.
 *
 * Limit: at most 2^24 = 16,777,216 sites (e.g. 64^4), each extent in
 * [1, 2^20].  Larger lattices and misaligned pointers are rejected with
 * QGB_ERR_INVALID_ARG (bad extents with QGB_ERR_BAD_GEOMETRY) before anything
 * is launched; so is a call made while an earlier, unrelated CUDA error is
 * pending (QGB_ERR_CUDA; that error is left for its owner).  The scratch is a
 * fixed 1 MiB device array inside the library, which every GPU that loads the
 * library holds until the process exits.  The first call on each device looks
 * up that array's device address (cudaGetSymbolAddress) with the device
 * current.  All calls share
 * the one array and it keeps the last call's partial sums (each call
 * overwrites every entry it reads, so nothing needs to start at zero): calls
 * that overlap on the GPU -- two streams, or two host threads -- race and must
 * be serialised by the caller. */
int qgb_gf_action_sums_noalloc(const double* links_dev, const int32_t total_site[4], int32_t rect, double* out_dev,
                               void* stream);

/* Number of kernels this library has launched since it was loaded. */
int qgb_launch_count(int64_t* out);
/* Number of Gaussian draws whose logarithm could not be proven correctly
 * rounded (expected 0); cumulative since library load. */
int qgb_rng_ambiguous_count(int64_t* out);

#ifdef __cplusplus
}
#endif

#endif /* QLAT_B200_H */
