/*
 * edge_b200: B200-native (sm_100a) tet4 ADER-DG elastic / viscoelastic element update behind a
 * plain C ABI, plus the host-side setup that keeps EDGE's semantics.
 *
 * All functions return 0 on success or a negative edge_b200_status. Arrays are row-major, runs are
 * the fastest dimension of every DOF array: dofsE[nEl][9][B][R], dofsA[nEl][rm][6][B][R], with
 * B = O(O+1)(O+2)/6 element modes and F = O(O+1)/2 face modes for order O.
 * Stress order is xx, yy, zz, xy, yz, xz, followed by the velocities u, v, w.
 *
 * The reference has no FFI for this path: its element update is the C++ template class
 * AderDg<real, nRms, TET4, O, O, nCfr, sparse> (src/impl/seismic/solvers/AderDg.hpp), constructed in
 * src/impl/seismic/setup.inc:265-290 and driven by src/impl/seismic/steps.inc:24-77. Each entry
 * point below names the reference interface it replaces.
 */
#ifndef EDGE_B200_H
#define EDGE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  EDGE_B200_OK = 0,
  EDGE_B200_EINVAL = -1,     /* invalid argument */
  EDGE_B200_ENOMEM = -2,     /* allocation failed (host or device) */
  EDGE_B200_EDEVICE = -3,    /* CUDA error */
  EDGE_B200_ETIMEOUT = -4,   /* a bounded device wait gave up */
  EDGE_B200_ENOTSUP = -5,    /* configuration not compiled in (order / runs / mechanisms) */
  EDGE_B200_EMESH = -6,      /* inconsistent or degenerate mesh */
  EDGE_B200_ENOTFOUND = -7,  /* point not inside the mesh */
  EDGE_B200_EOVERFLOW = -8,  /* receiver buffer full */
  EDGE_B200_ESCRATCH = -9    /* problem too large for the static scratch of edge_b200_step_noalloc */
} edge_b200_status;

/* per element-face boundary types (t_spTypeElastic, src/impl/seismic/const.inc:143-149);
 * EDGE_FACE_PERIODIC is only a mesh-builder request: periodic faces become inner faces whose
 * neighbour sits on the opposite side of the box (PERIODIC = 106 in the reference) */
enum { EDGE_FACE_INNER = 0, EDGE_FACE_FREE_SURFACE = 1, EDGE_FACE_OUTFLOW = 2, EDGE_FACE_PERIODIC = 3 };

/* ============================== host setup (EDGE semantics) ================================== */

typedef struct edge_mesh edge_mesh;

/* Box [0,ext]^3 of nx*ny*nz cubes, each split into 6 congruent tets along its main diagonal;
 * interior vertices jittered by seeded uniform +-jitter*h per coordinate (tets with detJ <= 0 are
 * redrawn). The top face (z = ext[2]) gets bc_top, all other boundary faces bc_sides
 * (EDGE_FACE_FREE_SURFACE or EDGE_FACE_OUTFLOW; both EDGE_FACE_PERIODIC for a periodic box with at
 * least 2 cubes per direction). Vertex / face / neighbour conventions follow
 * EDGE-V: tools/edge_v/src/mesh/Mesh.cpp:288-375 (sorting), geom/Tet4.cpp:80-112 (orientation),
 * geom/Tet4.cpp:114-229 and geom/Generic.cpp:92-116 (neighbour vertex / face ids),
 * mesh/Mesh.cpp:763-841 with geom/Tria3.cpp:48-120 (normals, tangents). */
int edge_mesh_box(int nx, int ny, int nz, const double ext[3], double jitter, uint64_t seed,
                  int bc_top, int bc_sides, edge_mesh **out);
/* Tet4 mesh from vertices ve[n_ve][3] and elements el_ve[n_el][4] (any vertex order), e.g. as read
 * from a gmsh file (EDGE-V io/Gmsh.cpp:120-251), with the same EDGE-V conventions as
 * edge_mesh_box. Boundary faces bf_ve[n_bf][3] carry the reference's physical-group tags bf_tag
 * (101 free surface, 105 outflow, src/impl/seismic/const.inc:144-146; any other tag, periodic 106
 * included, gives EDGE_B200_ENOTSUP); boundary faces not listed get default_type
 * (EDGE_FACE_FREE_SURFACE / EDGE_FACE_OUTFLOW, or -1 to reject the mesh with EDGE_B200_EMESH);
 * tags on inner faces are ignored. reorder != 0 sorts the elements along a Z-order curve of their
 * centroids (locality of the neighbour gathers); el_perm[n_el] (may be NULL) receives the input
 * index of each mesh element. Faces shared by more than two elements or degenerate elements give
 * EDGE_B200_EMESH. */
int edge_mesh_from_arrays(int64_t n_ve, const double *ve, int64_t n_el, const int64_t *el_ve, int64_t n_bf,
                          const int64_t *bf_ve, const int32_t *bf_tag, int default_type, int reorder,
                          int64_t *el_perm, edge_mesh **out);
int edge_mesh_sizes(const edge_mesh *m, int64_t *n_ve, int64_t *n_fa, int64_t *n_el);
/* Any output pointer may be NULL. Shapes: ve[nVe][3], el_ve[nEl][4], el_fa[nEl][4],
 * fa_el[nFa][2] (-1 = none), fa_normal[nFa][3], fa_tangent[nFa][2][3], fa_area[nFa],
 * fa_type[nFa], el_vol[nEl], el_india[nEl], el_fa_el[nEl][4] (-1 = none),
 * fid_el_fa_el / vid_el_fa_el / el_fa_type [nEl][4]. Replaces mesh::EdgeV getters
 * (src/mesh/EdgeV.h:166-395). */
int edge_mesh_arrays(const edge_mesh *m, double *ve, int64_t *el_ve, int64_t *el_fa,
                     int64_t *fa_el, double *fa_normal, double *fa_tangent, double *fa_area,
                     uint8_t *fa_type, double *el_vol, double *el_india, int32_t *el_fa_el,
                     uint8_t *fid_el_fa_el, uint8_t *vid_el_fa_el, uint8_t *el_fa_type);
void edge_mesh_free(edge_mesh *m);

/* Elastic star matrices starE[nEl][3][24] (AderDgInit::initStar, AderDgInit.hpp:129-174 with
 * Elasticity::star, Elasticity.cpp:167-301). lam/mu must already be the unrelaxed values when
 * attenuation is on (AderDgInit::initSrcA, AderDgInit.hpp:91-117). */
int edge_setup_star(const edge_mesh *m, const double *rho, const double *lam, const double *mu,
                    double *star_e);
/* Anelastic star matrices starA[nEl][3][9] (ViscoElasticity::star, ViscoElasticity.cpp:233-316). */
int edge_setup_star_anelastic(const edge_mesh *m, double *star_a);
/* Flux solvers fsE[2][nEl][4][81] and, if n_rms > 0, fsA[2][nEl][4][54]
 * (AderDgInit::initFs / setUpFs, AderDgInit.hpp:288-665). */
int edge_setup_flux_solvers(const edge_mesh *m, int n_rms, const double *rho, const double *lam,
                            const double *mu, double *fs_e, double *fs_a);
/* Relaxation frequencies, 2n-1 values (ViscoElasticity::frequencies, ViscoElasticity.h:168-183). */
int edge_setup_frequencies(int n_rms, double freq_cen, double freq_rat, double *freqs);
/* Per element: anelastic source matrices srcA[nEl][rm][12]; lam/mu are overwritten by the
 * unrelaxed Lame parameters (AderDgInit::initSrcA, ViscoElasticity::src,
 * ViscoElasticity.h:379-508 and ViscoElasticity.cpp:30-176). omega[rm] = freqs[2m]
 * (AderDg.hpp:248-258). */
int edge_setup_attenuation(int n_rms, double freq_cen, double freq_rat, int64_t n_el,
                           const double *qp, const double *qs, double *lam, double *mu,
                           double *src_a, double *omega);
/* Least-squares anelastic coefficients of one wave type (ViscoElasticity::anelasticCoeffPs). */
int edge_setup_anelastic_coeffs(int n_rms, double quality, const double *freqs, double *coeffs);
/* Unrelaxed Lame parameters (ViscoElasticity::elasticLame). */
int edge_setup_elastic_lame(int n_rms, double freq_ref, const double *freqs,
                            const double *coeffs_kappa, const double *coeffs_mu, double lam_phase,
                            double mu_phase, double *lam_el, double *mu_el);
/* CFL time step: min over elements of 0.5 * inDia / vp / (2O-1) (common.hpp:84-133). */
int edge_setup_dt_cfl(const edge_mesh *m, int order, const double *rho, const double *lam,
                      const double *mu, double *dt_min);
/* Per-element CFL time steps dt_el[nEl] (the quantity edge_setup_dt_cfl minimises). */
int edge_setup_dt_cfl_el(const edge_mesh *m, int order, const double *rho, const double *lam,
                         const double *mu, double *dt_el);
/* Rate-2 LTS time groups el_tg[nEl] of EDGE-V (time/Groups.cpp:84-100 setElTg, 47-82
 * normalizeElTgs): with ts = dt_el / min(dt_el), an element joins the first group g with
 * ts < fun_dt * 2^(g+1) (the last of n_groups takes the rest); groups are then lowered until face
 * neighbours differ by at most one. Group g steps with fun_dt * min(dt_el) * 2^g. *n_norm
 * (may be NULL) receives the number of lowerings. */
int edge_setup_time_groups(const edge_mesh *m, const double *dt_el, int n_groups, double fun_dt, uint8_t *el_tg,
                           int64_t *n_norm);
/* Locates n points; per point the element, reference coordinates and basis values
 * basis[n][B]. scale_mass_jac != 0 multiplies by M^-1 and divides by detJ as point sources do
 * (PointSources::initBasisEvals, PointSources.hpp:388-509); 0 gives plain basis values as
 * receivers use (io/Receivers.cpp:33-180). */
int edge_setup_locate(const edge_mesh *m, int order, int n, const double *xyz, int64_t *el,
                      double *ref, double *basis, int scale_mass_jac);
/* Basis of the given order evaluated at reference coordinates (dg::Basis::evalBasis). */
int edge_setup_eval_basis(int order, const double ref[3], double *vals);
/* Face-aligned <-> xyz transforms of the 9 quantities (common::setupTrafo3d / setupTrafoInv3d,
 * src/impl/seismic/common.hpp:314-343) and the Godunov middle states (Elasticity::fs 3D,
 * Elasticity.cpp:372-441; ViscoElasticity::fs 3D). Exposed for parity tests. */
int edge_setup_trafo(const double n[3], const double s[3], const double t[3], double *t_mat,
                     double *t_inv);
int edge_setup_fs_pair(double rho_l, double rho_r, double lam_l, double lam_r, double mu_l,
                       double mu_r, const double n[3], const double s[3], const double t[3],
                       int free_surface, double *fs_el, double *fs_er, double *fs_al,
                       double *fs_ar);

/* ================================ device element update ======================================= */

typedef struct edge_b200_ctx edge_b200_ctx;

typedef struct {
  int order;     /* O: 2..6 */
  int n_runs;    /* R fused forward runs: 1, 2, 4, 8, 16 */
  int n_rms;     /* relaxation mechanisms: 0..3 */
  int precision; /* 64: plain FP64 path; 32: FP32 fused-run path (element data kept in FP64 on host) */
  void *stream;  /* cudaStream_t; NULL = the legacy default stream */
  int device;    /* CUDA device ordinal */
} edge_b200_cfg;

/* Creates the device context for n_el elements (replaces the AderDg constructor,
 * AderDg.hpp:225-312, and the DOF allocations of data::Internal::initDense, Internal.hpp:559-568). */
int edge_b200_create(const edge_b200_cfg *cfg, int64_t n_el, edge_b200_ctx **out);
int edge_b200_destroy(edge_b200_ctx *ctx);
/* Connectivity per element face (the elFaEl / fIdElFaEl / vIdElFaEl / faChars arguments of
 * AderDg::neigh, AderDg.hpp:553-567). el_fa_el = -1 where there is no neighbour. */
int edge_b200_upload_mesh(edge_b200_ctx *ctx, const int32_t *el_fa_el, const uint8_t *fid_el_fa_el,
                          const uint8_t *vid_el_fa_el, const uint8_t *el_fa_type);
/* FP64 element data: starE[nEl][3][24], fsE[2][nEl][4][81]; with mechanisms also
 * starA[nEl][3][9], srcA[nEl][rm][12], fsA[2][nEl][4][54], omega[rm] (the m_starE / m_fsE /
 * m_starA / m_srcA / m_fsA members the AderDg constructor builds). */
int edge_b200_upload_element_data(edge_b200_ctx *ctx, const double *star_e, const double *fs_e,
                                  const double *star_a, const double *src_a, const double *fs_a,
                                  const double *omega);
/* Element data (star matrices, flux solvers, anelastic data, relaxation frequencies) borrowed from
 * another context of the same mesh size, mechanisms and device instead of uploaded: the two share
 * one device copy, src must outlive dst, and a later edge_b200_upload_element_data on dst gives dst
 * arrays of its own again. Used by pools of one mesh at different orders or run counts (element
 * data do not depend on either). No counterpart in the reference (one solver per mesh). */
int edge_b200_share_element_data(edge_b200_ctx *dst, const edge_b200_ctx *src);
/* DOFs in the context precision (double for 64, float for 32); dofs_a may be NULL without
 * mechanisms. */
int edge_b200_upload_dofs(edge_b200_ctx *ctx, const void *dofs_e, const void *dofs_a);
int edge_b200_download_dofs(edge_b200_ctx *ctx, void *dofs_e, void *dofs_a);
/* Asynchronous forms for host-resident DOFs that change every step: the copies run on two copy
 * streams of the context (one per direction) and overlap each other and the kernels, ordered with
 * the step kernels on the device by events. Uploads move chunks of about 1 GB through a ring of
 * three staging slots, so each chunk's layout kernel overlaps the next chunk's copy; downloads
 * convert the rows at once into one of two full-size buffers (allocated on first use), so the next
 * step need not wait for the previous download's copy. Host buffers must be pinned (cudaHostAlloc / cudaHostRegister)
 * and left alone until edge_b200_sync returns. edge_b200_join_transfers(ctx, 0) makes the context
 * stream wait (on the device) for the last download, e.g. before an event that should cover it;
 * (ctx, 1) makes the copy streams start after the work the context stream holds now. The
 * synchronous forms do not wait for the copy streams: join (or sync) before mixing them. No
 * counterpart in the reference (its DOFs are host arrays). */
int edge_b200_upload_dofs_async(edge_b200_ctx *ctx, const void *dofs_e, const void *dofs_a);
int edge_b200_download_dofs_async(edge_b200_ctx *ctx, void *dofs_e, void *dofs_a);
int edge_b200_join_transfers(edge_b200_ctx *ctx, int after_stream);
/* Sets the DOFs of one fused run only (the other runs keep theirs): dofs_e [nEl][9][B] and, with
 * mechanisms, dofs_a [nEl][rm][6][B] in the context precision; NULL sets that run to zero. Used
 * when a run slot is handed to a new simulation while the others continue (no counterpart in the
 * reference, whose fused runs start and end together). */
int edge_b200_set_run_dofs(edge_b200_ctx *ctx, int run, const void *dofs_e, const void *dofs_a);
/* Copies fused run src_run of context src into run dst_run of context dst on the device (elastic
 * and anelastic DOFs; the other runs of dst keep theirs), on dst's stream after the work queued on
 * src's stream. Both contexts must have the same mesh size, order, mechanisms, precision and
 * device; their numbers of fused runs may differ. Used to move running simulations between pools
 * of different run counts (no counterpart in the reference, whose fused runs start and end
 * together). */
int edge_b200_copy_run(edge_b200_ctx *dst, int dst_run, edge_b200_ctx *src, int src_run);
/* Keep the time-integrated DOFs tDofs[nEl][9][B][R] of each local step (the tDofs[0] of
 * steps.inc) in device memory (allocated on first enable; off by default, which saves their HBM
 * writes), and copy the last step's to the host (EDGE_B200_EINVAL unless kept). */
int edge_b200_keep_tdofs(edge_b200_ctx *ctx, int enable);
int edge_b200_download_tdofs(edge_b200_ctx *ctx, void *tdofs);
/* Point sources sorted by (element, run); source s adds
 *   int_t^{t+dt} series_s * scal[s][q] * b_eval[s][md]  to run run[s] of element el[s]
 * (PointSources::apply, PointSources.hpp:887-931, with Series<1>::integrate, Series.hpp:59-134).
 * Series s: n_pts[s] samples at ts[ts_off[s]...], start t0[s], spacing dt[s]. */
int edge_b200_set_sources(edge_b200_ctx *ctx, int n, const int64_t *el, const int32_t *run,
                          const double *scal, const double *b_eval, const double *t0,
                          const double *dt, const int64_t *ts_off, const int64_t *n_pts,
                          int64_t n_ts, const double *ts);
/* Several simulations of one configuration (order, fused runs, mechanisms, precision, relaxation
 * frequencies) merged into one context: their meshes side by side as disjoint element ranges, each
 * padded to a multiple of the 32 / n_runs elements of a kernel group, so that one persistent launch
 * per kernel steps all of them. edge_b200_set_group_dt gives every element group its own time
 * step (dt_group[ceil(nEl / (32 / n_runs))]; NULL: the step's dt for all; GTS only), and
 * edge_b200_set_source_clocks every point source its own clock (in the order of
 * edge_b200_set_sources; NULL: the step's time): step k after the call integrates source i over
 * [t0[i] + k dt[i], t0[i] + (k + 1) dt[i]]. Simulations that stop are dropped by ordering them last
 * and lowering edge_b200_set_active_elements to the end of the ones still running: the kernels then
 * step elements [0, n_active) only (multi-step calls still fuse their neighbour steps; the elements
 * behind must share no face with those before) and sources beyond are skipped. No counterpart in
 * the reference (one solver per process; uneven batches of one configuration family in one
 * launch). */
int edge_b200_set_group_dt(edge_b200_ctx *ctx, const double *dt_group);
int edge_b200_set_source_clocks(edge_b200_ctx *ctx, const double *t0, const double *dt);
int edge_b200_set_active_elements(edge_b200_ctx *ctx, int64_t n_active);
/* Receivers grouped by element (el ascending; equal elements adjacent), basis[n][B] plain basis
 * values, first output time t_first and sampling period (Receivers::init / getRecvTimeRel /
 * writeRecvAll, io/Receivers.cpp:33-290). Up to max_buf samples are buffered per receiver. */
int edge_b200_set_receivers(edge_b200_ctx *ctx, int n, const int64_t *el, const double *basis,
                            double t_first, double period, int max_buf);
/* Restarts receiver sampling at t_first with an empty buffer, keeping receivers and buffer
 * allocation (no device allocation, so other streams keep running). */
int edge_b200_rewind_receivers(edge_b200_ctx *ctx, double t_first);
/* n_steps GTS steps from time t with step dt: local -> sources -> neighbour
 * (TimeGroupStatic::computeStep, src/time/TimeGroupStatic.cpp:113-127, steps.inc:24-77). */
int edge_b200_step(edge_b200_ctx *ctx, double t, double dt, int n_steps);
/* Error norms of the device solution (InitialDofs::err, src/setups/InitialDofs.hpp:277-373, and
 * the reduction of src/impl/seismic/fin.inc:23-64): per quantity and run, the L1, L2 and Linf norms
 * of (DG solution - reference) over the owned elements at time t, with quadrature points
 * qp_xi[n_qp][3] on the unit tet, weights qp_w[n_qp] and basis values qp_basis[n_qp][B] chosen by the
 * caller (the reference uses its order+1 rule). The reference solution is a sum of plane waves
 * (the family of EDGE's convergence setups; its exprtk expressions are not evaluated on the
 * device): waves[n_waves][15] = k[3], omega, phase, amp[9], run (-1 = every run), adding
 * amp[q] * sin(k . x - omega t + phase) to quantity q. Outputs l1 / l2 / linf [9][R] (host, any may
 * be NULL). Needs edge_b200_upload_geometry (element vertex coordinates [nEl][4][3], FP64). */
int edge_b200_upload_geometry(edge_b200_ctx *ctx, const double *el_ve_crds);
int edge_b200_error_norms(edge_b200_ctx *ctx, double t, int n_waves, const double *waves, int n_qp,
                          const double *qp_xi, const double *qp_w, const double *qp_basis, double *l1, double *l2,
                          double *linf);
/* Wave-field snapshot (io::WaveField / io::Vtk::write, src/io/Vtk.cpp:83-121): the mode-0
 * coefficient of every element, quantity and run, as FP32 in the reference's output order
 * out[run][quantity][element] ([n_runs][9][nEl]); the DOFs stay on the device. */
int edge_b200_wavefield(edge_b200_ctx *ctx, float *out);
/* Halo exchange between the halves of a step (EDGE's MPI path: the local step packs the
 * face-projected time integrals of the send faces, AderDg.hpp:419-473, the neighbour step reads
 * the received ones, 675-684). With edge_b200_set_owned the kernels update only the elements
 * [0, n_owned); the elements behind are ghosts whose face projections arrive by
 * edge_b200_unpack_faces. edge_b200_step_phase runs one step's first half (phase 0: receivers,
 * local, sources) or second half (phase 1: neighbour). pack / unpack move the face blocks
 * [9][R][GF] of n face slots (slots[i] = element * 4 + face, a device int32 array) to / from the
 * device buffer out / in ([n] blocks of edge_b200_face_block_bytes each, GF = F rounded up to 16
 * bytes), ordered on the context stream; slots outside the mesh are skipped. Time groups need the
 * whole mesh owned. To overlap the exchange with work, as the reference's inner / send regions do
 * (src/impl/seismic/setup.inc:337-399), number the owned elements with a face neighbour in another
 * part first and give their count to edge_b200_set_send_count: phase 2 runs the receivers and the
 * local step of those [0, n_send), phase 3 the local step of the others [n_send, n_owned) and the
 * sources; phases 2 and 3 together equal phase 0, and the send faces can be packed and sent between
 * them. */
int edge_b200_set_owned(edge_b200_ctx *ctx, int64_t n_owned);
int edge_b200_set_send_count(edge_b200_ctx *ctx, int64_t n_send);
int edge_b200_step_phase(edge_b200_ctx *ctx, double t, double dt, int phase);
int64_t edge_b200_face_block_bytes(const edge_b200_ctx *ctx);
int edge_b200_pack_faces(edge_b200_ctx *ctx, int n, const int32_t *slots, void *out);
int edge_b200_unpack_faces(edge_b200_ctx *ctx, int n, const int32_t *slots, const void *in);
/* Rate-2 local time stepping (EDGE's LTS: TimeGroupStatic, src/time/TimeGroupStatic.cpp:46-111,
 * the work-region dependencies of src/impl/seismic/inc/time/man_sched.inc:37-206 and the LTS
 * branches of AderDg::local / ::neigh, AderDg.hpp:384-417 and 620-674). The mesh elements must be
 * ordered by time group: group g holds the elements [group_first[g], group_first[g+1]) and steps
 * with dt_fun * 2^g; face neighbours differ by at most one group (edge_setup_time_groups gives
 * such groups; sort the elements by group before building the context). Elements at group
 * interfaces get device buffers for the face projections of their summed and half-step time
 * integrals. EDGE_B200_ENOTSUP when n_groups > 1 and the configuration has no LTS kernels (the
 * half-step integral needs shared memory the largest FP64 orders lack). */
int edge_b200_set_time_groups(edge_b200_ctx *ctx, int n_groups, const int64_t *group_first);
/* n_cycles steps of the largest group starting at t: per cycle 2^(n_groups-1) fundamental steps;
 * at fundamental step k every group with k % 2^g == 0 samples its receivers and runs local +
 * sources over [t_k, t_k + dt_fun 2^g), then every group whose step ends ((k+1) % 2^g == 0) runs
 * neigh; t_k = t + k dt_fun counted from t. The first step of each rate-2 pair of a group starts the
 * two-step sums. Receivers keep one clock per group (counts per receiver in read_receivers). */
int edge_b200_step_lts(edge_b200_ctx *ctx, double t, double dt_fun, int n_cycles);
/* Receiver samples buf[n][max_buf][9][R] (FP64), their times buf_time[n][max_buf], counts[n]. */
int edge_b200_read_receivers(edge_b200_ctx *ctx, double *buf, double *buf_time, int32_t *counts);
/* Waits for all work of the context's stream. */
int edge_b200_sync(edge_b200_ctx *ctx);
/* Device pointers of the resident DOF arrays (for callers that keep data on the device). They use
 * the kernels' row layout, not the reference layout: dofsE [nEl][9][R][GB], dofsA [nEl][rm*6][R][GB],
 * tdofs like dofsE, with GB = B rounded up to 16 bytes (a multiple of 4 floats / 2 doubles). */
int edge_b200_device_dofs(edge_b200_ctx *ctx, void **dofs_e, void **dofs_a, void **tdofs);
/* Kernel launches issued by the last edge_b200_step call. */
int64_t edge_b200_last_launches(const edge_b200_ctx *ctx);
/* Per-kernel timing with CUDA events recorded on the context's stream around every launch
 * (0 = off, the default). edge_b200_kernel_times returns, for kernels 0 = local, 1 = neighbour,
 * 2 = sources, 3 = receivers, the summed milliseconds and launch counts since timing was enabled
 * (synchronises the stream). */
int edge_b200_set_timing(edge_b200_ctx *ctx, int enable);
/* Fused GTS steps (1, the default; 0 turns them off): in configurations that pre-mix their face
 * projections and without halo parts, edge_b200_step with n_steps > 1 runs each step's neighbour
 * step inside the next step's local kernel (which adds the previous projections' lifted fluxes to
 * each element's DOF rows before its recursion; the receiver kernel does the same for its
 * elements), with the face projections alternating between two buffers; the last step's
 * neighbour step runs on its own before the call returns, so the DOFs are complete between calls.
 * Same arithmetic as the separate neighbour kernel: the results are identical. No counterpart in
 * the reference. */
int edge_b200_set_fused(edge_b200_ctx *ctx, int enable);
int edge_b200_kernel_times(edge_b200_ctx *ctx, double *ms, int64_t *launches);
/* Launch shape of the context's compiled configuration (no counterpart in the reference, whose
 * kernels run one element per thread team): info[0] elements per CTA, info[1] 1 when GTS face
 * projections leave the local kernel pre-mixed with the reading element's flux solver (the local
 * kernel then reads per element face the padded pair [2][info[2]] of flux solvers in the
 * configuration's precision, the neighbour kernel none), 2 when the local kernel does both of those
 * mixes through the rank-3 factors of the face's flux-solver pair (it then reads 108 factor values
 * per face instead of the pair; the form of the next GTS step once its factors are built),
 * info[3] / info[4] persistent CTAs of the
 * local / neighbour kernel, info[5] 1 when multi-step calls fuse each neighbour step into the next
 * local kernel (edge_b200_set_fused). */
int edge_b200_kernel_config(const edge_b200_ctx *ctx, int32_t info[6]);

/* No counterpart in the reference. n_steps GTS steps (local kernel, then neighbour kernel; no
 * sources, no receivers) over caller-owned DEVICE arrays, without allocating anything: no
 * context, no cudaMalloc / cudaFree, no allocating library call. It is meant for callers that
 * cannot allocate device memory while they run, e.g. a host that has handed every byte of the GPU
 * to a fixed memory budget or pool, or one that must not hit the device-wide synchronisation
 * cudaMalloc and cudaFree imply in the middle of its time loop.
 * Its scratch -- the face projections the two kernels exchange and a copy of the DOFs in the
 * kernels' row layout (rows of B and F padded to 16 bytes) -- lives in one file-scope device array
 * of EDGE_B200_NOALLOC_SCRATCH_BYTES (32 MiB) that every GPU loading the library holds until exit;
 * a problem needing more (about n_el * R * (4 * 9 * F + (9 + 6 * n_rms) * B) * sizeof(real)
 * bytes) is rejected with EDGE_B200_ESCRATCH. The first call on a device looks up that array's
 * device address, and the first call of each configuration on a device sets its kernels'
 * shared-memory limits and grid sizes, with that device current; make those first calls before any
 * stream capture. The call makes cfg->device current while it runs and restores the caller's
 * current device before it returns. Every call shares the array: calls that overlap on the GPU
 * (other streams, other host threads) race and must be serialised by the caller. Nothing in it
 * needs to start at zero: each step writes every face projection before reading it.
 * Arguments: cfg as for edge_b200_create (order, n_runs, n_rms, precision, stream, device);
 * dofs_e / dofs_a in the cfg precision, element data in FP64 with the layouts of
 * edge_b200_upload_element_data, connectivity as in edge_b200_upload_mesh, all on cfg->device
 * (el_fa_el 16-byte aligned, the three byte arrays 4-byte aligned, as cudaMalloc returns them;
 * EDGE_B200_EINVAL otherwise); only omega (n_rms relaxation frequencies) is a host array. */
#define EDGE_B200_NOALLOC_SCRATCH_BYTES (32u << 20)
int edge_b200_step_noalloc(const edge_b200_cfg *cfg, int64_t n_el, double dt, int n_steps,
                           void *dofs_e, void *dofs_a, const double *star_e, const double *fs_e,
                           const double *star_a, const double *src_a, const double *fs_a,
                           const double *omega, const int32_t *el_fa_el,
                           const uint8_t *fid_el_fa_el, const uint8_t *vid_el_fa_el,
                           const uint8_t *el_fa_type);
/* ---------------------------- batches of simulations, autotuner --------------------------- */

/* A batch of contexts (different meshes, orders, fused runs, physics; one device) stepped
 * together: one batch step is every active context's GTS step (local, sources, neighbour), each
 * context's kernels on a stream of its own, so the independent contexts' kernels run side by side.
 * Two batch steps are captured once into a CUDA graph and replayed; contexts whose edge_b200_step
 * folds each neighbour step into the next local step do the same here (the first step of a call and
 * an odd last one are launched directly, and every call ends with the fused contexts' last
 * neighbour step, so nothing is pending between calls; each context's step form is fixed when the
 * graph is captured). Context k steps from time t0[k] by dt[k];
 * a device counter per context gives its sources the step's time. The contexts keep their data;
 * upload DOFs and element data before creating the batch, and call edge_b200_batch_sync before
 * using a context on its own again. Contexts with receivers, halo parts or kernel timing on are
 * refused (EDGE_B200_ENOTSUP): those run through edge_b200_step. No counterpart in the reference
 * (one solver per process; here uneven batches of simulations on one GPU). */
typedef struct edge_b200_batch edge_b200_batch;
int edge_b200_batch_create(edge_b200_ctx *const *ctxs, int n, const double *t0, const double *dt,
                           edge_b200_batch **out);
/* active[k] != 0: context k takes part in the following steps (all do after create); the graph is
 * captured again at the next step when the set changed, e.g. when a simulation finished. */
int edge_b200_batch_set_active(edge_b200_batch *b, const int32_t *active);
/* n_steps batch steps on the batch's own stream; returns without waiting. */
int edge_b200_batch_step(edge_b200_batch *b, int n_steps);
/* Waits for the batch; steps[n] (may be NULL) receives the steps each context has taken. */
int edge_b200_batch_sync(edge_b200_batch *b, int64_t *steps);
const char *edge_b200_batch_last_error(const edge_b200_batch *b);
int edge_b200_batch_destroy(edge_b200_batch *b);
/* Launch-shape autotuner for this context's mesh: times the local and then the neighbour kernel
 * with its grid at the persistent default (resident CTAs per SM x SMs), half of it, and one CTA
 * per element group, keeps the fastest for later GTS steps, and restores the DOFs it stepped
 * (needs device memory for one copy of them). caps[2] (may be NULL) receives the chosen grid caps
 * (0 = the default). The element-group shape itself (32 / runs elements per CTA) is fixed per
 * compiled configuration. No counterpart in the reference. */
int edge_b200_autotune(edge_b200_ctx *ctx, double dt, int32_t caps[2]);

/* Last CUDA error string of the context (static storage). */
const char *edge_b200_last_error(const edge_b200_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
