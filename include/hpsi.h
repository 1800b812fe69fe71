/*
 * hpsi.h -- C ABI of the B200 Hamiltonian-apply and Taylor-propagation library.
 *
 * The library is a drop-in behind Octopus' X(hamiltonian_elec_apply_batch)
 * and the Taylor branch of exponential_apply_batch.  The host keeps the mesh,
 * the finite-difference weights, the projector matrices and the state batches;
 * it hands them to the library as plain pointers and sizes.  Every entry point
 * is `extern "C"`, callable from Fortran through iso_c_binding `bind(C)`
 * interfaces (no hidden string arguments, no Fortran name mangling).
 *
 * Conventions
 *  - Indices are 0-based.  Point arrays list the np inner points first and the
 *    np_part - np boundary points after them, as mesh%idx does.
 *  - A batch is "packed" in the reference's sense (src/grid/batch.F90:58-59,
 *    zff_pack(ist, ip)): states fastest, `ld` complex numbers per point.
 *  - Batch pointers may be device pointers (used in place, zero copy) or host
 *    pointers (the library stages them through device memory; the call then
 *    returns only when the result is back in host memory).
 *  - Every call that takes a `stream` is ordered on that CUDA stream
 *    (cudaStream_t passed as void*; NULL is the legacy default stream).
 *  - Handles own device scratch that their calls reuse: a hamiltonian its
 *    Taylor work batches, projection and split-K buffers; a mesh its
 *    reduction scratch and the staging buffers of host batches.  Calls that
 *    share a handle (a mesh included) must be ordered on the GPU: one stream,
 *    or events between streams.
 *  - Errors are returned as hpsi_status; the library never exits the process.
 *    hpsi_last_error_string() gives a one-line message for the calling thread.
 */
#ifndef HPSI_H
#define HPSI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t hpsi_status;
#define HPSI_OK 0
#define HPSI_ERR_ARG 1         /* bad argument (size, null pointer, layout) */
#define HPSI_ERR_INDEX 2       /* an index map points outside its range */
#define HPSI_ERR_NONFINITE 3   /* NaN or Inf found in an input or a result */
#define HPSI_ERR_CUDA 4        /* a CUDA runtime call failed */
#define HPSI_ERR_TIMEOUT 5     /* a bounded device wait gave up */
#define HPSI_ERR_STATE 6       /* handle not ready (e.g. weights not set) */
#define HPSI_ERR_NOMEM 7       /* device allocation failed */
#define HPSI_ERR_RUNAWAY 8     /* norm growth beyond the runaway limit */
#define HPSI_ERR_UNSUPPORTED 9 /* valid request this build does not handle */

/* storage / arithmetic of a batch */
#define HPSI_C128 0 /* complex128 storage, FP64 arithmetic */
#define HPSI_C64 1  /* complex64 storage, FP32 arithmetic (FP64 reductions) */

/* Hamiltonian terms: the TERM_* bits of
 * src/hamiltonian/hamiltonian_elec_base.F90:149-158 that this path serves. */
#define HPSI_TERM_KINETIC 1
#define HPSI_TERM_LOCAL_POTENTIAL 2
#define HPSI_TERM_NON_LOCAL_POTENTIAL 4
#define HPSI_TERM_ALL 0x7fffffff

typedef struct hpsi_mesh hpsi_mesh;
typedef struct hpsi_hamiltonian hpsi_hamiltonian;

/* ------------------------------------------------------------------ */
/* Mesh: replaces the index arrays the reference builds in
 * mesh_init_stage_2 (src/grid/mesh_init.F90:185-360) and the stencil run
 * tables of nl_operator_build (src/grid/nl_operator.F90:308-456); the library
 * derives its own cell maps from the point coordinates. */
typedef struct {
  int32_t np;             /* inner points */
  int32_t np_part;        /* inner + boundary points */
  const int32_t *lxyz;    /* 3*np_part integer coordinates, (x,y,z) per point */
  double spacing[3];      /* mesh%spacing */
  int32_t order;          /* stencil half-width (DerivativesOrder); 4 */
  int32_t periodic;       /* 0: boundary points are zero-BC points,
                             1: boundary point b is a periodic image of
                                per_inner[b] (per_points, boundaries.F90) */
  const int32_t *per_inner; /* np_part-np entries when periodic, else NULL */
} hpsi_mesh_desc;

/* Builds the device cell maps.  Fails with HPSI_ERR_INDEX if a stencil point
 * of an inner point is not a mesh point (the reference asserts the same,
 * nl_operator.F90:367). */
hpsi_status hpsi_mesh_create(const hpsi_mesh_desc *desc, hpsi_mesh **out);
hpsi_status hpsi_mesh_destroy(hpsi_mesh *mesh);
/* dims[0..2]: padded cell box, dims[3..5]: inner bounding box */
hpsi_status hpsi_mesh_info(const hpsi_mesh *mesh, int32_t dims[6]);

/* ------------------------------------------------------------------ */
/* Hamiltonian: the state of hamiltonian_elec_t that H.psi reads
 * (src/hamiltonian/hamiltonian_elec.F90), bound to one mesh. */
hpsi_status hpsi_hamiltonian_create(hpsi_mesh *mesh, hpsi_hamiltonian **out);
hpsi_status hpsi_hamiltonian_destroy(hpsi_hamiltonian *ham);

/* Kinetic operator: the Laplacian weights op%w(:,1) of the order-4 star
 * (W = 25 points in stencil_star_get_lapl order, src/grid/stencil_star.F90:59-93,
 * solved by derivatives_make_discretization, src/grid/derivatives.F90:639-757)
 * and the factor -1/(2m) that X(derivatives_batch_start) applies
 * (src/hamiltonian/hamiltonian_elec_inc.F90:155).  `points` is 3*W offsets and
 * must be the star of the mesh's order. */
hpsi_status hpsi_hamiltonian_set_kinetic(hpsi_hamiltonian *ham, int32_t W,
                                         const int32_t *points, const double *w,
                                         double factor);

/* Local potential v(np) for the spin channel of the batch
 * (hm_base%potential, used by X(hamiltonian_elec_base_local_sub),
 * src/hamiltonian/hamiltonian_elec_base_inc.F90:233-242).  Set-up call: host
 * or device pointer, returns with the potential in place (it synchronises the
 * legacy default stream); NULL removes the term. */
hpsi_status hpsi_hamiltonian_set_vloc(hpsi_hamiltonian *ham, const double *v);

/* The same potential update ordered on `stream`, for hosts that rebuild
 * hm%potential every time step (hamiltonian_elec_update,
 * src/hamiltonian/hamiltonian_elec.F90:985-1304): no device synchronisation,
 * and no allocation after the first call on the handle (which allocates the
 * device copy and, for host input, a staging buffer of np doubles).  A device
 * `v` is read when the stream reaches the update, a pinned host `v` likewise
 * (keep it unchanged until then); a pageable host `v` is copied before the
 * call returns.  Host input is checked for NaN/Inf; device input is not. */
hpsi_status hpsi_hamiltonian_update_vloc(hpsi_hamiltonian *ham, const double *v,
                                         void *stream);

/* Length-gauge laser term folded into the local potential,
 * v(r) += amplitude * pol . r (laser_potential, src/hamiltonian/lasers.F90:823-853). */
hpsi_status hpsi_hamiltonian_set_field(hpsi_hamiltonian *ham, const double pol[3],
                                       double amplitude);

/* Bloch phase correction of the periodic boundary copy, one complex number
 * per boundary point (hm_base%phase_corr(np+1:np_part, ik),
 * src/hamiltonian/hamiltonian_elec.F90:634-647; applied in
 * src/grid/boundaries_inc.F90:650-700).  2*(np_part-np) doubles, or NULL to
 * remove it. */
hpsi_status hpsi_hamiltonian_set_phase_corr(hpsi_hamiltonian *ham,
                                            const double *phase_corr);

/* Kleinman-Bylander projector matrices (projector_matrix_t,
 * src/hamiltonian/projector_matrix.F90:37-90, built by
 * hamiltonian_elec_base_build_proj, src/hamiltonian/hamiltonian_elec_base.F90:436-911).
 * Matrix m has npoints[m] sphere points and nprojs[m] projectors; the arrays
 * are the matrices concatenated in order:
 *   map      sum(npoints)            mesh point of each sphere point (pmat%map)
 *   matrices sum(npoints*nprojs)     point fastest within a matrix (dprojectors)
 *   scal     sum(nprojs)             e_KB * vol_pp (pmat%scal, :628)
 * nmat = 0 removes the projectors. */
hpsi_status hpsi_hamiltonian_set_projectors(hpsi_hamiltonian *ham, int32_t nmat,
                                            const int32_t *npoints,
                                            const int32_t *nprojs,
                                            const int32_t *map,
                                            const double *matrices,
                                            const double *scal);

/* Projector phases for k != 0 (projector_phases, built by
 * projector_init_phases, src/hamiltonian/projector.F90:171-247, and applied
 * in src/hamiltonian/hamiltonian_elec_base_inc.F90:680-701 and :934-1025):
 * one complex number per sphere point of each matrix, in the order of the
 * map passed to hpsi_hamiltonian_set_projectors.  The bra gathers
 * psi(map) * phase, the ket adds its contribution times conj(phase).
 * Layout of `phases` (complex numbers as pairs of doubles):
 *   ld_points == 0: packed, the matrices' points concatenated in matrix
 *                   order (2*sum(npoints) doubles);
 *   ld_points >= max(npoints): padded, point k of matrix m at complex index
 *                   k + m*ld_points (2*nmat*ld_points doubles).  This is the
 *                   reference's hm_base%projector_phases(1:max_npoints, 1,
 *                   1:nmat, ik) slice (hamiltonian_elec_base.F90:1267, 1877:
 *                   projector_phases(max_npoints, nphase, nmat, kpt)), which a
 *                   Fortran caller passes as projector_phases(:, 1, :, ik) with
 *                   ld_points = max_npoints (the compiler copies the section
 *                   into a contiguous temporary).
 * ld_points below the largest sphere gives HPSI_ERR_ARG.  NULL removes the
 * phases; setting new projectors removes them too.  With phases the bra runs
 * on the SIMT kernel (at most 32 projectors per matrix). */
hpsi_status hpsi_hamiltonian_set_projector_phases(hpsi_hamiltonian *ham,
                                                  const double *phases,
                                                  int32_t ld_points);

/* ------------------------------------------------------------------ */
/* A borrowed state batch (batch_t / wfs_elec_t in packed status). */
typedef struct {
  void *ptr;       /* device or host pointer to npts * ld complex numbers */
  int64_t ld;      /* complex numbers per point (pack_size(1)) */
  int32_t nst;     /* states in use, nst <= ld */
  int32_t npts;    /* points held: np_part for an input, >= np for an output */
  int32_t dtype;   /* HPSI_C128 or HPSI_C64 */
} hpsi_batch;

/* hpsi = H psi on the np inner points: replaces
 * X(hamiltonian_elec_apply_batch)(hm, namespace, mesh, psib, hpsib, terms,
 * set_bc) (src/hamiltonian/hamiltonian_elec_inc.F90:77-261) for the kinetic,
 * local and KB terms.  set_bc != 0 applies the zero or periodic boundary
 * condition to the values the stencil reads (the caller's boundary rows are
 * not written); set_bc == 0 uses the boundary rows of psi as stored. */
hpsi_status hpsi_apply_h(hpsi_hamiltonian *ham, const hpsi_batch *psi,
                         hpsi_batch *hpsi, int32_t terms, int32_t set_bc,
                         void *stream);

/* Writes the boundary rows of psi as boundaries_set does
 * (src/grid/boundaries_inc.F90:275-745): zeros, or periodic copies times the
 * phase correction. */
hpsi_status hpsi_boundaries_set(hpsi_hamiltonian *ham, hpsi_batch *psi,
                                void *stream);

/* psi <- sum_{k=0..order} (-i dt H)^k / k! psi on the np inner points:
 * replaces the Taylor branch of exponential_apply_batch
 * (src/electrons/exponential.F90:581-674, exponential_taylor_series_batch
 * :677-757) without psib2 / inh_psib.  The polynomial is evaluated in Horner
 * form, one fused stencil pass per order.  If `energy`, `dipole` or `norm2`
 * is non-NULL, the per-state FP64 observables of the incoming psi are
 * returned (host arrays of nst doubles):
 *   energy[i] = dV * Re sum conj(psi_i) (H psi_i),
 *   dipole[i] = dV * sum |psi_i|^2 (pol . r)   (pol from set_field, else z),
 *   norm2[i]  = dV * sum |psi_i|^2. */
hpsi_status hpsi_taylor_step(hpsi_hamiltonian *ham, hpsi_batch *psi, double dt_re,
                             double dt_im, int32_t order, double *energy,
                             double *dipole, double *norm2, void *stream);

/* The Taylor step followed by the density of the propagated batch, as
 * propagation_ops_elec_fuse_density_exp_apply does per block
 * (src/td/propagation_ops_elec.F90:261-333, density_calc_accumulate,
 * src/states/density.F90:279-362):
 *   psi <- exp(-i dt H) psi (order-`order` Taylor series, as hpsi_taylor_step),
 *   rho[ip] = (accumulate ? rho[ip] : 0) + sum_i weight[i] |psi_i(ip)|^2.
 * The density is one pass over the propagated batch after the step (a form
 * fused into the last Horner pass and its KB ket exists, but its cross-lane
 * sums slow the stencil pass by more than the separate pass costs).  FP64
 * sums in a fixed order.
 * weight: nst host doubles (kweight x occupation), read before the call
 * returns; psi and rho (np doubles) device memory; stream ordered. */
hpsi_status hpsi_taylor_step_density(hpsi_hamiltonian *ham, hpsi_batch *psi,
                                     double dt_re, double dt_im, int32_t order,
                                     const double *weight, double *rho,
                                     int32_t accumulate, void *stream);

/* exponential_apply_batch with its second output (psib2 / deltat2,
 * src/electrons/exponential.F90:695-744, used by the self-consistent ETRS
 * predictor): psi2 <- exp(-i dt2 H) psi, psi <- exp(-i dt H) psi, both by the
 * order-`order` Taylor series (dt = dt_re + i dt_im, likewise dt2).  Device
 * batches with at least np points, same dtype and nst, distinct storage;
 * rows np.. of psi2 are not written.  No observables, no synchronisation. */
hpsi_status hpsi_taylor_step_dual(hpsi_hamiltonian *ham, hpsi_batch *psi,
                                  hpsi_batch *psi2, double dt_re, double dt_im,
                                  double dt2_re, double dt2_im, int32_t order,
                                  void *stream);

/* ------------------------------------------------------------------ */
/* Time propagation with exponential-midpoint steps
 * (TDPropagator = exp_mid, src/td/propagator_expmid.F90:52-100, driven by
 * td_run, src/td/td.F90:546-631) under a frozen local potential and a
 * length-gauge laser E(t) pol.r with E(t) = E0 sin^2(pi t/T) cos(omega t) on
 * [0, T] (zero outside).  Step n applies the order-`order` Taylor exponential
 * of H(t0 + (n + 1/2) dt).  Per-step FP64 observables of psi(t_n) under
 * H(t_n), summed over the states (host arrays of nsteps, any may be NULL):
 *   energy[n] = sum_i <psi_i|H(t_n)|psi_i>, dipole[n] = sum_i <psi_i|pol.r|psi_i>,
 *   norm2[n] = sum_i <psi_i|psi_i>.
 * use_graph != 0 captures one step (all passes and the observable reduction)
 * in a CUDA graph and replays it nsteps times; the field amplitude of each
 * step comes from a device table, so one graph serves every step.  Returns
 * HPSI_ERR_RUNAWAY if the norm grows by more than 1e-3 relative (the Taylor
 * series diverges for too large dt), HPSI_ERR_NONFINITE on NaN/Inf. */
typedef struct {
  double E0, omega, T;  /* amplitude, frequency, envelope length (a.u.) */
  double pol[3];        /* polarisation (also the dipole direction) */
} hpsi_laser;

hpsi_status hpsi_td_propagate(hpsi_hamiltonian *ham, hpsi_batch *psi, int32_t nsteps,
                              double dt, int32_t order, const hpsi_laser *laser,
                              double t0, int32_t use_graph, double *energy,
                              double *dipole, double *norm2, void *stream);

/* The same driver with the enforced-time-reversal-symmetry propagator
 * (td_etrs for independent particles, src/td/propagator_etrs.F90:70-152):
 * each step is exp(-i dt/2 H(t_n+1)) exp(-i dt/2 H(t_n)) psi (two Taylor
 * exponentials, 2 * order H.psi); the observables of step n are those of
 * psi(t_n) under H(t_n). */
hpsi_status hpsi_td_propagate_etrs(hpsi_hamiltonian *ham, hpsi_batch *psi, int32_t nsteps,
                                   double dt, int32_t order, const hpsi_laser *laser,
                                   double t0, int32_t use_graph, double *energy,
                                   double *dipole, double *norm2, void *stream);

/* ------------------------------------------------------------------ */
/* Independent systems advanced together (no reference counterpart: the
 * reference loops over state blocks on the host,
 * propagation_ops_elec_fuse_density_exp_apply, src/td/propagation_ops_elec.F90:261-333).
 * A group holds nsys Hamiltonians (borrowed, uneven meshes and state counts).
 * hpsi_group_taylor_steps applies nsteps order-`order` Taylor steps (real dt)
 * to psis[s] (device batches, one per system, one storage type): per Horner
 * pass, the KB bras of all systems, one persistent stencil launch over a
 * (system, tile column + z block, state chunk) work list sorted by cost
 * (up to 48 systems per launch), and the KB kets.  use_graph != 0 captures one
 * step in a CUDA graph and replays it. */
typedef struct hpsi_group hpsi_group;
hpsi_status hpsi_group_create(int32_t nsys, hpsi_hamiltonian *const *hams,
                              hpsi_group **out);
hpsi_status hpsi_group_destroy(hpsi_group *group);
hpsi_status hpsi_group_taylor_steps(hpsi_group *group, hpsi_batch *psis,
                                    int32_t nsteps, double dt, int32_t order,
                                    int32_t use_graph, void *stream);

/* Autotuner: times the candidate shapes of the fused stencil pass (state chunk
 * width, z block depth) on scratch batches of width ld and storage dtype and
 * keeps the fastest for this Hamiltonian's later calls with that width.
 * shape_out (optional): {state chunk, rows per thread, z block, tile height
 * (16: one-complex-per-thread pass, 8: register-blocked pass)};
 * ms_out: time of one pass with that shape. */
hpsi_status hpsi_autotune(hpsi_hamiltonian *ham, int32_t dtype, int64_t ld,
                          int32_t shape_out[4], double *ms_out, void *stream);

/* Lanczos exponential psi <- exp(-i dt H) psi of a complex128 device batch
 * (exponential_lanczos_batch, src/electrons/exponential.F90:766-901):
 * Krylov spaces of dimension up to max_order (TDExpOrder, 2..64) built per
 * state with classical Gram-Schmidt against the last two vectors, stopped
 * once every state's error estimate is below tol (TDLanczosTol) after more
 * than 3 iterations, or on breakdown.  iters_out: the dimension used;
 * res_out: the largest error estimate (above tol when the expansion did not
 * converge, which the reference reports as a warning). */
hpsi_status hpsi_lanczos_step(hpsi_hamiltonian *ham, hpsi_batch *psi, double dt,
                              int32_t max_order, double tol, int32_t *iters_out,
                              double *res_out, void *stream);

/* ------------------------------------------------------------------ */
/* Exact discrete adjoint of the Taylor propagator for optimal control
 * (served to opt_control's backward propagation, bwd_step / bwd_step_2,
 * src/opt_control/propagation.F90:477-783).  Forward: nsteps Taylor steps of
 * H_n = H + eps[n] pol.r from psi0 (psi0 is not modified); objective
 * J = sum_i |<phi_i|psi_i(T)>|^2 with phi = targets (target_groundstate,
 * src/opt_control/target_groundstate_inc.F90:83-152).  Backward with
 * lambda_n = T_n^dagger lambda_{n+1}; psi_n is recomputed from checkpoints
 * stored every `ckpt` steps.  Outputs (host, each optional):
 *   J_out;  grad_eps[nsteps] = dJ/d eps_n, exact for the discrete propagator;
 *   grad_v[np] = dJ/d v(r), the vector-Jacobian product for the local potential;
 *   grad_eps_cont[nsteps] = 2 dt Im <lambda_{n+1}|pol.r|psi_n>, the
 *   continuous-adjoint gradient the reference computes (calculate_g /
 *   update_field, propagation.F90:932-998, 1016-1103).  complex128 only. */
hpsi_status hpsi_adjoint_gradient(hpsi_hamiltonian *ham, const hpsi_batch *psi0,
                                  const hpsi_batch *targets, int32_t nsteps,
                                  double dt, int32_t order, const double *eps,
                                  const double pol[3], int32_t ckpt, double *J_out,
                                  double *grad_eps, double *grad_v,
                                  double *grad_eps_cont, void *stream);

/* The same adjoint one step at a time, for a host that drives the backward
 * propagation itself (bwd_step / bwd_step_2,
 * src/opt_control/propagation.F90:477-783, with its own update_field,
 * :1016-1103, between steps).  Step n of the forward run is
 * psi_{n+1} = T_n psi_n with T_n = sum_{k<=order} (-i dt H_n)^k / k! and
 * H_n = H + eps_n pol.r (the Hamiltonian's local potential, kinetic and KB
 * terms as set; the field of set_field is not used and is left unchanged).
 *
 * hpsi_adjoint_step: lambda <- T_n^dagger lambda in place (lambda =
 *   lambda_{n+1} on entry, lambda_n on return; T_n^dagger = T_n(-dt) as H_n is
 *   Hermitian), given psi_n (not modified).  It also returns the exact
 *   vector-Jacobian products of this step:
 *     grad_eps[0]      = dJ/d eps_n = 2 Re sum_{j+m<=order-1} c_{j+m+1}
 *                        <H_n^j lambda_{n+1}| pol.r |H_n^m psi_n>,
 *     grad_eps_cont[0] = its leading term 2 Re c_1 <lambda_{n+1}|pol.r|psi_n>
 *                        (= 2 dt Im <lambda_{n+1}|pol.r|psi_n>, calculate_g),
 *     grad_v[r]       += dJ/dv(r) contribution of the step (2 dV Re sum ...).
 *   grad_eps and grad_eps_cont: one double each, host or device, may be NULL
 *   (host outputs make the call wait for the stream); grad_v: np doubles of
 *   device memory, accumulated, may be NULL.  complex128 device batches with
 *   at least np rows and equal nst and ld.  For J = sum_i |<phi_i|psi_i(N)>|^2
 *   the backward run starts from lambda_N = phi_i <phi_i|psi_i(N)> and calls
 *   this for n = N-1 .. 0; the summed results equal hpsi_adjoint_gradient.
 *   The first call on a handle allocates its scratch (2 order - 1 batches).
 * hpsi_vjp_field: out[2i], out[2i+1] = Re, Im of dV sum_r conj(chi_i(r))
 *   (pol.r) psi_i(r) for every state i (host or device, 2 nst doubles): the
 *   dipole-coupling matrix element calculate_g sums
 *   (src/opt_control/propagation.F90:932-998, vlaser_operator_linear).
 * hpsi_vjp_vloc: grad_v[r] = (accumulate ? grad_v[r] : 0)
 *   + scale * sum_i Re(conj(lambda_i(r)) psi_i(r)) over the inner rows
 *   (device, np doubles): the local-potential VJP of one H application.
 * Both VJPs take complex128 or complex64 device batches (FP64 sums) and are
 * stream ordered. */
hpsi_status hpsi_adjoint_step(hpsi_hamiltonian *ham, hpsi_batch *lambda,
                              const hpsi_batch *psi_n, double eps_n,
                              const double pol[3], double dt, int32_t order,
                              double *grad_eps, double *grad_eps_cont,
                              double *grad_v, void *stream);
hpsi_status hpsi_vjp_field(hpsi_hamiltonian *ham, const hpsi_batch *chi,
                           const hpsi_batch *psi, const double pol[3],
                           double *out, void *stream);
hpsi_status hpsi_vjp_vloc(hpsi_hamiltonian *ham, const hpsi_batch *lambda,
                          const hpsi_batch *psi, double scale, double *grad_v,
                          int32_t accumulate, void *stream);

/* ------------------------------------------------------------------ */
/* FP64 reductions over the np inner points (dV = vol_pp), results in host
 * arrays:
 *   hpsi_nrm2        out[nst]      X(mesh_batch_nrm2), src/grid/mesh_batch_inc.F90:970-1167
 *   hpsi_dotp_matrix out[2*nst*nst] (interleaved complex, row i = bra state,
 *                    column j fastest) X(mesh_batch_dotp_matrix), :20-263
 *   hpsi_orthonormalize_cholesky   S = U^H U, psi <- psi U^-1 in place,
 *                    X(states_elec_orthogonalization_full) cholesky_serial,
 *                    src/states/states_elec_calc_inc.F90:66-98 */
hpsi_status hpsi_nrm2(hpsi_mesh *mesh, const hpsi_batch *psi, double *out,
                      void *stream);
hpsi_status hpsi_dotp_matrix(hpsi_mesh *mesh, const hpsi_batch *a,
                             const hpsi_batch *b, double *out, void *stream);
hpsi_status hpsi_orthonormalize_cholesky(hpsi_mesh *mesh, hpsi_batch *psi,
                                         void *stream);

/* Density accumulation of a propagated batch: replaces density_calc_accumulate
 * for unpolarised / spin-polarised packed batches
 * (src/states/density.F90:279-362):
 *   rho[ip] = (accumulate ? rho[ip] : 0) + sum_i weight[i] |psi_i(ip)|^2
 * over the np inner points.  weight: nst host doubles (kweight x occupation);
 * psi and rho (np doubles) on the device; FP64 sums in a fixed order. */
hpsi_status hpsi_density_accumulate(hpsi_mesh *mesh, const hpsi_batch *psi,
                                    const double *weight, double *rho,
                                    int32_t accumulate, void *stream);

/* Allocation-free variant of hpsi_nrm2 (no counterpart in the reference).
 * For callers that must not make the library allocate device memory at this
 * point (an application that owns the whole device-memory budget or pool, or
 * a per-step loop that may not reach the allocator): it takes np and the
 * volume element directly, needs no mesh handle and calls neither cudaMalloc
 * nor cudaFree.  Its partial sums live in one fixed device array of the
 * library (about 1 MiB, held by every GPU that loads the library until the
 * process exits), so at most HPSI_NOALLOC_MAX_STATES states are accepted;
 * larger batches get HPSI_ERR_ARG.  The first call in a CUDA context (the
 * device's primary context, or a context the application created and made
 * current) looks up that array's address in the context and should come
 * before any stream capture.  All
 * calls on a device share the array and it keeps the last call's contents:
 * calls that overlap on the GPU (for example on two streams) race and must be
 * ordered by the caller.  `out` (nst doubles) may be host or device memory;
 * with host memory the call waits for the stream. */
#define HPSI_NOALLOC_MAX_STATES 256
hpsi_status hpsi_nrm2_noalloc(int32_t np, double vol_pp, const hpsi_batch *psi,
                              double *out, void *stream);

/* ------------------------------------------------------------------ */
/* Ghost rows of a domain-parallel mesh (X(ghost_update_batch_start/finish),
 * src/grid/boundaries_inc.F90:57-231, par_vec_t layout: local points, then
 * ghost rows grouped by source partition, then boundary points).
 * hpsi_ghost_pack: sendbuf[i][s] = psi[sendmap[i]][s] for i < count, s < nst
 * (sendbuf contiguous, count x nst complex of psi's dtype; the reference's
 * ghost_reorder kernel).  hpsi_ghost_unpack: psi[pos[i]][s] = recvbuf[i][s],
 * for batches whose rows are not contiguous (ld > nst); with ld == nst the
 * received message can land in the ghost rows directly.  Maps and buffers
 * are device memory; map entries outside [0, npts) are skipped.  Stream
 * ordered, no synchronisation.  After the exchange, hpsi_apply_h with
 * set_bc = 0 reads the ghost rows as stored (boundary points must hold
 * their boundary values, zero for a zero boundary). */
hpsi_status hpsi_ghost_pack(const hpsi_batch *psi, const int32_t *sendmap,
                            int32_t count, void *sendbuf, void *stream);
hpsi_status hpsi_ghost_unpack(const void *recvbuf, const int32_t *pos,
                              int32_t count, hpsi_batch *psi, void *stream);

/* The KB term split at its reduction, for meshes whose projector spheres
 * cross partitions: X(hamiltonian_elec_base_nlocal_start) computes the
 * projections of the local points, mesh%allreduce sums them over the
 * partitions, X(hamiltonian_elec_base_nlocal_finish) adds the ket
 * (src/hamiltonian/hamiltonian_elec_base_inc.F90:444-790, :836, :794-1200).
 * hpsi_projector_bra:
 *   proj[r][s] = scal[r] * sum_k P[k][r] * psi[map[k]][s]
 * for every projection row r (matrices in order, their projectors in order)
 * and s < psi->ld; proj is device memory of nprojections x psi->ld complex
 * numbers of psi's dtype (row stride psi->ld).  A matrix with no points here
 * gives zero rows, so every partition's rows line up for the sum.
 * hpsi_projector_ket: hpsi[map[k]][s] += a * sum_r P[k][r] * proj[r][s]
 * (a = a_re + i a_im; 1 for H psi) for s < hpsi->nst, proj laid out as
 * the bra writes it, with row stride hpsi->ld.  hpsi_apply_h without HPSI_TERM_NON_LOCAL_POTENTIAL followed by
 * the bra, the sum and the ket equals hpsi_apply_h with every term.
 * Batches and proj on the device; stream ordered, no synchronisation. */
hpsi_status hpsi_projector_count(const hpsi_hamiltonian *ham,
                                 int32_t *nprojections);
hpsi_status hpsi_projector_bra(hpsi_hamiltonian *ham, const hpsi_batch *psi,
                               void *proj, void *stream);
hpsi_status hpsi_projector_ket(hpsi_hamiltonian *ham, const void *proj,
                               double a_re, double a_im, hpsi_batch *hpsi,
                               void *stream);

/* One level of the Horner form of the Taylor series
 * (src/electrons/exponential.F90:701-748 sums the same polynomial term by
 * term): out = psi0 + a * H psi on the np inner points, a = a_re + i a_im,
 * for the terms selected.  psi holds np_part points (its boundary rows, or
 * the ghost rows of a domain-parallel mesh, are read as stored with
 * set_bc = 0); psi0 and out hold >= np points and may be the same batch, out
 * may not be psi.  With the KB term split off (domain-parallel meshes), the
 * ket of the summed projections follows with hpsi_projector_ket(.., a, ..).
 * Order-K Taylor step: for k = K..1, in <- psi + (-i dt / k) H in.  Device
 * batches with equal dtype, ld and nst; stream ordered. */
hpsi_status hpsi_apply_h_horner(hpsi_hamiltonian *ham, const hpsi_batch *psi,
                                const hpsi_batch *psi0, hpsi_batch *out,
                                double a_re, double a_im, int32_t terms,
                                int32_t set_bc, void *stream);

/* Inner/outer split of a domain-parallel pass, so that the points whose
 * stencil reads no ghost row run while the ghost rows are in flight
 * (X(derivatives_batch_start/finish) with the ghost update overlapped,
 * src/grid/derivatives_inc.F90:82-102, op%inner / op%outer of
 * src/grid/nl_operator.F90:458-514).
 * hpsi_mesh_set_ghost_rows: rows [first, first + count) of the mesh (between
 * np and np_part) are ghost rows (par_vec_t order: local points, ghosts,
 * boundary); count = 0 clears it.
 * hpsi_apply_h_points / hpsi_apply_h_horner_points: hpsi_apply_h /
 * hpsi_apply_h_horner restricted to
 *   HPSI_POINTS_INNER  output rows whose stencil reads no ghost row (the
 *                      ghost rows are not read at all: they may change while
 *                      this runs),
 *   HPSI_POINTS_OUTER  the other output rows,
 *   HPSI_POINTS_ALL    every row (the plain call).
 * INNER then OUTER writes every row once, the same values as ALL.  Rows are
 * split per 16-cell tile column and z plane, conservatively (a plane whose
 * widened tile box holds a ghost cell is outer).  Device batches only; the KB
 * term must go through hpsi_projector_bra / hpsi_projector_ket (it is added
 * once, after both parts). */
#define HPSI_POINTS_ALL 0
#define HPSI_POINTS_INNER 1
#define HPSI_POINTS_OUTER 2
hpsi_status hpsi_mesh_set_ghost_rows(hpsi_mesh *mesh, int32_t first, int32_t count);
hpsi_status hpsi_apply_h_points(hpsi_hamiltonian *ham, const hpsi_batch *psi,
                                hpsi_batch *hpsi, int32_t terms, int32_t set_bc,
                                int32_t points, void *stream);
hpsi_status hpsi_apply_h_horner_points(hpsi_hamiltonian *ham, const hpsi_batch *psi,
                                       const hpsi_batch *psi0, hpsi_batch *out,
                                       double a_re, double a_im, int32_t terms,
                                       int32_t set_bc, int32_t points, void *stream);

/* ------------------------------------------------------------------ */
/* Library-wide controls and diagnostics. */
/* Status word of the kernels of a Hamiltonian that wait on the hardware with a
 * bound (the TMA fill of the stencil pass): HPSI_OK, or HPSI_ERR_TIMEOUT when a
 * wait gave up (its pass's results are then invalid).  Waits for the device,
 * returns the word and clears it. */
hpsi_status hpsi_hamiltonian_status(hpsi_hamiltonian *ham, int32_t *status);
const char *hpsi_last_error_string(void);
/* Number of this library's kernels launched since load (diagnostic). */
int64_t hpsi_kernel_launch_count(void);
/* Version string of this build. */
const char *hpsi_version(void);
/* Kernel timer (the analogue of the reference's profiling_in/out labels,
 * src/basic/profiling.F90:503-625): when enabled, CUDA events are recorded on
 * the launch stream around every kernel of the labels "pass_fp64",
 * "pass_fp32", "bra_fp64" and "bra_fp32".  Enabling clears the records;
 * hpsi_profile_query synchronises on them and returns the launch count and
 * the summed device time of one label. */
hpsi_status hpsi_profile_enable(int32_t on);
hpsi_status hpsi_profile_query(const char *label, int64_t *launches, double *total_ms);

#ifdef __cplusplus
}
#endif

#endif /* HPSI_H */
