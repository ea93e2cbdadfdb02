/*
 * ibpm_b200.h -- C ABI of the B200 IBPM time step (libibpm_b200.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status returns
 * (0 = success, < 0 = error; ibg_last_error() says why).  No call aborts.
 *
 * Array layouts are the reference's own, so a host State can be moved in
 * and out without reshuffling (paths are inside the reference project):
 *   Scalar (omega, psi, rhs): [lev][i-1][j-1], lev < ngrid, 1 <= i < nx,
 *       1 <= j < ny, j fastest                           (src/Scalar.h:76-90)
 *   Flux (q): [lev][index], x-fluxes i*ny + j (i <= nx, j < ny) then
 *       y-fluxes (nx+1)*ny + i*(ny+1) + j (i < nx, j <= ny) (src/Flux.h:176-185)
 *   BoundaryVector (f, b): [fx_0 .. fx_{n-1}, fy_0 .. fy_{n-1}]
 *                                                    (src/BoundaryVector.h:65-69)
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef IBPM_B200_H
#define IBPM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define IBG_API __attribute__((visibility("default")))
#else
#define IBG_API
#endif

typedef struct ibg_context ibg_context;

/* Grid(nx, ny, ngrid, length, xOffset, yOffset)  (src/Grid.h:36-44) */
typedef struct {
    int nx, ny, ngrid;
    double length, xoffset, yoffset;
} ibg_grid;

/* motion kinds of a rigid body, one per `motion` keyword of the geometry file
 * (src/RigidBody.cc:349-493; src/Motion.h and its subclasses) */
enum {
    IBG_MOTION_NONE = 0,
    IBG_MOTION_FIXED = 1,               /* fixed x y theta                    src/FixedPosition.h */
    IBG_MOTION_PITCHPLUNGE = 2,         /* pitchplunge Ap fp php Ay fy phy    src/PitchPlunge.h */
    IBG_MOTION_FIXEDVEL = 3,            /* fixedvel xdot ydot thetadot        src/FixedVelocity.h */
    IBG_MOTION_SIGMOIDALSTEP = 4,       /* sigmoidalstep AMP DUR t0           src/SigmoidalStep.h */
    IBG_MOTION_LAGSTEP1 = 5,            /* lagstep1 AMP PW TAU T0             src/LagStep1.h */
    IBG_MOTION_LAGSTEP2 = 6,            /* lagstep2 AMP PW TAU T0             src/LagStep2.h */
    IBG_MOTION_ELDREDGE = 7,            /* eldredge AMP a t1 t2 t3 t4         src/EldredgeManeuver.h */
    IBG_MOTION_ELDREDGECOMBINED2 = 8,   /* eldredgecombined2 AMPa a a1..a4 AMPb b b1..b4  src/EldredgeCombined2.h */
    IBG_MOTION_ELDREDGE1 = 9,           /* eldredge1 AMP a t1 t2 t3 t4        src/Eldredge1.h */
    IBG_MOTION_ELDREDGE2 = 10,          /* eldredge2 AMP a t1 t2 t3 t4        src/Eldredge2.h */
    IBG_MOTION_FILE = 11,               /* motionfile FILE                    src/MotionFile.h */
    IBG_MOTION_FILE_PERIODIC = 12       /* motionfileperiodic FILE period     src/MotionFilePeriodic.h */
};

/* RigidBody: reference points, centre and motion (src/RigidBody.h:35-190).
 * params holds the numbers of the geometry file's `motion` line in their
 * order (PITCHPLUNGE frequencies in cycles per time unit, as written there;
 * FILE_PERIODIC: params[0] = period).  FILE and FILE_PERIODIC take the
 * file's rows as `table`: table_rows rows of (t, x, y, theta, xdot, ydot,
 * thetadot), t non-decreasing (src/MotionFile.h:62-87).  FIXEDVEL, ELDREDGE2
 * and ELDREDGECOMBINED2 integrate over the times at which the bodies are
 * moved, as the reference's Motion objects do; that history belongs to the
 * context and starts at time 0 when it is created. */
typedef struct {
    int npoints;
    const double* xy;       /* npoints interleaved (x, y) reference points */
    double xcenter, ycenter;
    int motion;
    double params[12];
    int table_rows;
    const double* table;    /* table_rows x 7, row-major; NULL when table_rows == 0 */
} ibg_body;

/* time-stepping schemes (src/Scheme.h:13-61) */
enum { IBG_SCHEME_EULER = 0, IBG_SCHEME_AB2 = 1, IBG_SCHEME_RK3 = 2, IBG_SCHEME_RK3B = 3 };

/* arithmetic forms of the bulk fields: FP64 throughout, or FP32 vorticity,
 * flux, nonlinear term and transforms with the force solve (M^-1, CG dot
 * products and norms) and the forces kept in FP64 */
enum { IBG_PRECISION_FP64 = 0, IBG_PRECISION_FP32_REFINED = 1, IBG_PRECISION_FP32 = 2 };

typedef struct {
    double Re;              /* Reynolds number                                  */
    double dt;              /* time step                                        */
    int scheme;             /* IBG_SCHEME_*                                     */
    double cg_tol;          /* CG tolerance on |r| (moving bodies), 1e-7 default */
    int cg_max_iter;        /* CG iteration cap (the reference has none that works) */
    double u_mag;           /* base-flow magnitude (1 in the reference CLI)     */
    double alpha;           /* base-flow angle in radians                       */
    int precision;          /* IBG_PRECISION_*                                  */
    int device;             /* CUDA device ordinal, -1 = the calling thread's current device */
    int cg_precond;         /* moving bodies: IBG_PRECOND_* (NONE = the reference's plain CG) */
    int pc_refresh;         /* steps between rebuilds of the Cholesky preconditioner (default 10) */
    int cg_graph;           /* moving bodies: 1 = the whole step, CG loop included, is one CUDA graph
                               (the loop is a device-side WHILE node), 0 = host-driven CG loop */
    int pc_fallback_iter;   /* LEARNED: iterations after which the solve restarts as plain CG
                               (also when r.z <= 0); <= 0 means cg_max_iter / 4 */
} ibg_params;

/* preconditioners of the moving-body force solve (all keep the reference's
 * absolute test r.r <= tol^2; NONE is the reference's CG exactly):
 * CHOLESKY: the exact M^-1 of the body configuration at the last rebuild,
 * LEARNED: the boundary-point network (flexible CG, plain-CG fallback) */
enum { IBG_PRECOND_NONE = 0, IBG_PRECOND_CHOLESKY = 1, IBG_PRECOND_LEARNED = 2 };

/* --- lifetime ---------------------------------------------------------------
 * ibg_create replaces the constructors NavierStokesModel(grid, geom, Re, q0)
 * (src/NavierStokesModel.cc:19-33) and NonlinearIBSolver(grid, model, dt,
 * scheme, tol) (src/IBSolver.h:79-86).  `cuda_stream` is a cudaStream_t
 * (NULL: the library creates its own).  The geometry is moved to time 0 and
 * the regularizer updated (model->init(), src/NavierStokesModel.cc:52-57). */
IBG_API int ibg_create(const ibg_grid* grid, int nbodies, const ibg_body* bodies, const ibg_params* params,
               void* cuda_stream, ibg_context** out);
IBG_API int ibg_destroy(ibg_context* ctx);
/* message for the last failed call on ctx (ctx may be NULL for ibg_create) */
IBG_API const char* ibg_last_error(const ibg_context* ctx);

/* IBSolver::init (src/IBSolver.cc:62-66): builds the Cholesky factor of
 * M = C A^-1 B for every sub-step (fixed bodies); no-op for moving bodies. */
IBG_API int ibg_init(ibg_context* ctx);
/* IBSolver::save / load (src/IBSolver.cc:77-108): <basename>_01.cholesky ...
 * in the reference's ASCII format (src/CholeskySolver.cc:113-198).
 * ibg_load returns 1 when every factor was read and matched (n and alpha*beta), 0 otherwise. */
IBG_API int ibg_save(ibg_context* ctx, const char* basename);
IBG_API int ibg_load(ibg_context* ctx, const char* basename);

/* --- state -------------------------------------------------------------------
 * State (src/State.h:25-60): omega, q, f, timestep, time.  `q` may be NULL in
 * ibg_set_state; then it is recomputed from omega (model->refreshState). */
IBG_API int ibg_set_state(ibg_context* ctx, const double* omega, const double* q, const double* f, int timestep, double time);
IBG_API int ibg_get_state(ibg_context* ctx, double* omega, double* q, double* f, int* timestep, double* time);
/* only f, timestep and time (what the reference CLI reads every step) */
IBG_API int ibg_get_boundary_force(ibg_context* ctx, double* f, int* timestep, double* time);
/* NavierStokesModel::updateOperators(time) (src/NavierStokesModel.cc:93-99):
 * moves the base flow (moving frame) and the bodies to `time`; the state's
 * own time is unchanged. */
IBG_API int ibg_update_operators(ibg_context* ctx, double time);
/* The CLI's -ubf option (src/ibpm.cc:166-178): Geometry::transferMotion
 * (src/Geometry.cc:48-71) and BaseFlow::setMotion/setCenter
 * (src/BaseFlow.cc:104-112, src/BaseFlow.h:60).  The single body's motion
 * moves to the base flow, which from then on is the free stream seen from the
 * moving body plus its rotation about the body's centre (BaseFlow::setAlphaMag
 * and moveFlow, Flux::setFlow; src/BaseFlow.cc:114-150, src/Flux.cc:101-129),
 * recomputed at every sub-step; the body stays at its reference points, so
 * the force solve is the fixed-body Cholesky one.  Call before ibg_init.  A
 * stationary body leaves everything unchanged (the reference ignores the
 * flag); more than one body is an error (the reference exits). */
IBG_API int ibg_set_moving_frame(ibg_context* ctx);
/* Geometry::getPoints / getVelocities (src/Geometry.cc:79-110) at the last
 * time the bodies were moved: 2 npoints values each in the BoundaryVector
 * layout (every x, then every y).  Either pointer may be NULL. */
IBG_API int ibg_get_boundary(ibg_context* ctx, double* points, double* velocities);
/* FluxToVelocity(q, u, v) (src/VectorOperations.cc:924-927) of the device
 * state's flux: the node velocities OutputTecplot writes
 * (src/OutputTecplot.cc:41-47), S values each in the Scalar layout.  The
 * coarse-level interior nodes the reference leaves uninitialised are 0. */
IBG_API int ibg_flux_to_velocity(ibg_context* ctx, double* u, double* v);
IBG_API int ibg_refresh_state(ibg_context* ctx);

/* --- restart files ------------------------------------------------------------
 * State::save / State::load (src/State.cc:65-223) in the reference's binary
 * restart format (grid header, q, omega, f as (fx, fy) pairs, timestep, time).
 * ibg_save_restart writes the current state: 1 on success, 0 if the file
 * cannot be opened.  ibg_load_restart reads a file into the context: 1 on
 * success, 0 if the file cannot be opened, < 0 if its grid or point count
 * differs from the context's (the reference resizes its State instead) or it
 * is truncated.
 * ibg_snapshot copies the current state on the device in stream order and
 * sends it to pinned host memory on a side stream, so that the following
 * ibg_advance calls run while it travels; ibg_snapshot_save waits for that
 * copy and writes it as a restart file (the restart output of the reference's
 * logger, src/OutputRestart.cc, without stalling the GPU). */
IBG_API int ibg_save_restart(ibg_context* ctx, const char* filename);
IBG_API int ibg_load_restart(ibg_context* ctx, const char* filename);
IBG_API int ibg_snapshot(ibg_context* ctx);
IBG_API int ibg_snapshot_save(ibg_context* ctx, const char* filename);

/* --- inner products and energy ---------------------------------------------------
 * ibg_inner_product: kind 0 InnerProduct(Scalar, Scalar), 1 FineGridInnerProduct
 * (Scalar), 2 InnerProduct(Flux, Flux), 3 FineGridInnerProduct(Flux)
 * (src/VectorOperations.cc:222-412), with the reference's multi-domain weights, of
 * two host arrays in the Scalar or Flux layout, computed on the device.
 * ibg_energy: 0.5 InnerProduct(q, q) of the current state, what OutputEnergy
 * writes (src/OutputEnergy.cc:29-33), without moving q to the host. */
IBG_API int ibg_inner_product(ibg_context* ctx, int kind, const double* a, const double* b, double* ip);
IBG_API int ibg_energy(ibg_context* ctx, double* energy);

/* --- the other N(x) forms (src/IBSolver.cc:211-283), FP64 ------------------------
 * ibg_set_linearized: LinearizedIBSolver (period 1) or LinearizedPeriodicIBSolver
 * (period P): N(x) = Curl(q0 x omega + q x omega0) with the base state of phase
 * timestep % period; omega0 and q0 hold `period` states one after the other in
 * the Scalar and Flux layouts.  As the reference CLI builds the linear models,
 * create the context with u_mag = 0 (no uniform base flow).  period 0 restores
 * NonlinearIBSolver.
 * ibg_set_sfd: SFDSolver, N(x) = Curl(q x omega) - chi (omega - omega_hat) with
 * the filtered vorticity omega_hat advanced every sub-step by
 * (omega - omega_hat) / Delta; omega_hat starts from the given field (NULL: zero,
 * what the reference CLI's loadFilteredState leaves without a _xhat file).
 * ibg_get_sfd_state reads omega_hat (SFDSolver::saveFilteredState). */
IBG_API int ibg_set_linearized(ibg_context* ctx, int period, const double* omega0, const double* q0);
IBG_API int ibg_set_sfd(ibg_context* ctx, double chi, double Delta, const double* omega_hat);
/* AdjointIBSolver (src/IBSolver.cc:218-222): N(x) = Laplacian(CrossProduct(q0, q))
 * - Curl(CrossProduct(q, omega0)) about one base state (u_mag = 0, as for the
 * linear models); ibg_set_linearized(ctx, 0, NULL, NULL) restores the nonlinear N(x). */
IBG_API int ibg_set_adjoint(ibg_context* ctx, const double* omega0, const double* q0);
IBG_API int ibg_get_sfd_state(ibg_context* ctx, double* omega_hat);

/* IBSolver::advance (src/IBSolver.cc:142-149), nsteps times. */
IBG_API int ibg_advance(ibg_context* ctx, int nsteps);
/* State::computeNetForce (src/State.cc:53-63) of the current f */
IBG_API int ibg_get_net_force(ibg_context* ctx, double* xforce, double* yforce);
/* net force after each of the last `n` steps (device-side record, oldest first);
 * returns the number written (<= n, <= steps taken since ibg_set_state) */
IBG_API int ibg_get_force_history(ibg_context* ctx, int n, double* xy);

/* sizes: total Scalar values (ngrid*(nx-1)*(ny-1)), Flux values, BoundaryVector values */
IBG_API int ibg_sizes(const ibg_context* ctx, long long* n_scalar, long long* n_flux, int* n_boundary);
/* CG statistics of the last advance: iterations of the last sub-step solve,
 * the largest count seen and how many solves hit the cap */
IBG_API int ibg_cg_stats(const ibg_context* ctx, int* last_iterations, int* max_iterations, int* capped_solves);
/* total CG iterations and CG solves since ibg_create */
IBG_API int ibg_cg_totals(const ibg_context* ctx, long long* iterations, long long* solves);
/* the CUDA stream the context launches on (a cudaStream_t) */
IBG_API void* ibg_stream(const ibg_context* ctx);
/* number of kernel launches issued by the last ibg_advance call */
IBG_API long long ibg_last_launch_count(const ibg_context* ctx);

/* --- standalone multi-domain elliptic solvers --------------------------------------
 * PoissonSolver(grid) and HelmholtzSolver(grid, alpha) (src/EllipticSolver.h:26-76):
 * EllipticSolver::solve(f, u) (src/EllipticSolver.cc:47-73) with L u = f
 * (helmholtz 0) or (1 + alpha L) u = f (helmholtz 1) on every level of the
 * grid, coarsifying f first; with ngrid 1 it is EllipticSolver2d::solve with
 * zero boundary values (src/EllipticSolver2d.cc:53-85).  f and u are host arrays
 * in the Scalar layout.  `cuda_stream` as for ibg_create. */
typedef struct ibg_elliptic ibg_elliptic;
IBG_API int ibg_elliptic_create(const ibg_grid* grid, int helmholtz, double alpha, void* cuda_stream,
                                ibg_elliptic** out);
IBG_API int ibg_elliptic_solve(ibg_elliptic* solver, const double* f, double* u);
IBG_API int ibg_elliptic_destroy(ibg_elliptic* solver);
IBG_API const char* ibg_elliptic_last_error(const ibg_elliptic* solver);

/* --- bodies moved by the caller -----------------------------------------------------
 * Geometry::moveBodies (src/Geometry.cc:79-110) run by the caller: for motions the
 * device does not model (a caller's own Motion subclass), the caller moves its
 * bodies on the host and hands the device their points and velocities.
 * ibg_set_external_kinematics switches a context to that mode (the force solve
 * becomes CG, as for any moving body, src/IBSolver.cc:122-135); every slot starts
 * as the current configuration.  ibg_set_step_kinematics sets the points and
 * velocities (BoundaryVector layout, 2 npts values each) the next ibg_advance
 * uses at sub-step `slot` (the time t + c_slot dt of src/IBSolver.cc:165-166), or,
 * with slot -1, moves the bodies there now (NavierStokesModel::updateOperators). */
IBG_API int ibg_set_external_kinematics(ibg_context* ctx);
IBG_API int ibg_set_step_kinematics(ibg_context* ctx, int slot, const double* points, const double* velocities);

/* --- ensembles ------------------------------------------------------------------
 * No single reference interface: an ensemble of independent simulations, each an
 * ibg_context with fixed bodies and its own grid, Reynolds number, time step and
 * bodies (the reference would run one `ibpm` process per member).  The members'
 * captured step graphs become independent branches of one CUDA graph, so one
 * graph launch advances every member by one step and their kernels overlap on
 * the GPU.  Members keep their own state (ibg_get_state, ibg_get_force_history).
 * The first ibg_ensemble_advance captures the members' graphs; if any member has
 * not stepped yet, the first of its steps runs member by member (the start-up of
 * the previous-nonlinear-term history) and the rest as ensemble graphs. */
typedef struct ibg_ensemble ibg_ensemble;
IBG_API int ibg_ensemble_create(int n, ibg_context* const* members, ibg_ensemble** out);
IBG_API int ibg_ensemble_advance(ibg_ensemble* ens, int nsteps);
/* The reference's contract for every member at once (IBSolver::advance(State&),
 * src/IBSolver.cc:142-149: the State lives on the host): each of the nsteps
 * steps copies member i's omega[i], q[i], f[i] (its State arrays, reference
 * layouts, FP64) to the device, advances it and copies them back, all in one
 * graph launch per step, so that one member's copies overlap the other
 * members' steps.  The host arrays must be page-locked (cudaHostAlloc or
 * cudaHostRegister; IBG_ERR_ARG otherwise).  Call ibg_ensemble_advance at least once first; the step
 * counters and times stay the members' own (ibg_get_state).  The graph is
 * rebuilt when the host pointers change. */
IBG_API int ibg_ensemble_advance_host(ibg_ensemble* ens, int nsteps, double* const* omega, double* const* q,
                                      double* const* f);
/* kernels launched per ibg_ensemble_advance_host step (the members' steps plus their precision conversions) */
IBG_API long long ibg_ensemble_host_launches_per_step(const ibg_ensemble* ens);
IBG_API int ibg_ensemble_destroy(ibg_ensemble* ens);
/* one launch shape for every member's DST passes: pairs_per_cta 0 (the rule-based default), 1, 2 or 4
 * line pairs per CTA with `threads` threads; edge_maps 1 applies the precomputed sweep edge maps,
 * 0 the per-step line FFTs (the default for members).  The members' steps are recaptured at the next
 * ibg_ensemble_advance; results do not depend on the shape.  IBG_ERR_UNSUPPORTED when a member's
 * passes would need more than 200 KiB of shared memory with that shape (that member keeps its
 * previous shape; the others take the new one). */
IBG_API int ibg_ensemble_set_shapes(ibg_ensemble* ens, int pairs_per_cta, int threads, int edge_maps);
/* Choose the members' DST launch shapes by timing the ensemble itself: for each class of members with
 * the same grid (largest first) every candidate shape (line pairs per CTA, threads: 2/128, 1/128,
 * 2/256, 1/256, 2/96) runs 1 + steps_per_trial ensemble steps, and a class keeps the candidate whose
 * timed steps are at least 1 % faster than the best so far (else two pairs and 128 threads).  The
 * trials are real steps: every member advances by (1 + steps_per_trial) per trial, 1 + 4 x classes
 * trials in all.  Writes up to max_rows rows of 5 ints {nx, ny, us per ensemble step with that
 * class's choice, pairs per CTA, threads} and returns the number of classes (< 0 on error).  Call
 * ibg_ensemble_advance at least once first. */
IBG_API int ibg_ensemble_autotune(ibg_ensemble* ens, int steps_per_trial, int* out, int max_rows);
IBG_API void* ibg_ensemble_stream(const ibg_ensemble* ens);
IBG_API long long ibg_ensemble_launches_per_step(const ibg_ensemble* ens);
IBG_API const char* ibg_ensemble_last_error(const ibg_ensemble* ens);

/* --- launch-shape autotuner (no reference counterpart) -----------------------
 * The DST row and column passes time their launch shapes (line pairs per CTA,
 * threads per CTA, twiddles in shared memory or not) on whole solves the first
 * time a grid shape is created in the process; ensemble members use the rules.
 * ibg_autotune_log writes up to max_rows rows of 8 ints {bytes per word,
 * pass (0 rows, 1 columns), FFT length, lines, levels, pairs per CTA, threads,
 * twiddles in shared memory} and returns the number of tuned shapes. */
IBG_API int ibg_autotune_log(int* out, int max_rows);
/* The autotuner's choice of form for the FP32 DST passes (the FP32 and FP32-refined
 * contexts): the first time a grid shape is created in the process, whole FP32
 * Poisson solves are timed with the shared-memory FFT passes and with the
 * sine-matrix GEMM passes on the tensor cores (tcgen05 kind::tf32, 3xTF32), and
 * the GEMM form is kept if it is at least 3 % faster (IBG_DST_GEMM=0 or 1 in the
 * environment fixes the form instead).  ibg_dst_form_log writes up to max_rows
 * rows of 6 doubles {nx, ny, levels, GEMM chosen (0/1), FFT solve us, GEMM solve
 * us} and returns the number of grid shapes timed. */
IBG_API int ibg_dst_form_log(double* out, int max_rows);

/* --- learned preconditioner (no reference counterpart) -----------------------
 * For moving bodies the reference runs plain CG on M f = r every sub-step
 * (src/ConjugateGradientSolver.cc:35-65).  With IBG_PRECOND_LEARNED a network
 * (lpc.cu) maps the body geometry to an approximate inverse K of M: an MLP
 * (19 -> 256 -> 256 -> 4, ReLU) over every pair of boundary points whose
 * inputs are the two points' positions and normals, their means over 8
 * boundary neighbours and the pair's offset; its outputs are the 2 x 2 blocks
 * of K.  K is evaluated (BF16) at the start of every step and applied as the
 * PCG preconditioner z = K r; until a network is trained or loaded, and
 * whenever a solve falls back, the iteration is plain CG.
 * ibg_lpc_generate samples nconfig body configurations at times evenly spread
 * over [t0, t1] and returns their geometry features (geom, nconfig x npts x 4
 * floats) and operators M / beta (mb, nconfig x m x m floats, m = 2 npts,
 * row-major) from the solver's own exact force-operator build; column j of M
 * is the residual of the unit force e_j.  ibg_lpc_train fits the network to
 * them (Adam, FP32, loss |K M/(beta c0) - I|_F^2 / m averaged over the
 * configurations; c0 = mean diagonal of M / beta, stored as the last
 * parameter) and enables it; loss_history receives one mean loss per epoch.
 * ibg_lpc_loss_grad returns the loss and its gradient for checking. */
IBG_API size_t ibg_lpc_num_params(void);
IBG_API int ibg_lpc_generate(ibg_context* ctx, int nconfig, double t0, double t1, float* geom, float* mb);
IBG_API int ibg_lpc_train(ibg_context* ctx, int nconfig, const float* geom, const float* mb, int epochs, int batch,
                          float lr, unsigned int seed, float* loss_history);
IBG_API int ibg_lpc_loss_grad(ibg_context* ctx, int nconfig, const float* geom, const float* mb,
                              const float* params, float* loss, float* grad);
IBG_API int ibg_lpc_get_params(ibg_context* ctx, float* params, size_t n);
IBG_API int ibg_lpc_set_params(ibg_context* ctx, const float* params, size_t n);
/* z = K_k r with the current network at the current body configuration (host
 * buffers of 2 npts doubles); geom (optional, npts x 4 floats) receives the
 * geometry features it used */
IBG_API int ibg_lpc_apply(ibg_context* ctx, int substep, const double* r, double* z, float* geom);
/* beta_k of sub-step k (M_k = beta_k C A_k^-1 B, src/ProjectionSolver.cc:43-55) */
IBG_API int ibg_substep_beta(ibg_context* ctx, int substep, double* beta);

/* --- operator entry points (host buffers, reference layouts) ----------------- */
/* PoissonSolver::solve (src/EllipticSolver.cc:47-73, :83-94): L u = f on all levels */
IBG_API int ibg_poisson_solve(ibg_context* ctx, const double* f, double* u);
/* HelmholtzSolver::solve ((1 + alpha L) u = f), src/EllipticSolver.cc:96-108 */
IBG_API int ibg_helmholtz_solve(ibg_context* ctx, double alpha, const double* f, double* u);
/* NonlinearIBSolver::N = Curl(CrossProduct(q, omega)) (src/IBSolver.cc:205-209) */
IBG_API int ibg_nonlinear(ibg_context* ctx, const double* q, const double* omega, double* out);
/* Laplacian(Scalar) = -Curl(Curl(f)) (src/VectorOperations.cc:133-146) */
IBG_API int ibg_laplacian(ibg_context* ctx, const double* f, double* out);
/* NavierStokesModel::B: Curl(E^T f) (src/NavierStokesModel.cc:101-105) */
IBG_API int ibg_model_B(ibg_context* ctx, const double* f, double* omega);
/* NavierStokesModel::C: E(Curl(L^-1(-omega))) (src/NavierStokesModel.cc:107-112) */
IBG_API int ibg_model_C(ibg_context* ctx, const double* omega, double* f);
/* Regularizer::toFlux (src/Regularizer.cc:92-109): boundary vector -> Flux of every
 * level (level 0 holds the smeared values times dx, coarser levels are zero) */
IBG_API int ibg_reg_to_flux(ibg_context* ctx, const double* f, double* q);
/* Regularizer::toBoundary (src/Regularizer.cc:111-128): level-0 fluxes -> boundary */
IBG_API int ibg_reg_to_boundary(ibg_context* ctx, const double* q, double* f);
/* ProjectionSolver::solve for sub-step k's beta (src/ProjectionSolver.cc:57-79):
 * A omega + B f = a, C omega = b.  f is the warm start on input (CG). */
IBG_API int ibg_projection_solve(ibg_context* ctx, int substep, const double* a, const double* b, double* omega, double* f);

/* --- allocation-free variant -------------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc (code running while a CUDA graph is captured into a pool it does
 * not own, plug-ins whose host forbids device allocation after start-up,
 * services that budget every byte of HBM up front).
 * ibg_poisson_solve_static solves L u = f on all levels, like ibg_poisson_solve,
 * but takes DEVICE pointers f and u (reference Scalar layout), needs no context
 * and allocates nothing.  Its memory is file-scope device arrays, held by every
 * GPU that loads the library until the process exits: 4 MiB of scratch
 * (524288 doubles; a solve needs 2*ngrid*(nx-1)*(ny-1) + 2*(ngrid+1)*(nx+ny-2)
 * of them) and about 1.5 MiB of tables, room for the FFT twiddles and
 * eigenvalue/sine tables of 4 grid shapes (368 KiB each).
 * Limits: nx, ny <= 2048; the scratch need above <= 524288; the transform
 * kernels' shared memory 64*max(nx,ny) + 48*max(nx-1,ny-1) bytes <= 200 KiB
 * (max(nx, ny) <= 1828).  Other grids are rejected with IBG_ERR_UNSUPPORTED and
 * a message.
 * The first call on a device resolves the arrays' device addresses
 * (cudaGetSymbolAddress); the first call with a grid shape not among the last
 * four used uploads its tables (replacing the least recently used shape's) and
 * synchronises the stream.  Make both before any stream capture: a call that
 * would upload tables while its stream is capturing is refused with
 * IBG_ERR_UNSUPPORTED.  All calls share the scratch, which keeps the last
 * call's contents (each call writes every scratch value it reads, so nothing
 * needs clearing): calls that overlap on the GPU race on it.  The tables of a
 * shape are rewritten when a fifth shape replaces them, so a call (or a graph
 * captured from one) still in flight with that shape then reads the wrong
 * tables.  Runs on `cuda_stream` (a cudaStream_t, may be NULL).
 * ibg_static_last_error() describes the calling thread's last failure. */
IBG_API int ibg_poisson_solve_static(const ibg_grid* grid, const double* f, double* u, void* cuda_stream);
IBG_API const char* ibg_static_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
