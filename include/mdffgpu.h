/* mdffgpu: B200 (sm_100a) engine for the mdff20 force field and MD step -- C ABI.
 *
 * The reference (mdff20, plain C) has no plugin interface: its "operator API" is a set
 * of void functions that read and write process globals.  Each entry point below
 * replaces one of them; the comment names the reference function (file:line inside
 * the mdff20 repository) and what the call takes instead of the globals.  The shims
 * with the reference's exact names and signatures, working on the reference's globals
 * (engforce, prop_agate, check_verletlist, gen_pbc_verletlist, multipole_ES,
 * get_dipoles), are mdff20_b200/host/mdff_shim.c; `make -C mdff20_b200 dropin` links
 * them with the reference's own program.
 *
 * Conventions
 *  - every call returns an int status (MDFFGPU_OK = 0); the reference prints and calls
 *    exit(-1) instead (src/tools.c:63-67);
 *  - a context holds one system resident on one GPU; calls on a context are
 *    synchronous with respect to the host and must not be made from two threads at once;
 *  - host arrays are plain C arrays: positions/velocities/forces as three SoA arrays of
 *    length nion (the reference's rx,ry,rz / vx,vy,vz / fx,fy,fz, src/config.h:38-40);
 *    per-ion vectors (dipoles, fields) as [nion][3], EFG as [nion][3][3], the stress
 *    tensor as [3][3], all row-major doubles;
 *  - units are the reference's: control-file values in the parameter block, internal
 *    units (eV, Å, amu, Å*(amu/eV)^0.5) in the state arrays.
 */
#ifndef MDFFGPU_H
#define MDFFGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define MDFFGPU_NTMAX 16

/* status codes */
#define MDFFGPU_OK 0
#define MDFFGPU_ERR_ARG 1            /* bad argument or unsupported parameter */
#define MDFFGPU_ERR_CUDA 2           /* a CUDA call failed */
#define MDFFGPU_ERR_LIST_OVERFLOW 3  /* a neighbour list or cell exceeded its capacity */
#define MDFFGPU_ERR_SCF 4            /* induced dipoles did not converge in max_scf_pim_iter */
#define MDFFGPU_ERR_NONFINITE 5      /* a NaN/Inf appeared in positions, forces or dipoles */
#define MDFFGPU_ERR_STATE 6          /* call out of order (e.g. forces before a list exists) */
#define MDFFGPU_ERR_NOMEM 7          /* device allocation failed */
#define MDFFGPU_ERR_CELL 8           /* cutoff + skin exceeds half the cell width */
#define MDFFGPU_ERR_TIMEOUT 9        /* a device loop hit its iteration limit */

/* precision of the pair, Ewald and k-space arithmetic */
#define MDFFGPU_FP64 0
#define MDFFGPU_MIXED 1   /* FP32 arithmetic, compensated FP32/FP64 sums */

/* induced-dipole solver */
#define MDFFGPU_PIM_REFERENCE 0 /* the reference's algo_pim (scf: Jacobi + ASPC, scfkO) */
#define MDFFGPU_PIM_CG 1        /* preconditioned conjugate gradient on (alpha^-1 - T) mu = E_stat */
#define MDFFGPU_PIM_CG_FUSED 2  /* CG with E_stat and the first residual from one Ewald pass, and
                                   rho(k) carried along the iterates for the force pass */

/* Parameter block: the values the reference's parsers leave in its globals, in
 * control-file units (read_global src/global.c:13-60, read_md src/md.c:29-98,
 * read_field src/field.c:31-183, read_nmlj src/nmlj.c:39-107, read_bhmftd
 * src/bhmftd.c:26-90, read_pim src/pim.c:28-69) plus the POSFF header (cell, ions
 * per type, src/config.c:372-401).  Pair tables hold the upper triangle as read
 * (entries [i][j] with j >= i); the engine symmetrises them as the reference does. */
typedef struct mdffgpu_params {
    int nion, ntype;
    int nionit[MDFFGPU_NTMAX];
    double massit[MDFFGPU_NTMAX];
    double cell[3][3];                 /* simuCell.A: rows are the lattice vectors */
    int lreduced, lverletL;
    double skindiff, cutshortrange, cutlongrange;
    int lnmlj, trunctype;              /* 0 no, 1 linear, 2 quadratic */
    double sigmalj[MDFFGPU_NTMAX][MDFFGPU_NTMAX], epslj[MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double plj[MDFFGPU_NTMAX][MDFFGPU_NTMAX], qlj[MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    int lbhmft, lbhmftd;
    double Abhmftd[MDFFGPU_NTMAX][MDFFGPU_NTMAX], Bbhmftd[MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double Cbhmftd[MDFFGPU_NTMAX][MDFFGPU_NTMAX], Dbhmftd[MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double BDbhmftd[MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    int lcoulombic;
    double qit[MDFFGPU_NTMAX], dipit[MDFFGPU_NTMAX][3], polit[MDFFGPU_NTMAX][3][3];
    int lpoldamping[MDFFGPU_NTMAX][MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double pol_damp_b[MDFFGPU_NTMAX][MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double pol_damp_c[MDFFGPU_NTMAX][MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    int pol_damp_k[MDFFGPU_NTMAX][MDFFGPU_NTMAX][MDFFGPU_NTMAX];
    double alphaES;
    int kES[3];
    int algo_pim, algo_extrapolate_dipole, extrapolate_order, min_scf_pim_iter, max_scf_pim_iter;
    double conv_tol_ind, omegakO;
    int egrator;                       /* 0 nve-lf, 1 nve-vv, 2 nvt-nhcn */
    int nhc_n, nhc_mults, nhc_yosh_order, nequil, nequilT;
    double dt, temp, timesca_thermo, tauTberendsen;
} mdffgpu_params;

/* The reference's thermodynamic globals (src/thermo.h:3-14) plus solver counters. */
typedef struct mdffgpu_thermo {
    double e_kin, e_nvt, u_lj, u_bhmftd, u_coul, u_pol;
    double pvir_lj, pvir_bhmftd, pvir_coul;
    double tau_lj[9], tau_bhmftd[9], tau_coul[9];
    double utail, ptail, scf_rmsd;
    int scf_iter, nlist_builds;
} mdffgpu_thermo;

typedef struct mdffgpu_ctx mdffgpu_ctx;

/* Set-up: init_global/read_config/init_md/init_field/init_config
 * (src/mdff20.c:74-82) for one system whose positions (Cartesian, as read_config
 * leaves them after its wrap, src/config.c:442-444) and velocities are given as SoA
 * host arrays (vx may be NULL: zero velocities).  device < 0 uses the current device. */
int mdffgpu_create(const mdffgpu_params *p, const double *rx, const double *ry, const double *rz,
                   const double *vx, const double *vy, const double *vz, int device, mdffgpu_ctx **out);
int mdffgpu_destroy(mdffgpu_ctx *ctx);
const char *mdffgpu_last_error(const mdffgpu_ctx *ctx);
int mdffgpu_set_precision(mdffgpu_ctx *ctx, int precision);
int mdffgpu_set_pim_solver(mdffgpu_ctx *ctx, int solver);
/* No reference counterpart: the launch-shape half of the autotuner (the Ewald alpha and
 * kmax half is mdff20_b200/fit.py's ewald_tune).  For a mixed-precision context with
 * polarisable ions, times the CG field pass of the current system over candidate launch
 * shapes of the k space -- CUDA-core rho pass at 0.5x / 1x / 2x the default ion chunks or
 * tensor-core rho pass, CUDA-core or tensor-core ion pass at 0 (cost model) to 4 row
 * slices -- `reps` passes each, and keeps the fastest for this context.  choice (may be
 * NULL, else 4 ints) receives {tensor-core ion pass 0/1, CUDA-core rho chunks (0 with the
 * tensor-core rho pass), ion-pass row slices, tensor-core rho pass 0/1}, ms (may be NULL)
 * the chosen pass's time.  Runs one force evaluation first; the system's state is not
 * changed. */
int mdffgpu_tune_launch(mdffgpu_ctx *ctx, int reps, int *choice, double *ms);
/* No reference counterpart.  on != 0 (the default): mdffgpu_md_steps replays each MD
 * step as one CUDA graph (the CG loop a device-controlled while node) whenever the step
 * needs no host decision (Verlet lists on, a CG solver, the ASPC order at its final
 * value); 0: every step is issued kernel by kernel.  Results are the same either way. */
int mdffgpu_set_graph(mdffgpu_ctx *ctx, int on);

/* State transfer (the reference's rx..fz globals, src/config.h:38-40).  One copy per
 * array, packed / unpacked on the device; each call returns when its copies are done.
 * Page-locked arrays (cudaHostAlloc) are copied by DMA directly, others through the
 * driver's staging. */
int mdffgpu_set_positions(mdffgpu_ctx *ctx, const double *rx, const double *ry, const double *rz);
int mdffgpu_set_velocities(mdffgpu_ctx *ctx, const double *vx, const double *vy, const double *vz);
int mdffgpu_get_state(mdffgpu_ctx *ctx, double *rx, double *ry, double *rz, double *vx, double *vy,
                      double *vz, double *fx, double *fy, double *fz);
/* dipia_ind history used by the ASPC predictor, [nion][6][3] (src/config.h:48) */
int mdffgpu_set_dipole_history(mdffgpu_ctx *ctx, const double *hist);
int mdffgpu_get_dipole_history(mdffgpu_ctx *ctx, double *hist);
/* Nose-Hoover chain state xi, vxi (nhc_n values each, src/md.h:26) */
int mdffgpu_set_nhc(mdffgpu_ctx *ctx, const double *xi, const double *vxi);
int mdffgpu_get_nhc(mdffgpu_ctx *ctx, double *xi, double *vxi);
/* Exact restart.  No counterpart in the reference, whose restart file CONTFF
 * (write_config, src/config.c:291-345) keeps wrapped positions, velocities and forces
 * at 12 decimals and drops the ASPC dipole history (src/config.h:48), the Nose-Hoover
 * chain (src/md.h:26), the leap-frog r(t-dt) (src/config.h:39), the list-build
 * positions (src/verlet.c:124-170) and the step count that sets the ASPC order.
 * save_state writes the whole MD state after the last step run into buf (state_size
 * bytes, plain little-endian words); load_state puts it into a context created from
 * the same system and returns that step in *istep, so that
 * mdffgpu_md_steps(ctx, *istep + 1, ...) continues the saved run bit for bit. */
int mdffgpu_state_size(const mdffgpu_ctx *ctx, size_t *bytes);
int mdffgpu_save_state(mdffgpu_ctx *ctx, void *buf, size_t bytes);
int mdffgpu_load_state(mdffgpu_ctx *ctx, const void *buf, size_t bytes, int *istep);
/* info_thermo's inputs (src/thermo.c:12-35) */
int mdffgpu_get_thermo(mdffgpu_ctx *ctx, mdffgpu_thermo *t);

/* gen_pbc_verletlist (src/verlet.c:54-122): builds the short-range and Coulomb
 * neighbour lists from the current positions and stores them as list reference. */
int mdffgpu_gen_verletlist(mdffgpu_ctx *ctx);
/* check_verletlist (src/verlet.c:124-170): rebuilds when the largest plus second
 * largest displacement since the last build exceeds skindiff; *rebuilt (may be NULL)
 * tells whether it did. */
int mdffgpu_check_verletlist(mdffgpu_ctx *ctx, int *rebuilt);
/* The lists in the reference's CSR half-list format (verlet_nb / verlet_coul,
 * src/verlet.h:8-16): which = 0 short range, 1 Coulomb; point[nion+1], list[cap];
 * *count receives the number of pairs.  Pairs follow the reference's parity rule
 * (src/verlet.c:82-83), ascending j within each row. */
int mdffgpu_get_verletlist(mdffgpu_ctx *ctx, int which, int *point, int *list, int cap, int *count);

/* engforce (src/field.c:352-407): zeroes forces, then n-m LJ, BHMFT(D), induced
 * dipoles (get_dipoles, src/coulombic.c:67-130) and the multipole Ewald sum. */
int mdffgpu_engforce(mdffgpu_ctx *ctx);
/* engforce_nmlj_pbc (src/nmlj.c:254-385) and engforce_bhmftd_pbc
 * (src/bhmftd.c:117-271): ADD this evaluator's forces to the context forces and
 * return its energy, virial pressure and stress tensor [3][3]. */
int mdffgpu_engforce_nmlj(mdffgpu_ctx *ctx, double *u, double *pvir, double *tau);
int mdffgpu_engforce_bhmftd(mdffgpu_ctx *ctx, double *u, double *pvir, double *tau);
/* multipole_ES (src/ewald.c:75-348) on host arrays q[nion], mu[nion][3]; flags use
 * the bits below.  Outputs (any may be NULL): u, pvir, tau[3][3], ef[nion][3],
 * efg[nion][3][3], and this call's forces f[nion][3] (x coul_unit) -- the reference
 * adds them to its global forces.  alpha > 0 overrides alphaES (the kO inner loop
 * uses 0.001, src/pim.c:694). */
#define MDFFGPU_ES_LQ 1
#define MDFFGPU_ES_LD 2
#define MDFFGPU_ES_LDAMP 4
#define MDFFGPU_ES_FORCES 8
#define MDFFGPU_ES_STRESS 16
#define MDFFGPU_ES_EF 32
#define MDFFGPU_ES_EFG 64
#define MDFFGPU_ES_DIR 128
#define MDFFGPU_ES_REC 256
int mdffgpu_multipole_es(mdffgpu_ctx *ctx, const double *q, const double *mu, int flags, double alpha,
                         double *u, double *pvir, double *tau, double *ef, double *efg, double *f);
/* get_dipoles (src/coulombic.c:67-130) with momentpolaSCF / momentpolaSCFkO
 * (src/pim.c:177-306, 457-603) or CG: total dipoles mu[nion][3] (static + induced)
 * and the polarisation energy u_pol. */
int mdffgpu_get_dipoles(mdffgpu_ctx *ctx, double *mu, double *upol);

/* prop_agate (src/integration.c:298-333) for step istep (1-based): one velocity
 * Verlet, leap-frog or Nose-Hoover-chain step including the force evaluation. */
int mdffgpu_prop_agate(mdffgpu_ctx *ctx, int istep);
/* The MD loop body of run_md (src/md.c:229-241): for istep = first..first+nsteps-1,
 * prop_agate then check_verletlist, all on the device.  thermo (may be NULL) receives
 * nsteps records of 12 doubles: e_kin u_lj u_bhmftd u_coul u_pol e_nvt pvir_lj
 * pvir_bhmftd pvir_coul nlist_builds scf_iter scf_rmsd. */
int mdffgpu_md_steps(mdffgpu_ctx *ctx, int first, int nsteps, double *thermo);
/* No reference counterpart: mdffgpu_md_steps with the state on the host, as a caller
 * that keeps rx..fz in its own arrays runs it (the reference's MD loop over its
 * globals).  in (may be NULL): 6 arrays rx ry rz vx vy vz of nion doubles copied in
 * before the steps (an entry NULL keeps that component's device values); out (may be
 * NULL): 9 arrays rx ry rz vx vy vz fx fy fz the state after the last step is copied to
 * (entries may be NULL).  The copies are queued with the steps: one call and, as in
 * mdffgpu_md_steps, one synchronisation per step, the outgoing copies riding on the last
 * one.  Equivalent to set_positions + set_velocities + md_steps + get_state. */
int mdffgpu_md_steps_host(mdffgpu_ctx *ctx, int first, int nsteps, const double *const *in, double *thermo,
                          double *const *out);

/* Neighbour-list build that allocates no memory.  No counterpart in the reference; it
 * is for callers that cannot allocate device memory: an application that owns all GPU
 * memory through its own pool and forbids allocations after start-up, or a host that
 * runs the engine inside a fixed device-memory budget.  It runs the kernels of
 * mdffgpu_gen_verletlist without a context: d_pos is the caller's device array
 * [n][4] (x, y, z, unused; 32-byte aligned), cell the lattice rows [3][3] on the host,
 * cut_nb/cut_co the two list radii (rc + skin); the FULL lists go to the caller's
 * device buffers d_nb[n][cap_nb], d_nbn[n], d_co[n][cap_co], d_con[n] (each ion's
 * neighbours, both directions of every pair).  Scratch is a static device array of
 * about 5 MB, shared by every call on a device and holding the last call's data:
 * limits n <= 65536 (more returns MDFFGPU_ERR_ARG), a cell grid of at most 32768 cells
 * (a finer grid is coarsened to fit), at most 4096 ions per cell (so n <= 4096 when the
 * cell is too small for a cell grid; more returns MDFFGPU_ERR_CELL).  Calls that overlap on the GPU (other streams, other threads) race
 * on that array.  The first call on a device looks up the array's device address (with
 * that device current); make that first call before any stream capture.  Runs on
 * `stream` (NULL: the default stream) and synchronises it; *status_out (may be NULL)
 * receives the kernels' status bits; a list longer than its capacity returns
 * MDFFGPU_ERR_LIST_OVERFLOW with the true counts in d_nbn/d_con. */
int mdffgpu_build_lists_noalloc(const double *d_pos, int n, const double *cell, double cut_nb, double cut_co,
                                int cap_nb, int *d_nb, int *d_nbn, int cap_co, int *d_co, int *d_con,
                                void *stream, int *status_out);

/* Radial distribution function: the pair histogram of get_gr
 * (src/radial_distribution.c:180-230), accumulated over configurations on the GPU.
 * An accumulator is independent of any context: nion ions in blocks of nionit per
 * type (the order of POSFF), pairs closer than cutgr counted in bins of width resg,
 * nbins of them.  rdf_add adds one configuration given as Cartesian host arrays and
 * its cell rows [3][3] (read_next_traj + get_gr, src/radial_distribution.c:70-81);
 * rdf_add_ctx adds a context's current positions without leaving the device (same
 * ions and device).  rdf_counts returns the ordered-pair counts
 * pairs[nbins][ntype][ntype] (bin of (int)(r/resg), both orders of every pair, as
 * get_gr counts them; the reference additionally folds all pairs into its [0][0]
 * entry) and the number of configurations added. */
typedef struct mdffgpu_rdf mdffgpu_rdf;
int mdffgpu_rdf_create(int nion, int ntype, const int *nionit, double cutgr, double resg, int nbins, int device,
                       mdffgpu_rdf **out);
int mdffgpu_rdf_destroy(mdffgpu_rdf *rdf);
const char *mdffgpu_rdf_last_error(const mdffgpu_rdf *rdf);
int mdffgpu_rdf_reset(mdffgpu_rdf *rdf);
int mdffgpu_rdf_add(mdffgpu_rdf *rdf, const double *cell, const double *rx, const double *ry, const double *rz);
int mdffgpu_rdf_add_ctx(mdffgpu_rdf *rdf, mdffgpu_ctx *ctx);
int mdffgpu_rdf_counts(mdffgpu_rdf *rdf, long long *pairs, int *nconf);

/* Number of kernel launches the engine made so far (for accounting).  No counterpart
 * in the reference. */
long long mdffgpu_launch_count(const mdffgpu_ctx *ctx);
/* The cudaStream_t every call of this context runs on, so a caller can record CUDA
 * events around a call.  No counterpart in the reference. */
void *mdffgpu_stream(const mdffgpu_ctx *ctx);
/* Diagnostic: time every launch of one kernel family ("k_rho", "k_rec_ion", "k_dir")
 * with CUDA events on the context stream from now on (NULL stops and clears);
 * profile_result returns the summed device time (ms), the number of launches and the
 * algorithmic flops of those launches.  No counterpart in the reference. */
int mdffgpu_profile(mdffgpu_ctx *ctx, const char *kernel);
int mdffgpu_profile_result(mdffgpu_ctx *ctx, double *ms, long long *count, double *flops);
/* Diagnostic: measured fused-multiply-add throughput (TFLOP/s, 2 flops per FMA) of the
 * FP64 (precision 0) or FP32 (1) pipe of `device`; the roofline of the pair and
 * k-space kernels.  No counterpart in the reference. */
int mdffgpu_fma_peak(int device, int precision, double *tflops);

/* Force matching with adjoint gradients (no counterpart in the reference; the fit tools
 * of the reference's bin/ call its executable on perturbed inputs).  The parameter
 * vector of the polarisable silica model, types tSi and tO of the context:
 *   theta = { A, B, C (Si-O), A, B, C (O-O), q_Si (q_O = -q_Si/2), alpha_O (isotropic,
 *             A^3), b, c (Tang-Toennies damping of every declared charge-dipole
 *             damping), D (Si-O), D (O-O) (the C8 dispersion, -D/r^8) }
 * of the Born-Mayer-Huggins form without dispersion damping (lbhmft,
 * src/bhmftd.c:177-199 with f6 = f8 = 1: the damping BD of the lbhmftd variant is not a
 * parameter of this model).  mdffgpu_fit_set_params writes theta into the context's
 * tables.  mdffgpu_force_match evaluates the forces F at the converged induced dipoles
 * (a CG solver must be set), res[0] = sum_i |F_i - F_t,i|^2 and
 * res[1..MDFFGPU_FIT_NPARAM] = dL/dtheta of L = scale/2 res[0], from one adjoint
 * induced-dipole solve (FP64 adjoint arithmetic). */
#define MDFFGPU_FIT_NPARAM 12
int mdffgpu_fit_set_params(mdffgpu_ctx *ctx, int tSi, int tO, const double *theta);
int mdffgpu_force_match(mdffgpu_ctx *ctx, int tSi, int tO, const double *fx_t, const double *fy_t,
                        const double *fz_t, double scale, double *res);
/* The same over nconf contexts (independent configurations, one GPU): theta set on all,
 * targets[c] the AoS (x y z per ion) target forces of context c, res = the sums over
 * the configurations.  nthreads host threads drive the contexts' streams concurrently. */
int mdffgpu_fit_batch(mdffgpu_ctx **ctx, int nconf, int tSi, int tO, const double *theta,
                      const double *const *targets, double scale, int nthreads, double *res);
/* A fit plan: the batch above with each configuration's evaluation recorded once as a
 * CUDA graph (no counterpart in the reference).  In the graph both conjugate-gradient
 * solves (induced dipoles, adjoint) are device-controlled loops, theta is read from one
 * device buffer the plan shares across its configurations, and the loss, gradient and
 * status bits are assembled on the device, so an evaluation costs the host one copy of
 * theta, one graph launch per configuration (on its context's stream, all in flight
 * together) and one copy of the nconf results.  create: ctx[nconf] contexts on one
 * device with a CG solver set, targets[c] the AoS target forces of context c (copied to
 * the device once), scale as for mdffgpu_force_match.  eval: theta as above; res[0] =
 * sum over configurations of sum_i |F_i - F_t,i|^2, res[1..MDFFGPU_FIT_NPARAM] = the
 * summed gradient,
 * summed in configuration order; the first eval (and the first after a context's
 * precision or solver changed) records the graphs.  The contexts must not be used by
 * other calls while an eval runs; after evals each context's tables hold the last
 * theta.  mdffgpu_fit_plan_last_error: message of the last failed call. */
typedef struct mdffgpu_fit_plan mdffgpu_fit_plan;
int mdffgpu_fit_plan_create(mdffgpu_ctx **ctx, int nconf, int tSi, int tO, const double *const *targets,
                            double scale, mdffgpu_fit_plan **out);
int mdffgpu_fit_plan_eval(mdffgpu_fit_plan *plan, const double *theta, double *res);
int mdffgpu_fit_plan_destroy(mdffgpu_fit_plan *plan);
const char *mdffgpu_fit_plan_last_error(const mdffgpu_fit_plan *plan);

#ifdef __cplusplus
}
#endif
#endif
