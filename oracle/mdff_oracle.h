/* CPU restatement of the mdff20 hot path (TEST INFRASTRUCTURE, the oracle).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
 * library, as the checker.  It restates, in plain C without process globals, the
 * reference's force field and MD step so that the CUDA engine can be compared with it
 * on any machine (the compiled reference only exists where its sources were built).
 *
 * Each function cites the reference code it follows (paths relative to the mdff20
 * repository).  Deliberate differences from the reference, none of which changes a
 * result by more than rounding:
 *  - positions are never converted Cartesian->fractional->Cartesian in place; every
 *    evaluator computes fractional coordinates into scratch (the reference round-trips
 *    rx/ry/rz through kardir/dirkar around each evaluator, src/nmlj.c:277,380);
 *  - pair sums run in a fixed serial order (the reference uses OpenMP array
 *    reductions, src/nmlj.c:288);
 *  - k-vectors are kept in generation order (the reference sorts them by |k|^2 with
 *    qsort, src/kspace.c:106-150), which only reorders the k sum.
 *  - quantities the reference leaves uninitialised (u_dir/u_rec when the direct or
 *    reciprocal part is skipped, src/ewald.c:83,232) are taken as zero.
 */
#ifndef MDFF_ORACLE_H
#define MDFF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NTMAX 16
#define ORC_ASPC_MAX 5

/* Same layout as mdffgpu_params in include/mdffgpu.h (kept separate on purpose: the
 * oracle does not depend on the product). Values are in control-file units. */
typedef struct orc_params {
    int nion, ntype;
    int nionit[ORC_NTMAX];
    double massit[ORC_NTMAX];
    double cell[3][3];
    int lreduced, lverletL;
    double skindiff, cutshortrange, cutlongrange;
    int lnmlj, trunctype;
    double sigmalj[ORC_NTMAX][ORC_NTMAX], epslj[ORC_NTMAX][ORC_NTMAX];
    double plj[ORC_NTMAX][ORC_NTMAX], qlj[ORC_NTMAX][ORC_NTMAX];
    int lbhmft, lbhmftd;
    double Abhmftd[ORC_NTMAX][ORC_NTMAX], Bbhmftd[ORC_NTMAX][ORC_NTMAX];
    double Cbhmftd[ORC_NTMAX][ORC_NTMAX], Dbhmftd[ORC_NTMAX][ORC_NTMAX];
    double BDbhmftd[ORC_NTMAX][ORC_NTMAX];
    int lcoulombic;
    double qit[ORC_NTMAX], dipit[ORC_NTMAX][3], polit[ORC_NTMAX][3][3];
    int lpoldamping[ORC_NTMAX][ORC_NTMAX][ORC_NTMAX];
    double pol_damp_b[ORC_NTMAX][ORC_NTMAX][ORC_NTMAX];
    double pol_damp_c[ORC_NTMAX][ORC_NTMAX][ORC_NTMAX];
    int pol_damp_k[ORC_NTMAX][ORC_NTMAX][ORC_NTMAX];
    double alphaES;
    int kES[3];
    int algo_pim, algo_extrapolate_dipole, extrapolate_order, min_scf_pim_iter, max_scf_pim_iter;
    double conv_tol_ind, omegakO;
    int egrator, nhc_n, nhc_mults, nhc_yosh_order, nequil, nequilT;
    double dt, temp, timesca_thermo, tauTberendsen;
} orc_params;

typedef struct orc_thermo {
    double e_kin, e_nvt, u_lj, u_bhmftd, u_coul, u_pol;
    double pvir_lj, pvir_bhmftd, pvir_coul;
    double tau_lj[9], tau_bhmftd[9], tau_coul[9];
    double utail, ptail, scf_rmsd;
    int scf_iter, nlist_builds;
} orc_thermo;

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const orc_params *p, const double *pos, const double *vel);
void orc_destroy(orc_ctx *c);
int orc_nion(const orc_ctx *c);
int orc_nk(const orc_ctx *c);

void orc_set_positions(orc_ctx *c, const double *pos);   /* (N,3) Cartesian */
void orc_set_velocities(orc_ctx *c, const double *vel);
void orc_get_state(const orc_ctx *c, double *pos, double *vel, double *force);
void orc_get_thermo(const orc_ctx *c, orc_thermo *t);
void orc_get_dipoles(const orc_ctx *c, double *mu_ind);   /* last induced dipoles (N,3) */
void orc_set_dipole_history(orc_ctx *c, const double *hist); /* (N,6,3) ASPC history */
void orc_get_dipole_history(const orc_ctx *c, double *hist);
void orc_set_nhc(orc_ctx *c, const double *xi, const double *vxi);
void orc_get_nhc(const orc_ctx *c, double *xi, double *vxi);
void orc_set_istep(orc_ctx *c, int istep);

/* gen_pbc_verletlist (src/verlet.c:54-122) from the current positions; also
 * stores the reference positions used by check_verletlist. */
int orc_gen_verletlist(orc_ctx *c);
/* returns the reference-format half list: point has nion+1 entries; list `cap` max */
int orc_get_verletlist(const orc_ctx *c, int which, int *point, int *list, int cap);
/* check_verletlist (src/verlet.c:124-170); returns 1 if the list was rebuilt */
int orc_check_verletlist(orc_ctx *c);

/* engforce (src/field.c:352-407): forces, energies, stress, induced dipoles */
int orc_engforce(orc_ctx *c);

/* multipole_ES (src/ewald.c:75-348) on given q (N) and mu (N,3); ef (N,3), efg
 * (N,9) and f (N,3) are outputs (f receives only this call's forces).  flags bits:
 * 1 lq, 2 ld, 4 ldamp, 8 do_forces, 16 do_stress, 32 do_ef, 64 do_efg, 128 do_dir,
 * 256 do_rec. alpha overrides alphaES when > 0. */
int orc_multipole_es(orc_ctx *c, const double *q, const double *mu, int flags, double alpha,
                     double *u, double *pvir, double *tau, double *ef, double *efg, double *f);

/* one prop_agate step (src/integration.c:298-333), then check_verletlist as in the
 * MD loop (src/md.c:237-241).  istep is the step index (1-based). */
int orc_md_step(orc_ctx *c, int istep);
/* nsteps steps; thermo (nsteps+1, 12) records like the harness: e_kin u_lj u_bhmftd
 * u_coul u_pol e_nvt pvir_lj pvir_bhmftd pvir_coul nlist_builds scf_iter scf_rmsd */
int orc_md(orc_ctx *c, int nsteps, double *thermo);
/* the same with step indices first .. first+nsteps-1 (the index sets the ASPC order) */
int orc_md_from(orc_ctx *c, int first, int nsteps, double *thermo);

/* get_gr (src/radial_distribution.c:180-230) of one configuration: pos (N,3) Cartesian,
 * cell9 the rows of A, typ per ion; adds ordered-pair counts to hist[nbins][nt][nt]. */
void orc_gr(int n, const double *cell9, const double *pos, const int *typ, int nt, double cutgr, double resg,
            int nbins, long long *hist);

#ifdef __cplusplus
}
#endif
#endif
