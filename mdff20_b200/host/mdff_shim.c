/* The reference's hot-path functions, with their own names and signatures, running on
 * libmdffgpu: the drop-in for mdff20's C program.
 *
 * mdff20 has no plugin interface: its operators are void functions over process globals
 * (rx..fz, qia, dipia_ind, simuCell, u_*, pvir_*, tau_*, e_kin, e_nvt, xi/vxi, the
 * Verlet lists).  This file defines
 *
 *   gen_pbc_verletlist  src/verlet.c:54      check_verletlist  src/verlet.c:124
 *   engforce            src/field.c:352      prop_agate        src/integration.c:298
 *   multipole_ES        src/ewald.c:75       get_dipoles       src/coulombic.c:67
 *
 * with the reference's signatures and global side effects, and is linked with the
 * reference's own unmodified objects (main, parsers, run_md, outputs) whose definitions
 * of these six names are made weak (mdff20_b200/Makefile, target dropin).  One engine
 * context per process is created on the first call, after the reference's parsers and
 * init_config have filled the globals (src/mdff20.c:74-82); every call copies the host
 * globals in and the results out, so the rest of the reference program sees exactly
 * what its own functions would leave.  Failures print the engine's message and exit(-1),
 * as the reference's pError does (src/tools.c:63-67).
 *
 * Environment: MDFF20_GPU_PRECISION = fp64 (default) | mixed; MDFF20_GPU_SOLVER =
 * reference (default: the reference's algo_pim) | cg | cg-fused; MDFF20_GPU_DEVICE.
 */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mdffgpu.h"

/* the reference's headers: their globals are tentative definitions (built -fcommon) */
#include "bhmftd.h"
#include "cell.h"
#include "config.h"
#include "constants.h"
#include "coulombic.h"
#include "ewald.h"
#include "field.h"
#include "global.h"
#include "md.h"
#include "nmlj.h"
#include "pim.h"
#include "thermo.h"
#include "verlet.h"

static mdffgpu_ctx *g_ctx;
static int g_has_list;

static void die(const char *what, int rc) {
    fprintf(stderr, "ERROR mdffgpu %s (status %d): %s\n", what, rc, g_ctx ? mdffgpu_last_error(g_ctx) : "");
    exit(-1);
}

#define CK(call)                         \
    do {                                 \
        int rc_ = (call);                \
        if (rc_ != MDFFGPU_OK) die(#call, rc_); \
    } while (0)

/* the parameter block from the globals the reference's parsers left (control-file
 * units: init_md converted temp, dt, tauTberendsen and timesca_thermo in place,
 * src/md.c:124-127, so they are converted back) */
static void fill_params(mdffgpu_params *p) {
    memset(p, 0, sizeof *p);
    p->nion = nion;
    p->ntype = ntype;
    for (int t = 0; t < ntype && t < MDFFGPU_NTMAX; t++) {
        p->nionit[t] = nionit[t];
        p->massit[t] = massit[t];
        p->qit[t] = qit[t];
        for (int k = 0; k < 3; k++) p->dipit[t][k] = dipit[t][k];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) p->polit[t][a][b] = polit[t][a][b];
        for (int u = 0; u < ntype; u++) {
            p->sigmalj[t][u] = sigmalj[t][u];
            p->epslj[t][u] = epslj[t][u];
            p->plj[t][u] = plj[t][u];
            p->qlj[t][u] = qlj[t][u];
            p->Abhmftd[t][u] = Abhmftd[t][u];
            p->Bbhmftd[t][u] = Bbhmftd[t][u];
            p->Cbhmftd[t][u] = Cbhmftd[t][u];
            p->Dbhmftd[t][u] = Dbhmftd[t][u];
            p->BDbhmftd[t][u] = BDbhmftd[t][u];
            for (int v = 0; v < ntype; v++) {
                p->lpoldamping[t][u][v] = lpoldamping[t][u][v];
                p->pol_damp_b[t][u][v] = pol_damp_b[t][u][v];
                p->pol_damp_c[t][u][v] = pol_damp_c[t][u][v];
                p->pol_damp_k[t][u][v] = pol_damp_k[t][u][v];
            }
        }
    }
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) p->cell[a][b] = simuCell.A[a][b];
    p->lreduced = lreduced;
    p->lverletL = lverletL;
    p->skindiff = skindiff;
    p->cutshortrange = cutshortrange;
    p->cutlongrange = cutlongrange;
    p->lnmlj = lnmlj;
    p->trunctype = trunctype;
    p->lbhmft = lbhmft;
    p->lbhmftd = lbhmftd;
    p->lcoulombic = lcoulombic;
    p->alphaES = alphaES;
    for (int k = 0; k < 3; k++) p->kES[k] = kES[k];
    p->algo_pim = algo_pim;
    p->algo_extrapolate_dipole = algo_extrapolate_dipole;
    p->extrapolate_order = extrapolate_order;
    p->min_scf_pim_iter = min_scf_pim_iter;
    p->max_scf_pim_iter = max_scf_pim_iter;
    p->conv_tol_ind = conv_tol_ind;
    p->omegakO = omegakO;
    p->egrator = egrator;
    p->nhc_n = nhc_n;
    p->nhc_mults = nhc_mults;
    p->nhc_yosh_order = nhc_yosh_order;
    p->nequil = nequil;
    p->nequilT = nequilT;
    p->dt = dt / time_unit;
    p->temp = temp / boltz_unit;
    p->timesca_thermo = timesca_thermo / time_unit;
    p->tauTberendsen = tauTberendsen / time_unit;
}

static void ensure_ctx(void) {
    if (g_ctx) return;
    mdffgpu_params p;
    fill_params(&p);
    const char *dv = getenv("MDFF20_GPU_DEVICE");
    int rc = mdffgpu_create(&p, rx, ry, rz, vx, vy, vz, dv ? atoi(dv) : 0, &g_ctx);
    if (rc != MDFFGPU_OK) die("mdffgpu_create", rc);
    const char *pr = getenv("MDFF20_GPU_PRECISION");
    if (pr && strcmp(pr, "mixed") == 0) CK(mdffgpu_set_precision(g_ctx, MDFFGPU_MIXED));
    const char *sv = getenv("MDFF20_GPU_SOLVER");
    if (sv && strcmp(sv, "cg") == 0) CK(mdffgpu_set_pim_solver(g_ctx, MDFFGPU_PIM_CG));
    if (sv && strcmp(sv, "cg-fused") == 0) CK(mdffgpu_set_pim_solver(g_ctx, MDFFGPU_PIM_CG_FUSED));
}

/* the reference's thermodynamic globals from the engine (src/thermo.h:3-14) */
static void pull_thermo(bool kinetic) {
    mdffgpu_thermo t;
    CK(mdffgpu_get_thermo(g_ctx, &t));
    if (kinetic) {
        e_kin = t.e_kin;
        e_nvt = t.e_nvt;
    }
    u_lj = t.u_lj;
    u_bhmftd = t.u_bhmftd;
    u_coul = t.u_coul;
    u_pol = t.u_pol;
    pvir_lj = t.pvir_lj;
    pvir_bhmftd = t.pvir_bhmftd;
    pvir_coul = t.pvir_coul;
    memcpy(tau_lj, t.tau_lj, sizeof tau_lj);
    memcpy(tau_bhmftd, t.tau_bhmftd, sizeof tau_bhmftd);
    memcpy(tau_coul, t.tau_coul, sizeof tau_coul);
}

/* induced-dipole history dipia_ind[nion][6][3] (src/config.h:48), when the run has one */
static void pull_dipoles(void) {
    if (lcoulombic && lpim && dipia_ind) CK(mdffgpu_get_dipole_history(g_ctx, &dipia_ind[0][0][0]));
}

/* the host copies of the lists (verlet_nb / verlet_coul, src/verlet.h:8-16) */
static void pull_lists(void) {
    VERLETL *vl[2] = {verlet_nb, verlet_coul};
    for (int w = 0; w < 2; w++) {
        if (!vl[w] || !vl[w]->list || !vl[w]->point) continue;
        int cnt = 0;
        CK(mdffgpu_get_verletlist(g_ctx, w, vl[w]->point, vl[w]->list, VNLMAX * nion, &cnt));
    }
}

static void build_lists(void) {
    CK(mdffgpu_gen_verletlist(g_ctx));
    g_has_list = 1;
    pull_lists();
}

/* gen_pbc_verletlist (src/verlet.c:54-122) */
void gen_pbc_verletlist(void) {
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    build_lists();
}

/* check_verletlist (src/verlet.c:124-170): rebuild when the two largest displacements
 * since the last build exceed skindiff; counts rebuilds in updatevl.  The engine keeps
 * the build positions (the reference's xvl/yvl/zvl) and applies the same
 * Cartesian->direct->Cartesian round trip to the positions, which come back here. */
void check_verletlist(void) {
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    if (!g_has_list) {
        build_lists();
        updatevl += 1;
    } else {
        int rebuilt = 0;
        CK(mdffgpu_check_verletlist(g_ctx, &rebuilt));
        if (rebuilt) {
            updatevl += 1;
            pull_lists();
        }
    }
    CK(mdffgpu_get_state(g_ctx, rx, ry, rz, NULL, NULL, NULL, NULL, NULL, NULL));
}

/* engforce (src/field.c:352-407): forces, energies, virials, stress and induced dipoles */
void engforce(void) {
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    if (!g_has_list && lverletL) build_lists();
    CK(mdffgpu_engforce(g_ctx));
    CK(mdffgpu_get_state(g_ctx, NULL, NULL, NULL, NULL, NULL, NULL, fx, fy, fz));
    pull_thermo(false);
    pull_dipoles();
}

/* prop_agate (src/integration.c:298-333): one velocity-Verlet, leap-frog or
 * Nose-Hoover-chain step including its force evaluation */
void prop_agate(int step) {
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    CK(mdffgpu_set_velocities(g_ctx, vx, vy, vz));
    if (!g_has_list && lverletL) build_lists();
    CK(mdffgpu_prop_agate(g_ctx, step));
    CK(mdffgpu_get_state(g_ctx, rx, ry, rz, vx, vy, vz, fx, fy, fz));
    pull_thermo(true);
    pull_dipoles();
    if (egrator == 2 && xi && vxi) CK(mdffgpu_get_nhc(g_ctx, xi, vxi));
}

/* multipole_ES (src/ewald.c:75-348): the multipole Ewald sum of (q, mu) with the
 * reference's flag arguments; forces are added to the global fx, fy, fz as the
 * reference does.  Quadrupoles (lqua) are not part of the engine. */
void multipole_ES(double *q, double (*mu)[3], double (*theta)[3][3], double *u, double *pvir, double tau[3][3],
                  double (*ef)[3], double (*efg)[3][3], bool lqch, bool ldip, bool lqua, bool ldamp, bool do_forces,
                  bool do_stress, bool do_ef, bool do_efg, bool do_dir, bool do_rec, bool inpim, bool update_sf) {
    (void)theta;
    (void)inpim;
    (void)update_sf;
    if (lqua) {
        fprintf(stderr, "ERROR mdffgpu multipole_ES: quadrupoles are not supported\n");
        exit(-1);
    }
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    if (!g_has_list && lverletL) build_lists();
    int flags = (lqch ? MDFFGPU_ES_LQ : 0) | (ldip ? MDFFGPU_ES_LD : 0) | (ldamp ? MDFFGPU_ES_LDAMP : 0) |
                (do_forces ? MDFFGPU_ES_FORCES : 0) | (do_stress ? MDFFGPU_ES_STRESS : 0) |
                (do_ef ? MDFFGPU_ES_EF : 0) | (do_efg ? MDFFGPU_ES_EFG : 0) | (do_dir ? MDFFGPU_ES_DIR : 0) |
                (do_rec ? MDFFGPU_ES_REC : 0);
    double *f = do_forces ? malloc(sizeof(double) * 3 * (size_t)nion) : NULL;
    if (do_forces && !f) {
        fprintf(stderr, "ERROR mdffgpu multipole_ES: out of host memory\n");
        exit(-1);
    }
    CK(mdffgpu_multipole_es(g_ctx, q, &mu[0][0], flags, 0.0, u, pvir, &tau[0][0], ef ? &ef[0][0] : NULL,
                            efg ? &efg[0][0][0] : NULL, f));
    if (f) {
        for (int i = 0; i < nion; i++) {
            fx[i] += f[3 * i];
            fy[i] += f[3 * i + 1];
            fz[i] += f[3 * i + 2];
        }
        free(f);
    }
}

/* get_dipoles (src/coulombic.c:67-130): total dipoles (static + induced) and u_pol */
void get_dipoles(double (*mu)[3], double *upol) {
    ensure_ctx();
    CK(mdffgpu_set_positions(g_ctx, rx, ry, rz));
    if (!g_has_list && lverletL) build_lists();
    CK(mdffgpu_get_dipoles(g_ctx, &mu[0][0], upol));
    pull_dipoles();
}
