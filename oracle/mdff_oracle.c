/* CPU restatement of the mdff20 hot path -- TEST INFRASTRUCTURE (the oracle).
 * See mdff_oracle.h for the contract and the list of deliberate differences.
 * Every block cites the reference function it restates (paths inside mdff20). */
#include "mdff_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NT ORC_NTMAX
#define PI 3.1415926535897932385
#define TPI 6.2831853071795864770

struct orc_ctx {
    orc_params p;
    int n, nt;
    /* units, src/constants.c:8-18 (reduced_units, :38-45) */
    double boltz_unit, time_unit, press_unit, coul_unit, onethird, piroot;
    /* cell, src/cell.c:13-91 */
    double A[3][3], B[3][3], omega, inveOmega, inveOmegaPU, w[3];
    /* per ion */
    int *typ;
    double *mass, *invmass, *q, (*dip)[3], (*pol)[3][3], (*invpol)[3][3];
    double *rx, *ry, *rz, *vx, *vy, *vz, *fx, *fy, *fz, *rxs, *rys, *rzs;
    double *sx, *sy, *sz; /* fractional scratch */
    /* Verlet lists, src/verlet.c */
    int *nbp, *nbl, *cop, *col, cap, list_ok, nbuilds;
    double *xvl, *yvl, *zvl;
    /* short range */
    double srcutsq, lrcutsq;
    double sigsq[NT][NT], epsqp[NT][NT], fc[NT][NT], ptwo[NT][NT], qtwo[NT][NT], uc[NT][NT];
    double E_TT[9];
    int lpolar[NT];
    int lqch, ldip, lpol, ldmp, lpim;
    /* k space, src/kspace.c:64-102 */
    int nk;
    double *kx, *ky, *kz, *kk, *Ak, *kcoe;
    /* pim */
    double (*hist)[ORC_ASPC_MAX + 1][3];
    double (*mu_ind)[3];
    int istep;
    /* md */
    double dt, temp, tauT, timesca;
    double xi[16], vxi[16];
    orc_thermo th;
};

/* ------------------------------------------------------------------ cell */
static void expro(double H[3], const double *U1, const double *U2) {
    H[0] = U1[1] * U2[2] - U1[2] * U2[1];
    H[1] = U1[2] * U2[0] - U1[0] * U2[2];
    H[2] = U1[0] * U2[1] - U1[1] * U2[0];
}

/* lattice(), src/cell.c:13-91: B rows are A1xA2, A2xA0, A0xA1 over the volume; the
 * volume is sum_i B[i][0]*A[i][0] as written there (exact for orthorhombic cells). */
static void cell_setup(orc_ctx *c) {
    expro(c->B[0], c->A[1], c->A[2]);
    expro(c->B[1], c->A[2], c->A[0]);
    expro(c->B[2], c->A[0], c->A[1]);
    double omega = c->B[0][0] * c->A[0][0] + c->B[1][0] * c->A[1][0] + c->B[2][0] * c->A[2][0];
    c->omega = omega;
    c->inveOmega = 1.0 / omega;
    c->inveOmegaPU = 1.0 / (omega * c->press_unit);
    for (int i = 0; i < 3; i++)
        c->w[i] = omega / sqrt(c->B[0][i] * c->B[0][i] + c->B[1][i] * c->B[1][i] + c->B[2][i] * c->B[2][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c->B[i][j] = c->B[i][j] * c->inveOmega;
}

/* kardir, src/cell.c:125-143, into scratch (no in-place round trip) */
static void to_frac(orc_ctx *c) {
    for (int i = 0; i < c->n; i++) {
        double x = c->rx[i], y = c->ry[i], z = c->rz[i];
        c->sx[i] = x * c->B[0][0] + y * c->B[0][1] + z * c->B[0][2];
        c->sy[i] = x * c->B[1][0] + y * c->B[1][1] + z * c->B[1][2];
        c->sz[i] = x * c->B[2][0] + y * c->B[2][1] + z * c->B[2][2];
    }
}

/* pbc, src/pbc.c:7-14: nearest image by nearbyint in fractional space, then x A */
static inline void pbc(const orc_ctx *c, double *x, double *y, double *z) {
    double sx = *x - nearbyint(*x);
    double sy = *y - nearbyint(*y);
    double sz = *z - nearbyint(*z);
    *x = sx * c->A[0][0] + sy * c->A[1][0] + sz * c->A[2][0];
    *y = sx * c->A[0][1] + sy * c->A[1][1] + sz * c->A[2][1];
    *z = sx * c->A[0][2] + sy * c->A[1][2] + sz * c->A[2][2];
}

/* ------------------------------------------------------------------ TT damping */
/* TT_damping_functions, src/tt_damp.c:16-32; E_TT[k] = 1/k!, src/tt_damp.c:34-40 */
static inline void tt_damp(const orc_ctx *c, double b, double cc, double r, double *f, double *fd, int order) {
    double br = b * r;
    double expbdr = exp(-br) * cc;
    double ff = c->E_TT[order];
    for (int k = order - 1; k > -1; k--) ff = ff * br + c->E_TT[k];
    *f = 1.0 - ff * expbdr;
    *fd = c->E_TT[order] * pow(br, order) * expbdr * b;
}

/* ------------------------------------------------------------------ set-up */
orc_ctx *orc_create(const orc_params *p, const double *pos, const double *vel) {
    orc_ctx *c = calloc(1, sizeof(*c));
    c->p = *p;
    int n = c->n = p->nion;
    c->nt = p->ntype;
    if (p->lreduced) { /* src/constants.c:38-45, applied by check_global src/global.c:80-82 */
        c->boltz_unit = 1.0; c->time_unit = 1.0; c->press_unit = 1.0; c->coul_unit = 1.0;
    } else {
        c->boltz_unit = 8.61734229648141E-05;
        c->time_unit = 98.2269514139276;
        c->press_unit = 0.00624150964712042;
        c->coul_unit = 14.3996441494161;
    }
    c->onethird = 1. / 3.0;
    c->piroot = sqrt(PI);
    memcpy(c->A, p->cell, sizeof(c->A));
    cell_setup(c);

    c->typ = malloc(n * sizeof(int));
    c->mass = malloc(n * sizeof(double));
    c->invmass = malloc(n * sizeof(double));
    c->q = calloc(n, sizeof(double));
    c->dip = calloc(n, sizeof(*c->dip));
    c->pol = calloc(n, sizeof(*c->pol));
    c->invpol = calloc(n, sizeof(*c->invpol));
    double **arrs[] = {&c->rx, &c->ry, &c->rz, &c->vx, &c->vy, &c->vz, &c->fx, &c->fy, &c->fz,
                       &c->rxs, &c->rys, &c->rzs, &c->sx, &c->sy, &c->sz, &c->xvl, &c->yvl, &c->zvl};
    for (unsigned k = 0; k < sizeof(arrs) / sizeof(arrs[0]); k++) *arrs[k] = calloc(n, sizeof(double));
    c->hist = calloc(n, sizeof(*c->hist));
    c->mu_ind = calloc(n, sizeof(*c->mu_ind));

    /* field flags: read_field src/field.c:97-108, info_field src/field.c:195-221 */
    for (int it = 0; it < c->nt; it++) {
        c->lpolar[it] = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (p->polit[it][i][j] != 0.0) c->lpolar[it] = 1;
        if (p->qit[it] != 0.0) c->lqch = 1;
        for (int j = 0; j < 3; j++) {
            if (p->dipit[it][j] != 0.0) c->ldip = 1;
            for (int k = 0; k < 3; k++)
                if (p->polit[it][j][k] != 0.0) c->lpol = 1;
        }
    }
    /* damping tables: the same in-place symmetrisation loop as src/field.c:209-219 */
    for (int it = 0; it < c->nt; it++)
        for (int jt = 0; jt < c->nt; jt++)
            for (int kt = 0; kt < c->nt; kt++) {
                if (c->p.lpoldamping[jt][it][kt]) c->ldmp = 1;
                c->p.lpoldamping[jt][kt][it] = c->p.lpoldamping[jt][it][kt];
                c->p.pol_damp_b[jt][kt][it] = c->p.pol_damp_b[jt][it][kt];
                c->p.pol_damp_c[jt][kt][it] = c->p.pol_damp_c[jt][it][kt];
                c->p.pol_damp_k[jt][kt][it] = c->p.pol_damp_k[jt][it][kt];
            }
    c->lpim = 0;
    for (int it = 0; it < c->nt; it++)
        if (c->lpolar[it]) c->lpim = 1; /* is_pim, src/field.c:338-343 */
    /* E_TT, src/tt_damp.c:34-40 */
    c->E_TT[0] = 1.0;
    for (int i = 1; i < 9; i++) c->E_TT[i] = c->E_TT[i - 1] / ((double)i);

    /* init_config, src/config.c:124-198 */
    int cc = 0;
    for (int it = 0; it < c->nt; it++) {
        for (int ia = cc; ia < cc + p->nionit[it]; ia++) {
            c->typ[ia] = it;
            c->mass[ia] = p->massit[it];
            c->invmass[ia] = 1.0 / p->massit[it];
            if (p->lcoulombic) {
                c->q[ia] = p->qit[it];
                for (int i = 0; i < 3; i++) c->dip[ia][i] = p->dipit[it][i];
            }
            if (p->lcoulombic && c->lpolar[it]) {
                /* invertmatrix3x3 (src/config.c:171): Gauss-Jordan, 1/a_ii when diagonal */
                double m[3][6];
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) {
                        c->pol[ia][i][j] = p->polit[it][i][j];
                        m[i][j] = p->polit[it][i][j];
                        m[i][j + 3] = (i == j);
                    }
                for (int col = 0; col < 3; col++) {
                    int piv = col;
                    for (int r = col + 1; r < 3; r++)
                        if (fabs(m[r][col]) > fabs(m[piv][col])) piv = r;
                    if (m[piv][col] == 0.0) continue;
                    for (int j = 0; j < 6 && piv != col; j++) {
                        double t = m[col][j]; m[col][j] = m[piv][j]; m[piv][j] = t;
                    }
                    double inv = 1.0 / m[col][col];
                    for (int j = 0; j < 6; j++) m[col][j] = (j == col) ? 1.0 : m[col][j] * inv;
                    for (int r = 0; r < 3; r++) {
                        if (r == col || m[r][col] == 0.0) continue;
                        double f = m[r][col];
                        for (int j = 0; j < 6; j++) m[r][j] -= f * m[col][j];
                    }
                }
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) c->invpol[ia][i][j] = m[i][j + 3];
            }
        }
        cc += p->nionit[it];
    }
    orc_set_positions(c, pos);
    if (vel) orc_set_velocities(c, vel);

    c->srcutsq = p->cutshortrange * p->cutshortrange;
    c->lrcutsq = p->cutlongrange * p->cutlongrange;
    c->cap = 500 * n; /* VNLMAX, src/verlet.h:3 */
    if (p->lverletL) {
        c->nbp = calloc(n + 1, sizeof(int));
        c->nbl = calloc(c->cap, sizeof(int));
        c->cop = calloc(n + 1, sizeof(int));
        c->col = calloc(c->cap, sizeof(int));
    }

    /* init_nmlj, src/nmlj.c:123-251 */
    if (p->lnmlj) {
        double one16 = (1.0 / 6.0);
        double two16 = pow(2.0, one16);
        double srcut3 = c->srcutsq * p->cutshortrange;
        for (int it = 0; it < c->nt; it++)
            for (int jt = 0; jt < c->nt; jt++) {
                if (jt >= it) {
                    c->p.plj[jt][it] = c->p.plj[it][jt];
                    c->p.qlj[jt][it] = c->p.qlj[it][jt];
                    c->p.sigmalj[jt][it] = c->p.sigmalj[it][jt];
                    c->p.epslj[jt][it] = c->p.epslj[it][jt];
                }
                double pp = c->p.plj[it][jt], qq = c->p.qlj[it][jt];
                c->epsqp[it][jt] = c->p.epslj[it][jt] / (qq - pp);
                c->sigsq[it][jt] = two16 * two16 * c->p.sigmalj[it][jt] * c->p.sigmalj[it][jt];
                c->fc[it][jt] = (pp * qq * c->epsqp[it][jt]) / c->sigsq[it][jt];
                c->ptwo[it][jt] = pp * 0.5;
                c->qtwo[it][jt] = qq * 0.5;
                double epsppqq = c->epsqp[it][jt], ppqq = pp * qq;
                double sr2 = c->sigsq[it][jt] / c->srcutsq, sr = sqrt(sr2);
                double srp = pow(sr, pp), srq = pow(sr, qq);
                c->uc[it][jt] = epsppqq * (pp * srq - qq * srp);
                double ut = epsppqq * (pp * srq / (qq - 3.0) - qq * srp / (pp - 3.0));
                double pt = ppqq * epsppqq * (srq / (qq - 3.0) - srp / (pp - 3.0));
                ut *= srcut3 * TPI;
                pt *= srcut3 * TPI;
                if (p->nionit[it] != 0 && p->nionit[jt] != 0) {
                    c->th.utail += ut * p->nionit[it] * p->nionit[jt] * c->inveOmega;
                    c->th.ptail += pt * p->nionit[it] * p->nionit[jt] * c->inveOmega;
                }
            }
        c->th.ptail = c->th.ptail / (c->press_unit * 3.0);
    }
    /* init_bhmftd, src/bhmftd.c:93-115: symmetric tables */
    if (p->lbhmft || p->lbhmftd) {
        for (int it = 0; it < c->nt; it++)
            for (int jt = it; jt < c->nt; jt++) {
                c->p.Abhmftd[jt][it] = c->p.Abhmftd[it][jt];
                c->p.Bbhmftd[jt][it] = c->p.Bbhmftd[it][jt];
                c->p.Cbhmftd[jt][it] = c->p.Cbhmftd[it][jt];
                c->p.Dbhmftd[jt][it] = c->p.Dbhmftd[it][jt];
                c->p.BDbhmftd[jt][it] = c->p.BDbhmftd[it][jt];
            }
    }
    /* init_kspace + set_param_kmesh, src/kspace.c:14-41,64-102 (generation order) */
    if (p->lcoulombic) {
        int km0 = p->kES[0], km1 = p->kES[1], km2 = p->kES[2];
        int nk = km2 + km1 * (2 * km2 + 1) + km0 * (2 * km1 + 1) * (2 * km2 + 1);
        c->nk = nk;
        c->kx = malloc(nk * sizeof(double)); c->ky = malloc(nk * sizeof(double));
        c->kz = malloc(nk * sizeof(double)); c->kk = malloc(nk * sizeof(double));
        c->Ak = malloc(nk * sizeof(double)); c->kcoe = malloc(nk * sizeof(double));
        double alpha2 = p->alphaES * p->alphaES;
        int ik = 0;
        for (int nx = 0; nx < km0 + 1; nx++) {
            int nymin = (nx == 0) ? 0 : -km1;
            for (int ny = nymin; ny < km1 + 1; ny++) {
                int nzmin = (nx == 0 && ny == 0) ? 1 : -km2;
                for (int nz = nzmin; nz < km2 + 1; nz++) {
                    double kx = TPI * ((double)nx * c->B[0][0] + (double)ny * c->B[0][1] + (double)nz * c->B[0][2]);
                    double ky = TPI * ((double)nx * c->B[1][0] + (double)ny * c->B[1][1] + (double)nz * c->B[1][2]);
                    double kz = TPI * ((double)nx * c->B[2][0] + (double)ny * c->B[2][1] + (double)nz * c->B[2][2]);
                    double kk = kx * kx + ky * ky + kz * kz;
                    c->kx[ik] = kx; c->ky[ik] = ky; c->kz[ik] = kz; c->kk[ik] = kk;
                    c->Ak[ik] = exp(-kk * 0.25 / alpha2) / kk;
                    c->kcoe[ik] = 2.0 * (1.0 / kk + 1.0 / alpha2 / 4.0);
                    ik++;
                }
            }
        }
    }
    /* md parameters, check_md src/md.c:120-141 */
    c->tauT = p->tauTberendsen;
    if (p->nequil > 0 && c->tauT == 0.0) c->tauT = p->dt;
    c->temp = p->temp * c->boltz_unit;
    c->dt = p->dt * c->time_unit;
    c->tauT *= c->time_unit;
    c->timesca = p->timesca_thermo * c->time_unit;
    return c;
}

void orc_destroy(orc_ctx *c) {
    if (!c) return;
    void *ptrs[] = {c->typ, c->mass, c->invmass, c->q, c->dip, c->pol, c->invpol, c->rx, c->ry, c->rz,
                    c->vx, c->vy, c->vz, c->fx, c->fy, c->fz, c->rxs, c->rys, c->rzs, c->sx, c->sy,
                    c->sz, c->xvl, c->yvl, c->zvl, c->hist, c->mu_ind, c->nbp, c->nbl, c->cop, c->col,
                    c->kx, c->ky, c->kz, c->kk, c->Ak, c->kcoe};
    for (unsigned k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) free(ptrs[k]);
    free(c);
}

int orc_nion(const orc_ctx *c) { return c->n; }
int orc_nk(const orc_ctx *c) { return c->nk; }
void orc_set_istep(orc_ctx *c, int istep) { c->istep = istep; }

/* read_config's wrap into the box (src/config.c:442-444) is done by the caller */
void orc_set_positions(orc_ctx *c, const double *pos) {
    for (int i = 0; i < c->n; i++) {
        c->rx[i] = pos[3 * i]; c->ry[i] = pos[3 * i + 1]; c->rz[i] = pos[3 * i + 2];
    }
}
void orc_set_velocities(orc_ctx *c, const double *vel) {
    for (int i = 0; i < c->n; i++) {
        c->vx[i] = vel[3 * i]; c->vy[i] = vel[3 * i + 1]; c->vz[i] = vel[3 * i + 2];
    }
}
void orc_get_state(const orc_ctx *c, double *pos, double *vel, double *force) {
    for (int i = 0; i < c->n; i++) {
        if (pos) { pos[3 * i] = c->rx[i]; pos[3 * i + 1] = c->ry[i]; pos[3 * i + 2] = c->rz[i]; }
        if (vel) { vel[3 * i] = c->vx[i]; vel[3 * i + 1] = c->vy[i]; vel[3 * i + 2] = c->vz[i]; }
        if (force) { force[3 * i] = c->fx[i]; force[3 * i + 1] = c->fy[i]; force[3 * i + 2] = c->fz[i]; }
    }
}
void orc_get_thermo(const orc_ctx *c, orc_thermo *t) { *t = c->th; }
void orc_get_dipoles(const orc_ctx *c, double *mu) { memcpy(mu, c->mu_ind, 3 * sizeof(double) * c->n); }
void orc_set_dipole_history(orc_ctx *c, const double *h) { memcpy(c->hist, h, sizeof(*c->hist) * c->n); }
void orc_get_dipole_history(const orc_ctx *c, double *h) { memcpy(h, c->hist, sizeof(*c->hist) * c->n); }
void orc_set_nhc(orc_ctx *c, const double *xi, const double *vxi) {
    for (int i = 0; i < c->p.nhc_n && i < 16; i++) { c->xi[i] = xi[i]; c->vxi[i] = vxi[i]; }
}
void orc_get_nhc(const orc_ctx *c, double *xi, double *vxi) {
    for (int i = 0; i < c->p.nhc_n && i < 16; i++) { xi[i] = c->xi[i]; vxi[i] = c->vxi[i]; }
}

/* ------------------------------------------------------------------ Verlet lists */
/* gen_pbc_verletlist, src/verlet.c:54-122: O(N^2) scan, half list by the parity rule
 * (i>j, i+j even) or (i<j, i+j odd), inclusive test rij^2 <= (rc+skin)^2 */
static int gen_lists(orc_ctx *c) {
    double cutnb = c->p.cutshortrange + c->p.skindiff;
    double cutco = c->p.cutlongrange + c->p.skindiff;
    double rsq_nb = cutnb * cutnb, rsq_co = cutco * cutco;
    int inb = 0, ico = 0;
    for (int ia = 0; ia < c->n; ia++) {
        int knb = 0, kco = 0;
        for (int ja = 0; ja < c->n; ja++) {
            if (((ia > ja) && ((ia + ja) % 2 == 0)) || ((ia < ja) && ((ia + ja) % 2 != 0))) {
                double x = c->sx[ia] - c->sx[ja], y = c->sy[ia] - c->sy[ja], z = c->sz[ia] - c->sz[ja];
                pbc(c, &x, &y, &z);
                double r2 = x * x + y * y + z * z;
                if (r2 <= rsq_nb) {
                    if (inb >= c->cap) return -1;
                    c->nbl[inb++] = ja;
                    knb++;
                }
                if (r2 <= rsq_co) {
                    if (ico >= c->cap) return -1;
                    c->col[ico++] = ja;
                    kco++;
                }
            }
        }
        c->nbp[ia] = inb - knb;
        c->cop[ia] = ico - kco;
    }
    c->nbp[c->n] = inb;
    c->cop[c->n] = ico;
    return 0;
}

int orc_gen_verletlist(orc_ctx *c) {
    if (!c->p.lverletL) return -2;
    to_frac(c);
    int rc = gen_lists(c);
    for (int i = 0; i < c->n; i++) { c->xvl[i] = c->sx[i]; c->yvl[i] = c->sy[i]; c->zvl[i] = c->sz[i]; }
    c->list_ok = (rc == 0);
    c->nbuilds++;
    c->th.nlist_builds = c->nbuilds;
    return rc;
}

int orc_get_verletlist(const orc_ctx *c, int which, int *point, int *list, int cap) {
    const int *pp = which ? c->cop : c->nbp;
    const int *ll = which ? c->col : c->nbl;
    if (!pp) return -2;
    memcpy(point, pp, (c->n + 1) * sizeof(int));
    int cnt = pp[c->n];
    if (cnt > cap) return -1;
    memcpy(list, ll, cnt * sizeof(int));
    return cnt;
}

/* check_verletlist, src/verlet.c:124-170 */
int orc_check_verletlist(orc_ctx *c) {
    to_frac(c);
    double m1 = 0.0, m2 = 0.0;
    for (int ia = 0; ia < c->n; ia++) {
        double x = c->sx[ia] - c->xvl[ia], y = c->sy[ia] - c->yvl[ia], z = c->sz[ia] - c->zvl[ia];
        pbc(c, &x, &y, &z);
        double d = sqrt(x * x + y * y + z * z);
        if (d > m1) { m2 = m1; m1 = d; }
        else if (d > m2) m2 = d;
    }
    if (m1 + m2 > c->p.skindiff) {
        gen_lists(c);
        for (int i = 0; i < c->n; i++) { c->xvl[i] = c->sx[i]; c->yvl[i] = c->sy[i]; c->zvl[i] = c->sz[i]; }
        c->nbuilds++;
        c->th.nlist_builds = c->nbuilds;
        return 1;
    }
    return 0;
}

/* pair loop bounds shared by all evaluators (src/nmlj.c:293-309) */
#define FOR_PAIRS(LISTP, LISTL)                                               \
    int jb = c->p.lverletL ? LISTP[ia] : 0;                                   \
    int je = c->p.lverletL ? LISTP[ia + 1] : c->n;                            \
    for (int j1 = jb; j1 < je; j1++) {                                        \
        int ja = c->p.lverletL ? LISTL[j1] : j1;                              \
        if (!(((ja > ia) && !c->p.lverletL) || ((ja != ia) && c->p.lverletL))) \
            continue;

/* ------------------------------------------------------------------ n-m LJ */
/* engforce_nmlj_pbc, src/nmlj.c:254-385 (addtruncU :28-36: quadratic gives 0) */
static void nmlj(orc_ctx *c, double *u, double *pvir, double tau[9]) {
    double uu = 0.0, tt[6] = {0};
    double *gx = calloc(c->n, sizeof(double)), *gy = calloc(c->n, sizeof(double)), *gz = calloc(c->n, sizeof(double));
    to_frac(c);
    for (int ia = 0; ia < c->n; ia++) {
        FOR_PAIRS(c->nbp, c->nbl)
            double x = c->sx[ia] - c->sx[ja], y = c->sy[ia] - c->sy[ja], z = c->sz[ia] - c->sz[ja];
            pbc(c, &x, &y, &z);
            double r2 = x * x + y * y + z * z;
            if (r2 < c->srcutsq) {
                int p1 = c->typ[ia], p2 = c->typ[ja];
                double sr2 = c->sigsq[p1][p2] / r2;
                double srp = pow(sr2, c->ptwo[p1][p2]);
                double srq = pow(sr2, c->qtwo[p1][p2]);
                if (c->p.trunctype == 0)
                    uu += c->epsqp[p1][p2] * (c->p.plj[p1][p2] * srq - c->p.qlj[p1][p2] * srp);
                else if (c->p.trunctype == 1)
                    uu += c->epsqp[p1][p2] * (c->p.plj[p1][p2] * srq - c->p.qlj[p1][p2] * srp) - c->uc[p1][p2];
                double wij = c->fc[p1][p2] * (srq - srp) * sr2;
                double fxij = wij * x, fyij = wij * y, fzij = wij * z;
                gx[ia] += fxij; gy[ia] += fyij; gz[ia] += fzij;
                gx[ja] += -fxij; gy[ja] += -fyij; gz[ja] += -fzij;
                tt[0] += (x * fxij + x * fxij) * 0.5;
                tt[1] += (x * fyij + y * fxij) * 0.5;
                tt[2] += (x * fzij + z * fxij) * 0.5;
                tt[3] += (y * fyij + y * fyij) * 0.5;
                tt[4] += (y * fzij + z * fyij) * 0.5;
                tt[5] += (z * fzij + z * fzij) * 0.5;
            }
        }
    }
    for (int i = 0; i < c->n; i++) { c->fx[i] += gx[i]; c->fy[i] += gy[i]; c->fz[i] += gz[i]; }
    free(gx); free(gy); free(gz);
    double full[9] = {tt[0], tt[1], tt[2], tt[1], tt[3], tt[4], tt[2], tt[4], tt[5]};
    *pvir = 0.0;
    for (int k = 0; k < 9; k++) tau[k] = full[k] * c->inveOmegaPU;
    for (int i = 0; i < 3; i++) *pvir += tau[4 * i] * c->onethird;
    *u = uu;
}

/* ------------------------------------------------------------------ BHMFT(D) */
/* engforce_bhmftd_pbc, src/bhmftd.c:117-271 */
static void bhmftd(orc_ctx *c, double *u, double *pvir, double tau[9]) {
    double uu = 0.0, tt[6] = {0};
    double *gx = calloc(c->n, sizeof(double)), *gy = calloc(c->n, sizeof(double)), *gz = calloc(c->n, sizeof(double));
    to_frac(c);
    for (int ia = 0; ia < c->n; ia++) {
        FOR_PAIRS(c->nbp, c->nbl)
            int p1 = c->typ[ia], p2 = c->typ[ja];
            if (c->p.Abhmftd[p1][p2] == 0.0) continue;
            double x = c->sx[ia] - c->sx[ja], y = c->sy[ia] - c->sy[ja], z = c->sz[ia] - c->sz[ja];
            pbc(c, &x, &y, &z);
            double r2 = x * x + y * y + z * z;
            if (r2 < c->srcutsq) {
                double ir2 = 1.0 / r2, d = sqrt(r2);
                double erh = c->p.Abhmftd[p1][p2] * exp(-c->p.Bbhmftd[p1][p2] * d);
                double ir6 = ir2 * ir2 * ir2;
                double ir8 = ir6 * ir2;
                ir6 = ir6 * c->p.Cbhmftd[p1][p2];
                ir8 = ir8 * c->p.Dbhmftd[p1][p2];
                double f6, f8, fd6, fd8, ir6d, ir8d;
                if (c->p.lbhmftd) {
                    tt_damp(c, c->p.BDbhmftd[p1][p2], 1.0, d, &f6, &fd6, 6);
                    tt_damp(c, c->p.BDbhmftd[p1][p2], 1.0, d, &f8, &fd8, 8);
                    ir6d = ir6 * f6;
                    ir8d = ir8 * f8;
                } else {
                    fd6 = 0.0; fd8 = 0.0; ir6d = ir6; ir8d = ir8;
                }
                double ir7 = 6.0 * ir6d / d, ir9 = 8.0 * ir8d / d;
                uu += erh - ir6d - ir8d;
                double wij = c->p.Bbhmftd[p1][p2] * erh - ir7 - ir9 + ir6 * fd6 + ir8 * fd8;
                wij = wij / d;
                double fxij = wij * x, fyij = wij * y, fzij = wij * z;
                gx[ia] += fxij; gy[ia] += fyij; gz[ia] += fzij;
                gx[ja] += -fxij; gy[ja] += -fyij; gz[ja] += -fzij;
                tt[0] += (x * fxij + x * fxij) * 0.5;
                tt[1] += (x * fyij + y * fxij) * 0.5;
                tt[2] += (x * fzij + z * fxij) * 0.5;
                tt[3] += (y * fyij + y * fyij) * 0.5;
                tt[4] += (y * fzij + z * fyij) * 0.5;
                tt[5] += (z * fzij + z * fzij) * 0.5;
            }
        }
    }
    for (int i = 0; i < c->n; i++) { c->fx[i] += gx[i]; c->fy[i] += gy[i]; c->fz[i] += gz[i]; }
    free(gx); free(gy); free(gz);
    double full[9] = {tt[0], tt[1], tt[2], tt[1], tt[3], tt[4], tt[2], tt[4], tt[5]};
    *pvir = 0.0;
    for (int k = 0; k < 9; k++) tau[k] = full[k] * c->inveOmegaPU;
    for (int i = 0; i < 3; i++) *pvir += tau[4 * i] * c->onethird;
    *u = uu;
}

/* ------------------------------------------------------------------ Ewald, direct */
/* multipole_ES_dir, src/ewald.c:353-871, charges and dipoles (T0..T3; the T4/T5
 * tensors of the reference feed no output for charges and dipoles). */
static void ewald_dir(orc_ctx *c, const double *q, const double (*mu)[3], double alpha, int lq, int ld,
                      int lcouldamp, int do_forces, int do_stress, int do_ef, int do_efg, double *u,
                      double (*ef)[3], double (*efg)[9], double (*f)[3], double tau[9]) {
    double alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha5 = alpha3 * alpha2;
    double uu = 0.0, tt[3][3] = {{0}};
    int lqd = lq && ld;
    to_frac(c);
    for (int ia = 0; ia < c->n; ia++) {
        double qi = q[ia];
        int qch_i = (qi != 0.0), dip_i = 0, ita = c->typ[ia];
        double mui[3];
        for (int i = 0; i < 3; i++) { mui[i] = mu[ia][i]; if (mui[i] != 0.0) dip_i = 1; }
        FOR_PAIRS(c->cop, c->col)
            double qj = q[ja];
            int qch_j = (qj != 0.0), dip_j = 0, jta = c->typ[ja];
            double muj[3], fij[3] = {0, 0, 0};
            for (int i = 0; i < 3; i++) { muj[i] = mu[ja][i]; if (muj[i] != 0.0) dip_j = 1; }
            double qij = qi * qj;
            double r[3] = {c->sx[ia] - c->sx[ja], c->sy[ia] - c->sy[ja], c->sz[ia] - c->sz[ja]};
            pbc(c, &r[0], &r[1], &r[2]);
            double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (d2 > c->lrcutsq) continue;
            double d = sqrt(d2), d3 = d2 * d, d5 = d3 * d2;
            double dm1 = 1.0 / d, dm3 = dm1 / d2, dm5 = dm3 / d2, dm7 = dm5 / d2;
            int ldamp = (c->p.lpoldamping[ita][ita][jta] || c->p.lpoldamping[jta][ita][jta]) && lcouldamp;
            double fd1 = 1.0, fd2 = 1.0, fdd1 = 0.0, fdd2 = 0.0;
            if (ldamp) {
                tt_damp(c, c->p.pol_damp_b[ita][ita][jta], c->p.pol_damp_c[ita][ita][jta], d, &fd1, &fdd1,
                        c->p.pol_damp_k[ita][ita][jta]);
                tt_damp(c, c->p.pol_damp_b[jta][ita][jta], c->p.pol_damp_c[jta][ita][jta], d, &fd2, &fdd2,
                        c->p.pol_damp_k[jta][ita][jta]);
            }
            double expon = exp(-alpha2 * d2) / c->piroot;
            double F0 = erfc(alpha * d);
            double F1 = F0 + 2.0 * alpha * d * expon;
            double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
            double F3 = F2 + 8.0 * alpha5 * d5 * expon / 15.0;
            double F1d1 = -fd1 + 1.0, F1d2 = -fd2 + 1.0;
            double F2d1 = F1d1 + (d / 3.0) * fdd1, F2d2 = F1d2 + (d / 3.0) * fdd2;
            double T0 = dm1 * F0, T1[3], T1D1[3] = {0}, T1D2[3] = {0};
            for (int i = 0; i < 3; i++) {
                T1[i] = -r[i] * dm3;
                if (ldamp) { T1D1[i] = T1[i] * F1d1; T1D2[i] = T1[i] * F1d2; }
                T1[i] *= F1;
            }
            double F2_dm5 = 3.0 * F2 * dm5, F2d1_dm5 = 3.0 * F2d1 * dm5, F2d2_dm5 = 3.0 * F2d2 * dm5;
            double F1_dm3 = F1 * dm3, F1d1_dm3 = F1d1 * dm3, F1d2_dm3 = F1d2 * dm3;
            double T2[3][3], T2D1[3][3] = {{0}}, T2D2[3][3] = {{0}}, T3[3][3][3] = {{{0}}};
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++) {
                    T2[j][k] = r[j] * r[k] * F2_dm5;
                    if (j == k) T2[j][j] += -F1_dm3;
                    if (ldamp) {
                        T2D1[j][k] = r[j] * r[k] * F2d1_dm5;
                        T2D2[j][k] = r[j] * r[k] * F2d2_dm5;
                        if (j == k) { T2D1[j][j] += -F1d1_dm3; T2D2[j][j] += -F1d2_dm3; }
                    }
                }
            if (ld) {
                double F3_dm7 = F3 * dm7 * 15.0;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++) {
                            T3[i][j][k] = -r[i] * r[j] * r[k] * F3_dm7;
                            if (i == j) T3[i][j][k] += r[k] * F2_dm5;
                            if (i == k) T3[i][j][k] += r[j] * F2_dm5;
                            if (j == k) T3[i][j][k] += r[i] * F2_dm5;
                        }
            }
            /* charge-charge, src/ewald.c:703-731 */
            if (lq && (qch_i || qch_j)) {
                uu += qij * T0;
                for (int i = 0; i < 3; i++) {
                    if (do_ef) {
                        ef[ia][i] += -qj * T1[i];
                        ef[ja][i] += qi * T1[i];
                        if (ldamp) { ef[ia][i] += qj * T1D1[i]; ef[ja][i] += -qi * T1D2[i]; }
                    }
                    if (do_forces) fij[i] = qij * T1[i];
                    if (do_efg)
                        for (int j = 0; j < 3; j++) {
                            efg[ia][3 * i + j] += -qj * T2[i][j];
                            efg[ja][3 * i + j] += -qi * T2[i][j];
                        }
                }
            }
            /* dipole-dipole, src/ewald.c:737-761 */
            if (ld && dip_i && dip_j) {
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) {
                        uu += -mui[i] * T2[i][j] * muj[j];
                        if (do_ef) { ef[ia][i] += muj[j] * T2[i][j]; ef[ja][i] += mui[j] * T2[i][j]; }
                        if (do_efg || do_forces)
                            for (int k = 0; k < 3; k++) {
                                efg[ia][3 * i + j] += muj[k] * T3[i][j][k];
                                efg[ja][3 * i + j] += -mui[k] * T3[i][j][k];
                                fij[k] += -mui[i] * T3[i][k][j] * muj[j];
                            }
                    }
            }
            /* charge-dipole, src/ewald.c:767-812 */
            if (lqd && (dip_i || dip_j)) {
                for (int i = 0; i < 3; i++) {
                    uu += -qi * T1[i] * muj[i];
                    uu += qj * T1[i] * mui[i];
                    if (do_forces)
                        for (int j = 0; j < 3; j++) {
                            fij[j] += -qi * T2[j][i] * muj[i];
                            fij[j] += qj * T2[j][i] * mui[i];
                        }
                    if (ldamp) {
                        uu += qi * T1D2[i] * muj[i];
                        uu += -qj * T1D1[i] * mui[i];
                        if (do_forces)
                            for (int j = 0; j < 3; j++) {
                                fij[j] += -qj * T2D1[i][j] * mui[i];
                                fij[j] += qi * T2D2[i][j] * muj[i];
                            }
                    }
                }
            }
            if (do_forces)
                for (int i = 0; i < 3; i++) { f[ia][i] += -fij[i]; f[ja][i] += fij[i]; }
            if (do_stress)
                for (int i = 0; i < 3; i++)
                    for (int j = i; j < 3; j++) tt[i][j] += -(r[i] * fij[j] + r[j] * fij[i]);
        }
    }
    *u = uu;
    if (do_stress) {
        tt[1][0] = tt[0][1]; tt[2][0] = tt[0][2]; tt[2][1] = tt[1][2];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) tau[3 * i + j] = 0.5 * tt[i][j] * c->inveOmegaPU;
    }
}

/* ------------------------------------------------------------------ Ewald, reciprocal */
/* multipole_ES_rec, src/ewald.c:876-1051, with struct_fact / charge_density_* /
 * struct_fact_rhon (src/kspace.c:154-302): the same cos/sin(k.r) from Cartesian r. */
static void ewald_rec(orc_ctx *c, const double *q, const double (*mu)[3], int lq, int ld, int do_forces,
                      int do_stress, int do_ef, int do_efg, double *u, double (*ef)[3], double (*efg)[9],
                      double (*f)[3], double tau[9]) {
    double uu = 0.0, tt[3][3] = {{0}};
    double *ck = malloc(c->n * sizeof(double)), *sk = malloc(c->n * sizeof(double));
    for (int ik = 0; ik < c->nk; ik++) {
        if (c->kk[ik] == 0.0) continue;
        double kx = c->kx[ik], ky = c->ky[ik], kz = c->kz[ik], Ak = c->Ak[ik], kcoe = c->kcoe[ik];
        double rR = 0.0, rI = 0.0;
        for (int ia = 0; ia < c->n; ia++) {
            double kr = (kx * c->rx[ia] + ky * c->ry[ia] + kz * c->rz[ia]);
            ck[ia] = cos(kr);
            sk[ia] = sin(kr);
            if (lq) { rR += q[ia] * ck[ia]; rI += q[ia] * sk[ia]; }
            if (ld) {
                double kmu = (mu[ia][0] * kx + mu[ia][1] * ky + mu[ia][2] * kz);
                rR += -kmu * sk[ia];
                rI += kmu * ck[ia];
            }
        }
        double str = (rR * rR + rI * rI) * Ak;
        uu += str;
        for (int ia = 0; ia < c->n; ia++) {
            double recarg = Ak * (rI * ck[ia] - rR * sk[ia]);
            double recarg2 = Ak * (rR * ck[ia] + rI * sk[ia]);
            double fxij = kx * recarg, fyij = ky * recarg, fzij = kz * recarg;
            if (do_ef) { ef[ia][0] += -fxij; ef[ia][1] += -fyij; ef[ia][2] += -fzij; }
            if (do_efg) {
                efg[ia][0] += kx * kx * recarg2;
                efg[ia][4] += ky * ky * recarg2;
                efg[ia][8] += kz * kz * recarg2;
                efg[ia][1] += kx * ky * recarg2;
                efg[ia][2] += kx * kz * recarg2;
                efg[ia][5] += ky * kz * recarg2;
            }
            if (do_forces) {
                f[ia][0] += -q[ia] * fxij;
                f[ia][1] += -q[ia] * fyij;
                f[ia][2] += -q[ia] * fzij;
                if (ld) {
                    double kmu = (mu[ia][0] * kx + mu[ia][1] * ky + mu[ia][2] * kz) * recarg2;
                    f[ia][0] += kx * kmu;
                    f[ia][1] += ky * kmu;
                    f[ia][2] += kz * kmu;
                }
            }
        }
        if (do_stress) { /* the dipolar k-space stress term is absent, src/ewald.c:999-1006 */
            tt[0][0] += (1.0 - kcoe * kx * kx) * str;
            tt[0][1] += -kcoe * kx * ky * str;
            tt[0][2] += -kcoe * kx * kz * str;
            tt[1][1] += (1.0 - kcoe * ky * ky) * str;
            tt[1][2] += -kcoe * ky * kz * str;
            tt[2][2] += (1.0 - kcoe * kz * kz) * str;
        }
    }
    free(ck); free(sk);
    double ttpiV = 2.0 * TPI * c->inveOmega, tfpiV = 2.0 * ttpiV;
    *u = uu * ttpiV;
    for (int ia = 0; ia < c->n; ia++) {
        for (int j = 0; j < 3; j++) { f[ia][j] *= tfpiV; ef[ia][j] *= tfpiV; }
        for (int k = 0; k < 9; k++) efg[ia][k] *= tfpiV;
    }
    tt[1][0] = tt[0][1]; tt[2][0] = tt[0][2]; tt[2][1] = tt[1][2];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) tau[3 * i + j] = tt[i][j] * ttpiV * c->inveOmegaPU;
}

/* ------------------------------------------------------------------ multipole_ES */
/* multipole_ES, src/ewald.c:75-348: dir + rec + self, electrostatic units.  As in
 * the reference, the reciprocal EFG is computed when do_ef is set (src/ewald.c:169)
 * and `f` ACCUMULATES the forces (x coul_unit). */
static void multipole_es(orc_ctx *c, const double *q, const double (*mu)[3], double alpha, int lq, int ld,
                         int lcouldamp, int do_forces, int do_stress, int do_ef, int do_efg, int do_dir,
                         int do_rec, double *u, double *pvir, double tau[9], double (*ef)[3],
                         double (*efg)[9], double (*f)[3]) {
    int n = c->n;
    double u_dir = 0.0, u_rec = 0.0, tau_dir[9] = {0}, tau_rec[9] = {0};
    double (*efd)[3] = calloc(n, sizeof(*efd)), (*efr)[3] = calloc(n, sizeof(*efr));
    double (*egd)[9] = calloc(n, sizeof(*egd)), (*egr)[9] = calloc(n, sizeof(*egr));
    double (*fd)[3] = calloc(n, sizeof(*fd)), (*fr)[3] = calloc(n, sizeof(*fr));
    if (do_dir)
        ewald_dir(c, q, mu, alpha, lq, ld, lcouldamp, do_forces, do_stress, do_ef, do_efg, &u_dir, efd, egd,
                  fd, tau_dir);
    if (do_rec) ewald_rec(c, q, mu, lq, ld, do_forces, do_stress, do_ef, do_ef, &u_rec, efr, egr, fr, tau_rec);
    /* self terms, src/ewald.c:193-226 */
    double qsq = 0.0, musq = 0.0;
    for (int ia = 0; ia < n; ia++) {
        qsq += q[ia] * q[ia];
        musq += mu[ia][0] * mu[ia][0] + mu[ia][1] * mu[ia][1] + mu[ia][2] * mu[ia][2];
    }
    double alpha2 = alpha * alpha, selfa = alpha / c->piroot, selfa2 = 2.0 * selfa * alpha2 / 3.0;
    double u_self = -selfa * qsq + -selfa2 * musq;
    *u = (u_dir + u_rec + u_self) * c->coul_unit;
    for (int ia = 0; ia < n; ia++) {
        for (int i = 0; i < 3; i++) {
            ef[ia][i] = 2.0 * selfa2 * mu[ia][i];
            if (do_dir) ef[ia][i] += efd[ia][i];
            if (do_rec) ef[ia][i] += efr[ia][i];
            for (int j = 0; j < 3; j++) {
                efg[ia][3 * i + j] = (i == j) ? -2.0 * selfa2 * q[ia] : 0.0;
                if (do_dir) efg[ia][3 * i + j] += egd[ia][3 * i + j];
                if (do_rec) efg[ia][3 * i + j] += egr[ia][3 * i + j];
            }
        }
        for (int i = 0; i < 3; i++) {
            if (do_dir) f[ia][i] += fd[ia][i] * c->coul_unit;
        }
        for (int i = 0; i < 3; i++) {
            if (do_rec) f[ia][i] += fr[ia][i] * c->coul_unit;
        }
    }
    if (do_stress) {
        for (int k = 0; k < 9; k++) {
            tau[k] = 0.0;
            if (do_dir) tau[k] += tau_dir[k] * c->coul_unit;
            if (do_rec) tau[k] += tau_rec[k] * c->coul_unit;
        }
    }
    *pvir = 0.0;
    for (int i = 0; i < 3; i++) *pvir += tau[4 * i] * c->onethird;
    free(efd); free(efr); free(egd); free(egr); free(fd); free(fr);
}

int orc_multipole_es(orc_ctx *c, const double *q, const double *mu, int flags, double alpha, double *u,
                     double *pvir, double *tau, double *ef, double *efg, double *f) {
    if (!c->p.lcoulombic) return -2;
    if (c->p.lverletL && !c->list_ok) return -3;
    double a = alpha > 0.0 ? alpha : c->p.alphaES;
    for (int k = 0; k < 9; k++) tau[k] = 0.0;
    for (int k = 0; k < 3 * c->n; k++) f[k] = 0.0;
    multipole_es(c, q, (const double (*)[3])mu, a, flags & 1, (flags >> 1) & 1, (flags >> 2) & 1,
                 (flags >> 3) & 1, (flags >> 4) & 1, (flags >> 5) & 1, (flags >> 6) & 1, (flags >> 7) & 1,
                 (flags >> 8) & 1, u, pvir, tau, (double (*)[3])ef, (double (*)[9])efg, (double (*)[3])f);
    return 0;
}

/* ------------------------------------------------------------------ PIM */
/* induced_moment, src/pim.c:617-641: mu_i = sum_j pol[j][i] E_j on polarisable ions */
static void induced_moment(orc_ctx *c, double (*mu)[3], const double (*ef)[3]) {
    for (int ia = 0; ia < c->n; ia++) {
        if (!c->lpolar[c->typ[ia]]) continue;
        for (int i = 0; i < 3; i++) {
            mu[ia][i] = 0.0;
            for (int j = 0; j < 3; j++) mu[ia][i] += c->pol[ia][j][i] * ef[ia][j];
        }
    }
}

/* get_upol, src/pim.c:145-161 */
static double get_upol(orc_ctx *c, const double (*mu)[3]) {
    double up = 0.0;
    for (int ia = 0; ia < c->n; ia++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) up += mu[ia][i] * c->invpol[ia][i][j] * mu[ia][j];
    return up * 0.5;
}

/* get_rmsd_mu, src/pim.c:431-449 */
static double get_rmsd(orc_ctx *c, const double (*mu)[3], const double (*ef)[3]) {
    double r = 0.0;
    int npol = 0;
    for (int ia = 0; ia < c->n; ia++) {
        if (!c->lpolar[c->typ[ia]]) continue;
        npol++;
        for (int i = 0; i < 3; i++)
            if (c->pol[ia][i][i] != 0.0) {
                double e = mu[ia][i] / c->pol[ia][i][i] - ef[ia][i];
                r += e * e;
            }
    }
    return sqrt(r / (double)npol);
}

/* extrapolate_dipole_aspc, src/pim.c:314-424.  Kolafa ASPC coefficients B_k, W for
 * the order in effect.  The reference raises the order inside its ion loop, so that
 * during the first steps ions >= 1 read coefficients it never set; here every ion
 * uses the order in effect for the step (the converged dipoles do not depend on the
 * predictor).  The history shift is the reference's. */
static void aspc(orc_ctx *c, double (*mu)[3], const double (*ef)[3], int key) {
    int ord = c->p.extrapolate_order, e;
    if (c->istep >= ord + 1) e = ord;
    else e = (!c->istep) ? 0 : c->istep - 1;
    static const double Bt[6][6] = {{1.0},
                                    {2.0, -1.0},
                                    {2.5, -2.0, 0.5},
                                    {2.8, -2.8, 1.2, -0.2},
                                    {3.0, -24.0 / 7.0, 27.0 / 14.0, -4.0 / 7.0, 1.0 / 14.0},
                                    {22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0}};
    static const double Wt[6] = {0.0, 2.0 / 3.0, 0.6, 4.0 / 7.0, 5.0 / 9.0, 6.0 / 11.0};
    if (key == 1) {
        int es = (e != ord) ? e + 1 : e;
        for (int ia = 0; ia < c->n; ia++) {
            for (int i = 0; i < 3; i++) mu[ia][i] = 0.0;
            for (int k = 0; k < e + 1; k++)
                for (int i = 0; i < 3; i++) mu[ia][i] += Bt[e][k] * c->hist[ia][k][i];
            for (int k = es; k > 0; k--)
                for (int i = 0; i < 3; i++) c->hist[ia][k][i] = c->hist[ia][k - 1][i];
        }
    } else {
        double (*save)[3] = malloc(c->n * sizeof(*save));
        memcpy(save, mu, c->n * sizeof(*save));
        induced_moment(c, mu, ef);
        double W = Wt[e];
        for (int ia = 0; ia < c->n; ia++)
            for (int i = 0; i < 3; i++) mu[ia][i] = mu[ia][i] * W + (1.0 - W) * save[ia][i];
        free(save);
    }
}

/* momentpolaSCF, src/pim.c:177-306 */
static void pim_scf(orc_ctx *c, double (*mu_ind)[3], double *upol) {
    int n = c->n;
    double (*ef)[3] = calloc(n, sizeof(*ef)), (*efs)[3] = calloc(n, sizeof(*efs));
    double (*efi)[3] = calloc(n, sizeof(*efi)), (*eg)[9] = calloc(n, sizeof(*eg));
    double (*fdum)[3] = calloc(n, sizeof(*fdum)), *zero = calloc(n, sizeof(double)), tdum[9] = {0};
    double us, ui, pd, uupol = 0.0;
    int ldip_static = c->ldip || c->lpol;
    multipole_es(c, c->q, (const double (*)[3])c->dip, c->p.alphaES, c->lqch, ldip_static, c->ldmp, 0, 0, 1, 0,
                 1, 1, &us, &pd, tdum, efs, eg, fdum);
    memcpy(ef, efs, n * sizeof(*ef));
    int iscf = 0;
    double rmsd = DBL_MAX;
    while (((iscf < c->p.max_scf_pim_iter) && (rmsd > c->p.conv_tol_ind)) || (iscf < c->p.min_scf_pim_iter)) {
        memset(mu_ind, 0, n * sizeof(*mu_ind));
        if (!iscf) aspc(c, mu_ind, (const double (*)[3])ef, 1);
        else induced_moment(c, mu_ind, (const double (*)[3])ef);
        uupol = get_upol(c, (const double (*)[3])mu_ind);
        multipole_es(c, zero, (const double (*)[3])mu_ind, c->p.alphaES, 0, 1, 0, 0, 0, 1, 0, 1, 1, &ui, &pd,
                     tdum, efi, eg, fdum);
        for (int ia = 0; ia < n; ia++)
            for (int i = 0; i < 3; i++) ef[ia][i] = efs[ia][i] + efi[ia][i];
        if (!iscf) aspc(c, mu_ind, (const double (*)[3])ef, 2);
        rmsd = get_rmsd(c, (const double (*)[3])mu_ind, (const double (*)[3])ef);
        iscf++;
    }
    for (int ia = 0; ia < n; ia++)
        for (int i = 0; i < 3; i++) c->hist[ia][0][i] = mu_ind[ia][i];
    *upol = uupol * c->coul_unit;
    c->th.scf_iter = iscf;
    c->th.scf_rmsd = rmsd;
    free(ef); free(efs); free(efi); free(eg); free(fdum); free(zero);
}

/* induced_moment_inner_kO, src/pim.c:647-748: real-space-only relaxation with
 * alpha_Ewald = 0.001 (src/pim.c:694) and omega mixing */
static void inner_ko(orc_ctx *c, double (*mu)[3], const double (*ef_ext)[3]) {
    int n = c->n;
    double (*prev)[3] = calloc(n, sizeof(*prev)), (*zv)[3] = calloc(n, sizeof(*zv));
    double (*eft)[3] = calloc(n, sizeof(*eft)), (*efi)[3] = calloc(n, sizeof(*efi));
    double (*eg)[9] = calloc(n, sizeof(*eg)), (*fdum)[3] = calloc(n, sizeof(*fdum));
    double *zero = calloc(n, sizeof(double)), tdum[9] = {0}, ud, pd;
    memcpy(eft, ef_ext, n * sizeof(*eft));
    double rmsd_ext = get_rmsd(c, (const double (*)[3])zv, (const double (*)[3])eft);
    induced_moment(c, mu, (const double (*)[3])eft);
    double om = c->p.omegakO;
    for (int ia = 0; ia < n; ia++)
        for (int i = 0; i < 3; i++) mu[ia][i] *= om;
    int it = 0;
    double rmsd_in = DBL_MAX;
    while ((it <= 20) && (rmsd_in > 0.1 * rmsd_ext)) {
        it++;
        memcpy(prev, mu, n * sizeof(*prev));
        multipole_es(c, zero, (const double (*)[3])mu, 0.001, 0, 1, 0, 0, 0, 1, 0, 1, 0, &ud, &pd, tdum, efi, eg,
                     fdum);
        for (int ia = 0; ia < n; ia++)
            for (int i = 0; i < 3; i++) eft[ia][i] = ef_ext[ia][i] + efi[ia][i];
        rmsd_in = get_rmsd(c, (const double (*)[3])mu, (const double (*)[3])eft);
        induced_moment(c, mu, (const double (*)[3])eft);
        for (int ia = 0; ia < n; ia++)
            for (int i = 0; i < 3; i++) mu[ia][i] = (1 - om) * prev[ia][i] + om * mu[ia][i];
    }
    free(prev); free(zv); free(eft); free(efi); free(eg); free(fdum); free(zero);
}

/* momentpolaSCFkO, src/pim.c:457-603 */
static void pim_scfko(orc_ctx *c, double (*mu_ind)[3], double *upol) {
    int n = c->n;
    double (*ef)[3] = calloc(n, sizeof(*ef)), (*efs)[3] = calloc(n, sizeof(*efs));
    double (*efi)[3] = calloc(n, sizeof(*efi)), (*eg)[9] = calloc(n, sizeof(*eg));
    double (*find)[3] = calloc(n, sizeof(*find)), (*dmu)[3] = calloc(n, sizeof(*dmu));
    double (*fdum)[3] = calloc(n, sizeof(*fdum)), *zero = calloc(n, sizeof(double)), tdum[9] = {0};
    double us, ui, pd, uupol = 0.0;
    int ldip_static = c->ldip || c->lpol;
    multipole_es(c, c->q, (const double (*)[3])c->dip, c->p.alphaES, c->lqch, ldip_static, c->ldmp, 0, 0, 1, 0,
                 1, 1, &us, &pd, tdum, efs, eg, fdum);
    memcpy(ef, efs, n * sizeof(*ef));
    memcpy(find, efs, n * sizeof(*find));
    int iscf = 0;
    double rmsd = DBL_MAX;
    while (((iscf < c->p.max_scf_pim_iter) && (rmsd > c->p.conv_tol_ind)) || (iscf < c->p.min_scf_pim_iter)) {
        if ((!iscf) && (c->istep > 1)) aspc(c, mu_ind, (const double (*)[3])ef, 1);
        else {
            inner_ko(c, dmu, (const double (*)[3])find);
            for (int ia = 0; ia < n; ia++)
                for (int i = 0; i < 3; i++) mu_ind[ia][i] += dmu[ia][i];
        }
        uupol = get_upol(c, (const double (*)[3])mu_ind);
        multipole_es(c, zero, (const double (*)[3])mu_ind, c->p.alphaES, 0, 1, 0, 0, 0, 1, 0, 1, 1, &ui, &pd,
                     tdum, efi, eg, fdum);
        for (int ia = 0; ia < n; ia++)
            for (int i = 0; i < 3; i++) ef[ia][i] = efs[ia][i] + efi[ia][i];
        if (!iscf) aspc(c, mu_ind, (const double (*)[3])ef, 2);
        rmsd = get_rmsd(c, (const double (*)[3])mu_ind, (const double (*)[3])ef);
        for (int ia = 0; ia < n; ia++)
            for (int i = 0; i < 3; i++) {
                if (!c->lpolar[c->typ[ia]]) continue;
                find[ia][i] = ef[ia][i] - mu_ind[ia][i] * c->invpol[ia][i][i];
            }
        iscf++;
    }
    for (int ia = 0; ia < n; ia++)
        for (int i = 0; i < 3; i++) c->hist[ia][0][i] = mu_ind[ia][i];
    *upol = uupol * c->coul_unit;
    c->th.scf_iter = iscf;
    c->th.scf_rmsd = rmsd;
    free(ef); free(efs); free(efi); free(eg); free(find); free(dmu); free(fdum); free(zero);
}

/* ------------------------------------------------------------------ engforce */
/* engforce, src/field.c:352-407, with get_dipoles src/coulombic.c:67-130 */
int orc_engforce(orc_ctx *c) {
    int n = c->n;
    if (c->p.lverletL && !c->list_ok) return -3;
    for (int i = 0; i < n; i++) { c->fx[i] = 0.0; c->fy[i] = 0.0; c->fz[i] = 0.0; }
    if (c->p.lnmlj) nmlj(c, &c->th.u_lj, &c->th.pvir_lj, c->th.tau_lj);
    if (c->p.lbhmft || c->p.lbhmftd) bhmftd(c, &c->th.u_bhmftd, &c->th.pvir_bhmftd, c->th.tau_bhmftd);
    if (c->p.lcoulombic) {
        double (*mu)[3] = malloc(n * sizeof(*mu));
        memcpy(mu, c->dip, n * sizeof(*mu));
        if (c->lpol) {
            double (*mi)[3] = calloc(n, sizeof(*mi));
            if (c->p.algo_pim == 1) pim_scfko(c, mi, &c->th.u_pol);
            else pim_scf(c, mi, &c->th.u_pol);
            for (int ia = 0; ia < n; ia++)
                for (int i = 0; i < 3; i++) mu[ia][i] += mi[ia][i];
            memcpy(c->mu_ind, mi, n * sizeof(*mi));
            free(mi);
        }
        double (*ef)[3] = calloc(n, sizeof(*ef)), (*efg)[9] = calloc(n, sizeof(*efg));
        double (*f)[3] = calloc(n, sizeof(*f));
        for (int i = 0; i < n; i++) { f[i][0] = c->fx[i]; f[i][1] = c->fy[i]; f[i][2] = c->fz[i]; }
        int ldip_final = c->ldip || c->lpol;
        multipole_es(c, c->q, (const double (*)[3])mu, c->p.alphaES, c->lqch, ldip_final, c->ldmp, 1, 1, 0, 0, 1,
                     1, &c->th.u_coul, &c->th.pvir_coul, c->th.tau_coul, ef, efg, f);
        for (int i = 0; i < n; i++) { c->fx[i] = f[i][0]; c->fy[i] = f[i][1]; c->fz[i] = f[i][2]; }
        free(mu); free(ef); free(efg); free(f);
    }
    return 0;
}

/* ------------------------------------------------------------------ integrators */
static double calc_kin(const orc_ctx *c) { /* src/kinetic.c:68-75 */
    double kin = 0.0;
    for (int ia = 0; ia < c->n; ia++)
        kin += (c->vx[ia] * c->vx[ia] + c->vy[ia] * c->vy[ia] + c->vz[ia] * c->vz[ia]) * c->mass[ia];
    return kin * 0.5;
}

/* prop_velocity_verlet, src/integration.c:22-63 */
static int prop_vv(orc_ctx *c) {
    int n = c->n;
    double *fs = malloc(3 * n * sizeof(double));
    double dtsq2 = c->dt * c->dt * 0.5, dt2 = c->dt * 0.5;
    for (int ia = 0; ia < n; ia++) {
        fs[3 * ia] = c->fx[ia]; fs[3 * ia + 1] = c->fy[ia]; fs[3 * ia + 2] = c->fz[ia];
        c->rx[ia] += c->vx[ia] * c->dt + (c->fx[ia] * dtsq2) * c->invmass[ia];
        c->ry[ia] += c->vy[ia] * c->dt + (c->fy[ia] * dtsq2) * c->invmass[ia];
        c->rz[ia] += c->vz[ia] * c->dt + (c->fz[ia] * dtsq2) * c->invmass[ia];
    }
    int rc = orc_engforce(c);
    double kin = 0.0;
    for (int ia = 0; ia < n; ia++) {
        c->vx[ia] += (fs[3 * ia] + c->fx[ia]) * dt2 * c->invmass[ia];
        c->vy[ia] += (fs[3 * ia + 1] + c->fy[ia]) * dt2 * c->invmass[ia];
        c->vz[ia] += (fs[3 * ia + 2] + c->fz[ia]) * dt2 * c->invmass[ia];
        kin += (c->vx[ia] * c->vx[ia] + c->vy[ia] * c->vy[ia] + c->vz[ia] * c->vz[ia]) * c->mass[ia];
    }
    c->th.e_kin = kin * 0.5;
    free(fs);
    return rc;
}

/* prop_leap_frog, src/integration.c:93-137 (r(t-dt) starts at zero as in
 * alloc_config, src/config.c:61-70) */
static int prop_lf(orc_ctx *c) {
    int rc = orc_engforce(c);
    double dtsq = c->dt * c->dt, idt = 0.5 / c->dt, kin = 0.0;
    for (int ia = 0; ia < c->n; ia++) {
        double ux = 2.0 * c->rx[ia] - c->rxs[ia] + c->fx[ia] * dtsq * c->invmass[ia];
        double uy = 2.0 * c->ry[ia] - c->rys[ia] + c->fy[ia] * dtsq * c->invmass[ia];
        double uz = 2.0 * c->rz[ia] - c->rzs[ia] + c->fz[ia] * dtsq * c->invmass[ia];
        c->vx[ia] = idt * (ux - c->rxs[ia]);
        c->vy[ia] = idt * (uy - c->rys[ia]);
        c->vz[ia] = idt * (uz - c->rzs[ia]);
        kin += (c->vx[ia] * c->vx[ia] + c->vy[ia] * c->vy[ia] + c->vz[ia] * c->vz[ia]) * c->mass[ia];
        c->rxs[ia] = c->rx[ia]; c->rys[ia] = c->ry[ia]; c->rzs[ia] = c->rz[ia];
        c->rx[ia] = ux; c->ry[ia] = uy; c->rz[ia] = uz;
    }
    c->th.e_kin = kin * 0.5;
    return rc;
}

/* chain_nhcn, src/integration.c:189-294, including its loop bounds: the second
 * thermostat sweep stops at nhc_n-2 (src/integration.c:269) */
static void chain_nhcn(orc_ctx *c, double *kin, const double *Q, double L) {
    int nn = c->p.nhc_n, yo = c->p.nhc_yosh_order, mu = c->p.nhc_mults;
    double w[7] = {0}, dty[7] = {0}, G[16] = {0};
    double temp = c->temp;
    double *vxi = c->vxi, *xi = c->xi;
    switch (yo) {
    case 1: w[0] = 1.0; break;
    case 3:
        w[0] = 1.0 / (2.0 - pow(2.0, 1.0 / 3.0));
        w[1] = 1.0 - 2.0 * w[0];
        w[2] = w[0];
        break;
    case 5:
        w[0] = 1.0 / (4.0 - pow(4, 1.0 / 3.0));
        w[1] = w[0]; w[2] = w[0]; w[3] = w[0];
        w[4] = 1.0 - 4.0 * w[0];
        break;
    case 7:
        w[0] = .78451361047756; w[1] = .235573213359357; w[2] = -1.17767998417887;
        w[3] = 1.0 - 2.0 * (w[0] + w[1] + w[2]);
        w[4] = w[2]; w[5] = w[1]; w[6] = w[0];
        break;
    default: break;
    }
    for (int i = 0; i < yo && i < 7; i++) dty[i] = w[i] * c->dt / ((double)mu);
    double s = 1.0;
    G[0] = 2.0 * (*kin) - L * temp;
    for (int k = 0; k < mu; k++) {
        for (int j = 0; j < yo && j < 7; j++) {
            double dts = dty[j], dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
            G[nn - 1] = (vxi[nn - 2] * vxi[nn - 2] / Q[nn - 2] - temp);
            vxi[nn - 1] += G[nn - 1] * dts4;
            for (int inh = nn - 2; inh > -1; inh--) {
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] += G[inh] * dts4;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
            }
            s *= exp(-vxi[0] * dts2 / Q[0]);
            for (int i = 0; i < nn; i++) xi[i] += vxi[i] * dts2 / Q[i];
            G[0] = 2.0 * (*kin) * s * s - L * temp;
            for (int inh = 0; inh < nn - 2; inh++) {
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] += G[inh] * dts4;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                G[inh + 1] = (vxi[inh] * vxi[inh] / Q[inh] - temp);
            }
            vxi[nn - 1] += G[nn - 1] * dts4;
        }
    }
    double kk = 0.0;
    for (int ia = 0; ia < c->n; ia++) {
        c->vx[ia] *= s; c->vy[ia] *= s; c->vz[ia] *= s;
        kk += (c->vx[ia] * c->vx[ia] + c->vy[ia] * c->vy[ia] + c->vz[ia] * c->vz[ia]) * c->mass[ia];
    }
    *kin = kk * 0.5;
}

/* prop_pos_vel_verlet, src/integration.c:66-90 */
static int prop_pos_vel(orc_ctx *c, double *kin) {
    double dt2 = c->dt * 0.5;
    for (int ia = 0; ia < c->n; ia++) {
        c->vx[ia] += c->fx[ia] * dt2 * c->invmass[ia];
        c->vy[ia] += c->fy[ia] * dt2 * c->invmass[ia];
        c->vz[ia] += c->fz[ia] * dt2 * c->invmass[ia];
        c->rx[ia] += c->vx[ia] * c->dt;
        c->ry[ia] += c->vy[ia] * c->dt;
        c->rz[ia] += c->vz[ia] * c->dt;
    }
    int rc = orc_engforce(c);
    double k = 0.0;
    for (int ia = 0; ia < c->n; ia++) {
        c->vx[ia] += c->fx[ia] * dt2 * c->invmass[ia];
        c->vy[ia] += c->fy[ia] * dt2 * c->invmass[ia];
        c->vz[ia] += c->fz[ia] * dt2 * c->invmass[ia];
        k += (c->vx[ia] * c->vx[ia] + c->vy[ia] * c->vy[ia] + c->vz[ia] * c->vz[ia]) * c->mass[ia];
    }
    *kin = k * 0.5;
    return rc;
}

/* nhcn, src/integration.c:140-182 */
static int nhcn(orc_ctx *c) {
    double L = 3.0 * (double)c->n, Q[16];
    int nn = c->p.nhc_n;
    for (int i = 0; i < nn; i++) Q[i] = c->timesca * c->timesca * c->temp;
    Q[0] = Q[0] * L;
    double kin = calc_kin(c);
    chain_nhcn(c, &kin, Q, L);
    int rc = prop_pos_vel(c, &kin);
    chain_nhcn(c, &kin, Q, L);
    c->th.e_kin = calc_kin(c);
    double nvt1 = L * c->temp * c->xi[0], nvt2 = c->vxi[0] * c->vxi[0] * 0.5 / Q[0], nvt3 = 0.0, nvt4 = 0.0;
    for (int i = 1; i < nn; i++) {
        nvt3 += c->vxi[i] * c->vxi[i] * 0.5 / Q[i];
        nvt4 += c->temp * c->xi[i];
    }
    c->th.e_nvt = nvt1 + nvt2 + nvt3 + nvt4;
    return rc;
}

/* prop_agate (src/integration.c:298-333) then check_verletlist (src/md.c:237-241) */
int orc_md_step(orc_ctx *c, int istep) {
    c->istep = istep;
    int rc;
    switch (c->p.egrator) {
    case 0: rc = prop_lf(c); break;
    case 2: rc = nhcn(c); break;
    default: rc = prop_vv(c); break;
    }
    if (rc) return rc;
    if (c->p.lverletL) orc_check_verletlist(c);
    return 0;
}

static void rec_thermo(const orc_ctx *c, double *t) {
    t[0] = c->th.e_kin; t[1] = c->th.u_lj; t[2] = c->th.u_bhmftd; t[3] = c->th.u_coul;
    t[4] = c->th.u_pol; t[5] = c->th.e_nvt; t[6] = c->th.pvir_lj; t[7] = c->th.pvir_bhmftd;
    t[8] = c->th.pvir_coul; t[9] = (double)c->nbuilds; t[10] = (double)c->th.scf_iter; t[11] = c->th.scf_rmsd;
}

/* the run_md loop (src/md.c:196-247): forces at t=0, then nsteps steps with step indices
 * first, first+1, ... (the index drives the ASPC order, src/pim.c:321-333) */
int orc_md_from(orc_ctx *c, int first, int nsteps, double *thermo) {
    if (c->p.lverletL && !c->list_ok) {
        int rc = orc_gen_verletlist(c);
        if (rc) return rc;
    }
    c->istep = 0;
    c->th.e_kin = calc_kin(c);
    int rc = orc_engforce(c);
    if (rc) return rc;
    if (thermo) rec_thermo(c, thermo);
    for (int s = 1; s <= nsteps; s++) {
        rc = orc_md_step(c, first + s - 1);
        if (rc) return rc;
        if (thermo) rec_thermo(c, thermo + 12 * s);
    }
    return 0;
}

int orc_md(orc_ctx *c, int nsteps, double *thermo) { return orc_md_from(c, 1, nsteps, thermo); }

/* ------------------------------------------------------------------ g(r) */
/* get_gr, src/radial_distribution.c:180-230, for one configuration: every ordered pair
 * (ia, ja != ia) closer than cutgr adds 1 to hist[(int)(r/resg)][type ia][type ja].
 * (The reference also tallies every pair into [0][0]; callers add that themselves.) */
void orc_gr(int n, const double *cell9, const double *pos, const int *typ, int nt, double cutgr, double resg,
            int nbins, long long *hist) {
    orc_ctx *c = calloc(1, sizeof *c);
    memcpy(c->A, cell9, 9 * sizeof(double));
    c->press_unit = 1.0;
    cell_setup(c);
    double *s = malloc(3 * (size_t)n * sizeof(double));
    for (int i = 0; i < n; i++) {
        double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        s[3 * i] = x * c->B[0][0] + y * c->B[0][1] + z * c->B[0][2];
        s[3 * i + 1] = x * c->B[1][0] + y * c->B[1][1] + z * c->B[1][2];
        s[3 * i + 2] = x * c->B[2][0] + y * c->B[2][1] + z * c->B[2][2];
    }
    double cut2 = cutgr * cutgr;
    for (int ia = 0; ia < n; ia++)
        for (int ja = 0; ja < n; ja++) {
            if (ja == ia) continue;
            double x = s[3 * ia] - s[3 * ja], y = s[3 * ia + 1] - s[3 * ja + 1], z = s[3 * ia + 2] - s[3 * ja + 2];
            pbc(c, &x, &y, &z);
            double rijsq = x * x + y * y + z * z;
            if (rijsq < cut2) {
                int igr = (int)(sqrt(rijsq) / resg);
                if (igr >= 0 && igr < nbins) hist[((size_t)igr * nt + typ[ia]) * nt + typ[ja]]++;
            }
        }
    free(s);
    free(c);
}
