/* Control-file scans and parameter set-up of the reference, restated.
 *
 * Each module of the reference opens the control file and reads it token by token
 * with fscanf("%s"); a token equal to one of the module's keywords makes it read the
 * values that follow with fscanf %d / %lf / %s (src/global.c:13-60, src/md.c:29-98,
 * src/field.c:31-183, src/nmlj.c:39-107, src/bhmftd.c:26-90, src/pim.c:28-69).  Here
 * each module is a table of keywords with a value kind; one scanner runs a table over
 * the file.  The scanner keeps the reference's semantics:
 *   - every table entry is compared with the current token in table order, and a
 *     string-valued entry replaces the token by its value (as the reference reads the
 *     value into the same buffer), so a later entry sees the value;
 *   - read_field lists epsw twice (src/field.c:159-164): the field table does too, so
 *     "epsw" reads two numbers when two follow;
 *   - per-type keys (massit, qit, dipit, quadit, polit) fill types in the order they
 *     appear; pair tables read the upper triangle it <= jt;
 *   - a value that fails to convert leaves the parameter unchanged.
 * Out-of-range type indices and values outside a keyword's allowed strings are errors,
 * as in check_string (src/tools.c:56-69).
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mdffhost.h"

#define NT MDFFGPU_NTMAX

/* constants.c:8-18 and the allowed strings of src/constants.c:20-35 */
static const double BOLTZ_UNIT = 8.61734229648141e-05;
static const double TIME_UNIT = 98.2269514139276;
static const double PRESS_UNIT = 0.00624150964712042;
static const double COUL_UNIT = 14.3996441494161;
static const char *const BOOL_WORDS[] = {"yes", "no", "y", "n", "Y", "N", "Yes", "No",
                                         "true", "false", "t", "f", "T", "F", "True", "False"};
static const char *const FPOSFF_WORDS[] = {"rnn", "rvn", "rvf"};
static const char *const INTEGRATOR_WORDS[] = {"nve-lf", "nve-vv", "nvt-nhcn"};
static const char *const TRUNC_WORDS[] = {"no", "linear", "quadratic"};
static const char *const ALGO_PIM_WORDS[] = {"scf", "scfkO"};
static const char *const EXTRAPOLATE_WORDS[] = {"poly", "aspc"};
#define NWORDS(a) ((int)(sizeof(a) / sizeof((a)[0])))

int mdffh_fail(mdffh_run *run, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(run->err, sizeof run->err, fmt, ap);
    va_end(ap);
    return -1;
}

enum kind {
    K_BOOL,      /* one of BOOL_WORDS: even index true (check_boolstring, src/tools.c:78) */
    K_INT,       /* %d */
    K_DBL,       /* %lf */
    K_WORD,      /* one of `words`, stored as its index */
    K_INT3,      /* three %d (kES) */
    K_UPPER,     /* %lf for it <= jt of a [NT][NT] table */
    K_TYPE_D,    /* %lf into slot (*count)++ of a per-type array */
    K_TYPE_V3,   /* three %lf into row (*count)++ of [NT][3] */
    K_TYPE_M9,   /* nine %lf into row (*count)++ of [NT][3][3] */
    K_DAMP_BOOL, /* "%d %d %d %s": [t][i][j] of an int [NT][NT][NT] table */
    K_DAMP_D,    /* "%d %d %d" then %lf */
    K_DAMP_I,    /* "%d %d %d" then %d */
    K_FLAG       /* no value: sets an int to 1 */
};

struct key {
    const char *name;
    enum kind kind;
    void *dst;
    const char *const *words;
    int nwords;
    int *count;
};

static int word_index(mdffh_run *run, const char *label, const char *tok, const char *const *words, int n,
                      int *out) {
    int hit = -1;
    for (int k = 0; k < n; k++)
        if (strcmp(tok, words[k]) == 0) hit = k;
    if (hit < 0) return mdffh_fail(run, "value not allowed in input file: %s %s", label, tok);
    *out = hit;
    return 0;
}

static int type_triple(mdffh_run *run, const char *label, int t, int i, int j) {
    if (t < 0 || i < 0 || j < 0 || t >= NT || i >= NT || j >= NT)
        return mdffh_fail(run, "%s: type index out of range (%d %d %d)", label, t, i, j);
    return 0;
}

/* One value of entry k after its keyword; tok is the scan buffer (may be replaced). */
static int read_value(mdffh_run *run, FILE *fp, const struct key *k, char *tok, int ntype) {
    int t = 0, i = 0, j = 0;
    switch (k->kind) {
    case K_FLAG:
        *(int *)k->dst = 1;
        return 0;
    case K_BOOL: {
        int idx = 0;
        if (fscanf(fp, "%80s", tok) != 1) return 0;
        if (word_index(run, k->name, tok, BOOL_WORDS, NWORDS(BOOL_WORDS), &idx)) return -1;
        *(int *)k->dst = (idx % 2 == 0);
        return 0;
    }
    case K_WORD: {
        int idx = 0;
        if (fscanf(fp, "%80s", tok) != 1) return 0;
        if (word_index(run, k->name, tok, k->words, k->nwords, &idx)) return -1;
        *(int *)k->dst = idx;
        return 0;
    }
    case K_INT:
        if (fscanf(fp, "%d", (int *)k->dst) < 0) return 0;
        return 0;
    case K_DBL:
        if (fscanf(fp, "%lf", (double *)k->dst) < 0) return 0;
        return 0;
    case K_INT3:
        for (int c = 0; c < 3; c++)
            if (fscanf(fp, "%d", (int *)k->dst + c) < 0) break;
        return 0;
    case K_UPPER: {
        double(*tab)[NT] = (double(*)[NT])k->dst;
        for (int a = 0; a < ntype; a++)
            for (int b = a; b < ntype; b++)
                if (fscanf(fp, "%lf", &tab[a][b]) < 0) return 0;
        return 0;
    }
    case K_TYPE_D:
    case K_TYPE_V3:
    case K_TYPE_M9: {
        int slot = *k->count;
        int nval = k->kind == K_TYPE_D ? 1 : (k->kind == K_TYPE_V3 ? 3 : 9);
        if (slot >= NT) return mdffh_fail(run, "%s: more than %d types", k->name, NT);
        double *row = (double *)k->dst + (size_t)slot * nval;
        for (int c = 0; c < nval; c++)   /* one fscanf of nval numbers: stops at the first miss */
            if (fscanf(fp, "%lf", row + c) != 1) break;
        *k->count = slot + 1;
        return 0;
    }
    case K_DAMP_BOOL: {
        int idx = 0;
        if (fscanf(fp, "%d %d %d %80s", &t, &i, &j, tok) != 4) return mdffh_fail(run, "%s: bad line", k->name);
        if (type_triple(run, k->name, t, i, j)) return -1;
        if (word_index(run, k->name, tok, BOOL_WORDS, NWORDS(BOOL_WORDS), &idx)) return -1;
        ((int(*)[NT][NT])k->dst)[t][i][j] = (idx % 2 == 0);
        return 0;
    }
    case K_DAMP_D:
    case K_DAMP_I:
        if (fscanf(fp, "%d %d %d", &t, &i, &j) != 3) return mdffh_fail(run, "%s: bad type indices", k->name);
        if (type_triple(run, k->name, t, i, j)) return -1;
        if (k->kind == K_DAMP_D)
            (void)!fscanf(fp, "%lf", &((double(*)[NT][NT])k->dst)[t][i][j]);
        else
            (void)!fscanf(fp, "%d", &((int(*)[NT][NT])k->dst)[t][i][j]);
        return 0;
    }
    return 0;
}

/* Runs one module's table over the whole control file. */
static int scan(mdffh_run *run, const char *controlfn, const struct key *keys, int nkeys, int ntype) {
    FILE *fp = fopen(controlfn, "r");
    if (!fp) return mdffh_fail(run, "opening control file %s", controlfn);
    char tok[MDFFH_NAMELEN];
    int rc = 0;
    while (rc == 0 && fscanf(fp, "%80s", tok) == 1) {
        for (int k = 0; k < nkeys && rc == 0; k++)
            if (strcmp(tok, keys[k].name) == 0) rc = read_value(run, fp, &keys[k], tok, ntype);
    }
    fclose(fp);
    return rc;
}

#define KEY(n, k, d) {n, k, (void *)(d), NULL, 0, NULL}
#define WKEY(n, d, w) {n, K_WORD, (void *)(d), w, NWORDS(w), NULL}
#define TKEY(n, k, d, c) {n, k, (void *)(d), NULL, 0, c}

/* init_global: default_global, read_global, check_global (src/global.c:85-107). */
int mdffh_init_global(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    run->Fposff = 2;
    p->skindiff = 0.15;
    run->lstatic = run->lpstress = run->lrdf = 0;
    p->lverletL = 1;
    const struct key keys[] = {
        KEY("lverletL", K_BOOL, &p->lverletL),   KEY("lstatic", K_BOOL, &run->lstatic),
        KEY("lrdf", K_BOOL, &run->lrdf),         KEY("lpstress", K_BOOL, &run->lpstress),
        KEY("cutshortrange", K_DBL, &p->cutshortrange), KEY("cutlongrange", K_DBL, &p->cutlongrange),
        WKEY("Fposff", &run->Fposff, FPOSFF_WORDS), KEY("skindiff", K_DBL, &p->skindiff),
        KEY("lreduced", K_BOOL, &p->lreduced),
    };
    if (scan(run, controlfn, keys, NWORDS(keys), 0)) return -1;
    if (p->lreduced) {
        run->boltz_unit = run->time_unit = run->press_unit = run->coul_unit = 1.0;
    } else {
        run->boltz_unit = BOLTZ_UNIT;
        run->time_unit = TIME_UNIT;
        run->press_unit = PRESS_UNIT;
        run->coul_unit = COUL_UNIT;
    }
    return 0;
}

/* init_md: default_md, read_md (src/md.c:29-118).  The unit conversions of check_md
 * (src/md.c:120-127) happen inside the engine, which takes the control-file values;
 * its TRAJFF removal happens in the host program. */
int mdffh_init_md(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    p->egrator = 1;
    run->nprint = 1;
    run->fprint = 1;
    run->cprint = 1000;
    run->tprint = 1000;
    run->tstart = 0;
    const struct key keys[] = {
        WKEY("integrator", &p->egrator, INTEGRATOR_WORDS),
        KEY("dt", K_DBL, &p->dt),
        KEY("temp", K_DBL, &p->temp),
        KEY("npas", K_INT, &run->npas),
        KEY("nprint", K_INT, &run->nprint),
        KEY("fprint", K_INT, &run->fprint),
        KEY("cprint", K_INT, &run->cprint),
        KEY("tstart", K_INT, &run->tstart),
        KEY("tprint", K_INT, &run->tprint),
        KEY("nequil", K_INT, &p->nequil),
        KEY("nequilT", K_INT, &p->nequilT),
        KEY("tauTberendsen", K_DBL, &p->tauTberendsen),
        KEY("nhc_n", K_INT, &p->nhc_n),
        KEY("nhc_mults", K_INT, &p->nhc_mults),
        KEY("nhc_yosh_order", K_INT, &p->nhc_yosh_order),
        KEY("timesca_thermo", K_DBL, &p->timesca_thermo),
        KEY("timesca_baro", K_DBL, &run->timesca_baro),
    };
    return scan(run, controlfn, keys, NWORDS(keys), 0);
}

/* default_nmlj (src/nmlj.c:110-119) + read_nmlj. */
static int init_nmlj(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    int nt = p->ntype;
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < nt; j++) {
            p->plj[i][j] = 6.0;
            p->qlj[i][j] = 12.0;
            p->sigmalj[i][j] = 3.405;
            p->epslj[i][j] = 0.010323576;
        }
    const struct key keys[] = {
        KEY("sigmalj", K_UPPER, p->sigmalj), KEY("epslj", K_UPPER, p->epslj),
        KEY("plj", K_UPPER, p->plj),         KEY("qlj", K_UPPER, p->qlj),
        WKEY("trunc", &p->trunctype, TRUNC_WORDS),
    };
    if (scan(run, controlfn, keys, NWORDS(keys), nt)) return -1;
    for (int i = 0; i < nt; i++)   /* init_nmlj copies the read upper triangle down (src/nmlj.c:198-207) */
        for (int j = i; j < nt; j++) {
            p->plj[j][i] = p->plj[i][j];
            p->qlj[j][i] = p->qlj[i][j];
            p->sigmalj[j][i] = p->sigmalj[i][j];
            p->epslj[j][i] = p->epslj[i][j];
        }
    return 0;
}

static int init_bhmftd(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    const struct key keys[] = {
        KEY("Abhmftd", K_UPPER, p->Abhmftd), KEY("Bbhmftd", K_UPPER, p->Bbhmftd),
        KEY("Cbhmftd", K_UPPER, p->Cbhmftd), KEY("Dbhmftd", K_UPPER, p->Dbhmftd),
        KEY("BDbhmftd", K_UPPER, p->BDbhmftd),
    };
    if (scan(run, controlfn, keys, NWORDS(keys), p->ntype)) return -1;
    for (int i = 0; i < p->ntype; i++)   /* init_bhmftd's symmetric copy (src/bhmftd.c:98-110) */
        for (int j = i; j < p->ntype; j++) {
            p->Abhmftd[j][i] = p->Abhmftd[i][j];
            p->Bbhmftd[j][i] = p->Bbhmftd[i][j];
            p->Cbhmftd[j][i] = p->Cbhmftd[i][j];
            p->Dbhmftd[j][i] = p->Dbhmftd[i][j];
            p->BDbhmftd[j][i] = p->BDbhmftd[i][j];
        }
    return 0;
}

/* default_pim (src/pim.c:72-85) + read_pim. */
static int init_pim(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    p->conv_tol_ind = 1e-6;
    p->min_scf_pim_iter = 3;
    p->max_scf_pim_iter = 100;
    p->extrapolate_order = 0;
    p->algo_extrapolate_dipole = 0;
    p->algo_pim = 0;
    const struct key keys[] = {
        WKEY("algo_pim", &p->algo_pim, ALGO_PIM_WORDS),
        WKEY("algo_extrapolate_dipole", &p->algo_extrapolate_dipole, EXTRAPOLATE_WORDS),
        KEY("conv_tol_ind", K_DBL, &p->conv_tol_ind),
        KEY("extrapolate_order", K_INT, &p->extrapolate_order),
        KEY("min_scf_pim_iter", K_INT, &p->min_scf_pim_iter),
        KEY("max_scf_pim_iter", K_INT, &p->max_scf_pim_iter),
        KEY("omegakO", K_DBL, &p->omegakO),
    };
    return scan(run, controlfn, keys, NWORDS(keys), p->ntype);
}

/* init_field (src/field.c:313-335) after read_field (src/field.c:31-183). */
int mdffh_init_field(mdffh_run *run, const char *controlfn) {
    mdffgpu_params *p = &run->p;
    double quadit[NT][3][3] = {{{0}}}; /* read and checked: the engine has no quadrupoles */
    run->nmass = run->nqch = run->ndip = run->nqua = run->npol = 0;
    const struct key keys[] = {
        KEY("lbhmft", K_BOOL, &p->lbhmft),
        KEY("lbhmftd", K_BOOL, &p->lbhmftd),
        KEY("lnmlj", K_BOOL, &p->lnmlj),
        KEY("lcoulombic", K_BOOL, &p->lcoulombic),
        TKEY("massit", K_TYPE_D, p->massit, &run->nmass),
        TKEY("qit", K_TYPE_D, p->qit, &run->nqch),
        TKEY("dipit", K_TYPE_V3, p->dipit, &run->ndip),
        TKEY("quadit", K_TYPE_M9, quadit, &run->nqua),
        TKEY("polit", K_TYPE_M9, p->polit, &run->npol),
        KEY("lpoldamping", K_DAMP_BOOL, p->lpoldamping),
        KEY("pol_damp_b", K_DAMP_D, p->pol_damp_b),
        KEY("pol_damp_c", K_DAMP_D, p->pol_damp_c),
        KEY("pol_damp_k", K_DAMP_I, p->pol_damp_k),
        KEY("alphaES", K_DBL, &p->alphaES),
        KEY("kES", K_INT3, p->kES),
        KEY("epsw", K_DBL, &run->epsw),
        KEY("epsw", K_DBL, &run->epsw),
        KEY("lautoES", K_BOOL, &run->lautoES),
    };
    if (scan(run, controlfn, keys, NWORDS(keys), p->ntype)) return -1;
    if (run->nmass != p->ntype && run->nmass != 0)
        return mdffh_fail(run, "massit, some are missing: %d != ntype %d", run->nmass, p->ntype);
    for (int t = 0; t < run->nqua; t++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (quadit[t][i][j] != 0.0)
                    return mdffh_fail(run, "quadit: static quadrupoles are not supported by the engine");
    if (p->lnmlj || p->lbhmft || p->lbhmftd) {
        const struct key nb[] = {KEY("lsymmetric", K_FLAG, &run->lsymmetric)};
        if (scan(run, controlfn, nb, 1, p->ntype)) return -1;
        if (p->lnmlj && init_nmlj(run, controlfn)) return -1;
        if ((p->lbhmft || p->lbhmftd) && init_bhmftd(run, controlfn)) return -1;
    }
    if (p->lcoulombic) {
        if (run->lautoES) mdffh_auto_es(run);
        if (init_pim(run, controlfn)) return -1;
    }
    return 0;
}

/* set_autoES (src/ewald.c:48-71).  alpha takes the C library's integer abs() of the
 * logarithm, which truncates it toward zero: that quantisation is kept. */
void mdffh_auto_es(mdffh_run *run) {
    mdffgpu_params *p = &run->p;
    double wmin = run->w[0];
    for (int i = 1; i < 3; i++)
        if (run->w[i] < wmin) wmin = run->w[i];
    double rcut = 0.5 * wmin;
    if (p->cutlongrange < rcut) {
        printf("WARNING : cutlongrange will be changed according to simuCell.W[]\n");
        p->cutlongrange = rcut;
    }
    double rc = p->cutlongrange;
    double eps = fabs(run->epsw) < 0.5 ? fabs(run->epsw) : 0.5;
    double tol = sqrt(fabs(log(eps * rc)));
    double alpha = sqrt((double)abs((int)log(eps * rc * tol))) / rc;
    double tol1 = sqrt(-log(eps * rc * (2.0 * tol * alpha) * (2.0 * tol * alpha)));
    p->alphaES = alpha;
    for (int k = 0; k < 3; k++) p->kES[k] = (int)nearbyint(0.25 + run->Anorm[k] * alpha * tol1 / M_PI);
}

int mdffh_load(mdffh_run *run, const char *controlfn, const char *posff) {
    memset(run, 0, sizeof *run);
    if (mdffh_init_global(run, controlfn)) return -1;
    if (mdffh_read_config(run, posff ? posff : "POSFF")) return -1;
    if (mdffh_init_md(run, controlfn)) return -1;
    return mdffh_init_field(run, controlfn);
}

void mdffh_free(mdffh_run *run) {
    free(run->atypia);
    double **arrs[] = {&run->rx, &run->ry, &run->rz, &run->vx, &run->vy, &run->vz, &run->fx, &run->fy, &run->fz};
    for (int k = 0; k < 9; k++) {
        free(*arrs[k]);
        *arrs[k] = NULL;
    }
    run->atypia = NULL;
}

int mdffh_iopnode(int step, int npas, int every) {
    return mdffh_iopsnode(step, npas, every, 0);
}

/* A period <= 0 never fires (the reference would divide by zero). */
int mdffh_iopsnode(int step, int npas, int every, int start) {
    if (every <= 0) return 0;
    return (step % every == 0 || step == npas) && step >= start;
}
