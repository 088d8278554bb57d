/* Harness main for the compiled reference mdff20 (test infrastructure only).
 *
 * It replaces the reference driver src/mdff20.c:32-144 and runs the same set-up
 * sequence (src/mdff20.c:59-87): gen_constants, init_global, read_config, init_md,
 * init_field, init_config, do_split.  Then, instead of run_md or the static branch,
 * it executes ONE task and dumps the reference's own outputs to `out.bin` in the
 * working directory, as tagged binary records read back by oracle/ref.py:
 *
 *   record = name[32] (NUL padded) | kind 'd'/'i' | 7 pad bytes | int64 count | data
 *
 * usage (run inside a directory holding POSFF):
 *   harness <control> list
 *   harness <control> engforce
 *   harness <control> ewald lq ld ldamp do_forces do_stress do_ef do_efg do_dir do_rec
 *   harness <control> md <nsteps> <record_positions_every>
 *   harness <control> engforce_timing <reps>
 *   harness <control> kmesh
 *   harness <control> rdf [write]
 *
 * Parity deviations from src/mdff20.c, each required for a deterministic harness:
 *  - velocities come from POSFF (Fposff rvn/rvf, src/config.c:415-417) instead of
 *    init_velocities, which draws from glibc rand() (src/mdff20.c:90);
 *  - the NHC state vxi/xi, malloc'ed uninitialised in alloc_md (src/md.c:159-164),
 *    is zeroed;
 *  - the first Verlet list is built by the rebuild branch of check_verletlist
 *    (src/verlet.c:148-157) directly, because xvl/yvl/zvl are uninitialised before
 *    the first check (src/verlet.c:35-37).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdbool.h>
#include <omp.h>
#include "constants.h"
#include "global.h"
#include "cell.h"
#include "config.h"
#include "field.h"
#include "verlet.h"
#include "md.h"
#include "io.h"
#include "timing.h"
#include "thermo.h"
#include "coulombic.h"
#include "kspace.h"
#include "ewald.h"
#include "pim.h"
#include "kinetic.h"
#include "integration.h"
#include "mpi_mdff.h"
#include "radial_distribution.h"

static FILE *g_out;

static void put_rec(const char *name, char kind, const void *data, long long count) {
    char hdr[48];
    memset(hdr, 0, sizeof(hdr));
    strncpy(hdr, name, 31);
    hdr[32] = kind;
    memcpy(hdr + 40, &count, 8);
    fwrite(hdr, 1, 48, g_out);
    size_t sz = (kind == 'i') ? sizeof(int) : sizeof(double);
    if (count > 0) fwrite(data, sz, (size_t)count, g_out);
}
static void put_d(const char *name, const double *d, long long n) { put_rec(name, 'd', d, n); }
static void put_i(const char *name, const int *d, long long n) { put_rec(name, 'i', d, n); }
static void put_s(const char *name, double v) { put_rec(name, 'd', &v, 1); }

static void force_rebuild(void) {
    /* the rebuild branch of check_verletlist, src/verlet.c:131,150-157,168 */
    kardir(nion, rx, ry, rz, simuCell.B);
    updatevl += 1;
    gen_pbc_verletlist();
    for (int ia = 0; ia < nion; ia++) {
        xvl[ia] = rx[ia];
        yvl[ia] = ry[ia];
        zvl[ia] = rz[ia];
    }
    dirkar(nion, rx, ry, rz, simuCell.A);
}

static void put_xyz(const char *name, double *ax, double *ay, double *az) {
    double *t = malloc(3 * (size_t)nion * sizeof(double));
    for (int i = 0; i < nion; i++) {
        t[3 * i] = ax[i];
        t[3 * i + 1] = ay[i];
        t[3 * i + 2] = az[i];
    }
    put_d(name, t, 3LL * nion);
    free(t);
}

static void put_thermo(void) {
    put_s("u_lj", u_lj);
    put_s("u_bhmftd", u_bhmftd);
    put_s("u_coul", u_coul);
    put_s("u_pol", u_pol);
    put_s("pvir_lj", pvir_lj);
    put_s("pvir_bhmftd", pvir_bhmftd);
    put_s("pvir_coul", pvir_coul);
    put_d("tau_lj", &tau_lj[0][0], 9);
    put_d("tau_bhmftd", &tau_bhmftd[0][0], 9);
    put_d("tau_coul", &tau_coul[0][0], 9);
    put_s("e_kin", e_kin);
    put_s("e_nvt", e_nvt);
}

static double *read_raw(const char *fn, long long n) {
    FILE *fp = fopen(fn, "rb");
    if (!fp) return NULL;
    double *d = malloc((size_t)n * sizeof(double));
    size_t got = fread(d, sizeof(double), (size_t)n, fp);
    fclose(fp);
    if ((long long)got != n) {
        fprintf(stderr, "short read %s\n", fn);
        exit(3);
    }
    return d;
}

int main(int argc, char *argv[]) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <control> <task> [args]\n", argv[0]);
        return 2;
    }
    myrank = 0;
    numprocs = 1;
    init_io();
    gen_constants();
    controlfn = argv[1];
    const char *task = argv[2];

    init_global(controlfn);
    read_config();
    init_md(controlfn);
    init_field(controlfn);
    init_config();
    do_split(nion, numprocs, myrank, &atomDec, "atoms");
    do_split(kcoul.nk, numprocs, myrank, &kcoul.kptDec, "k-points");
    if (egrator == 2) {
        for (int i = 0; i < nhc_n; i++) {
            vxi[i] = 0.0;
            xi[i] = 0.0;
        }
    }
    e_nvt = 0.0;

    g_out = fopen("out.bin", "wb");
    if (!g_out) {
        fprintf(stderr, "cannot write out.bin\n");
        return 2;
    }
    int ithreads = omp_get_max_threads();
    put_s("omp_threads", (double)ithreads);

    if (strcmp(task, "list") == 0) {
        put_xyz("r_in", rx, ry, rz);
        force_rebuild();
        put_i("nb_point", verlet_nb->point, nion + 1);
        put_i("nb_list", verlet_nb->list, verlet_nb->point[nion]);
        put_i("coul_point", verlet_coul->point, nion + 1);
        put_i("coul_list", verlet_coul->list, verlet_coul->point[nion]);
        put_xyz("r", rx, ry, rz);
    } else if (strcmp(task, "kmesh") == 0) {
        put_d("kx", kcoul.kx, kcoul.nk);
        put_d("ky", kcoul.ky, kcoul.nk);
        put_d("kz", kcoul.kz, kcoul.nk);
        put_d("kk", kcoul.kk, kcoul.nk);
        put_d("Ak", kcoul.Ak, kcoul.nk);
        put_d("kcoe", kcoul.kcoe, kcoul.nk);
        put_s("alphaES", alphaES);
        put_i("kES", kES, 3);
        put_s("cutlongrange", cutlongrange);
    } else if (strcmp(task, "engforce") == 0) {
        put_xyz("r_in", rx, ry, rz);
        if (lverletL) force_rebuild();
        istep = 0;
        e_kin = calc_kin();
        engforce();
        put_xyz("f", fx, fy, fz);
        put_xyz("r", rx, ry, rz);
        put_thermo();
        if (lcoulombic && lpim) {
            double *mu = malloc(3 * (size_t)nion * sizeof(double));
            for (int i = 0; i < nion; i++)
                for (int k = 0; k < 3; k++) mu[3 * i + k] = dipia_ind[i][0][k];
            put_d("mu_ind", mu, 3LL * nion);
            free(mu);
        }
    } else if (strcmp(task, "engforce_timing") == 0) {
        int reps = (argc > 3) ? atoi(argv[3]) : 1;
        if (lverletL) force_rebuild();
        istep = 0;
        engforce();
        double t0 = omp_get_wtime();
        for (int r = 0; r < reps; r++) engforce();
        double t1 = omp_get_wtime();
        put_s("wall", t1 - t0);
        put_s("reps", (double)reps);
        put_thermo();
    } else if (strcmp(task, "ewald") == 0) {
        if (argc < 12) {
            fprintf(stderr, "ewald needs 9 flags\n");
            return 2;
        }
        int fl[9];
        for (int k = 0; k < 9; k++) fl[k] = atoi(argv[3 + k]);
        put_xyz("r_in", rx, ry, rz);
        if (lverletL) force_rebuild();
        double *q = read_raw("in_q.bin", nion);
        double *mu = read_raw("in_mu.bin", 3LL * nion);
        if (!q) {
            q = malloc((size_t)nion * sizeof(double));
            for (int i = 0; i < nion; i++) q[i] = qia[i];
        }
        if (!mu) {
            mu = malloc(3 * (size_t)nion * sizeof(double));
            for (int i = 0; i < nion; i++)
                for (int k = 0; k < 3; k++) mu[3 * i + k] = dipia[i][k];
        }
        double (*ef)[3] = calloc((size_t)nion, sizeof(*ef));
        double (*efg)[3][3] = calloc((size_t)nion, sizeof(*efg));
        double u = 0.0, pvir = 0.0, tau[3][3];
        memset(tau, 0, sizeof(tau));
        for (int i = 0; i < nion; i++) {
            fx[i] = 0.0;
            fy[i] = 0.0;
            fz[i] = 0.0;
        }
        /* lq ld ldamp do_forces do_stress do_ef do_efg do_dir do_rec; the structure
           factor tables are always refreshed (update_sf true, src/kspace.c:154) */
        multipole_ES(q, (double (*)[3])mu, quadia, &u, &pvir, tau, ef, efg, fl[0], fl[1], false, fl[2],
                     fl[3], fl[4], fl[5], fl[6], fl[7], fl[8], false, true);
        put_s("u", u);
        put_s("pvir", pvir);
        put_d("tau", &tau[0][0], 9);
        put_d("ef", &ef[0][0], 3LL * nion);
        put_d("efg", &efg[0][0][0], 9LL * nion);
        put_xyz("f", fx, fy, fz);
    } else if (strcmp(task, "md") == 0) {
        int nsteps = (argc > 3) ? atoi(argv[3]) : 1;
        int every = (argc > 4) ? atoi(argv[4]) : 0;
        /* first step index: istep drives the ASPC order (src/pim.c:324-334); starting
           past extrapolate_order avoids the first-steps order switch, whose predictor
           reads coefficients the reference never sets for ions >= 1 */
        int first = (argc > 5) ? atoi(argv[5]) : 1;
        npas = first - 1 + nsteps;
        put_xyz("r_in", rx, ry, rz);
        if (lverletL) force_rebuild();
        istep = 0;
        e_kin = calc_kin();
        engforce();
        int nrec = nsteps + 1;
        double *th = calloc((size_t)nrec * 12, sizeof(double));
        int nframes = (every > 0) ? nsteps / every + 1 : 0;
        double *traj = calloc((size_t)nframes * 9 * nion + 1, sizeof(double));
        int iframe = 0;
#define REC_THERMO(s)                                                    \
    do {                                                                 \
        double *t = th + 12 * (size_t)(s);                               \
        t[0] = e_kin; t[1] = u_lj; t[2] = u_bhmftd; t[3] = u_coul;       \
        t[4] = u_pol; t[5] = e_nvt; t[6] = pvir_lj; t[7] = pvir_bhmftd;  \
        t[8] = pvir_coul; t[9] = (double)updatevl; t[10] = 0; t[11] = 0; \
    } while (0)
#define REC_FRAME()                                                          \
    do {                                                                     \
        double *p = traj + 9 * (size_t)nion * iframe;                        \
        for (int i = 0; i < nion; i++) {                                     \
            p[9 * i + 0] = rx[i]; p[9 * i + 1] = ry[i]; p[9 * i + 2] = rz[i]; \
            p[9 * i + 3] = vx[i]; p[9 * i + 4] = vy[i]; p[9 * i + 5] = vz[i]; \
            p[9 * i + 6] = fx[i]; p[9 * i + 7] = fy[i]; p[9 * i + 8] = fz[i]; \
        }                                                                    \
        iframe++;                                                            \
    } while (0)
        REC_THERMO(0);
        if (every > 0) REC_FRAME();
        double *step_wall = calloc((size_t)nsteps + 1, sizeof(double));
        double t0 = omp_get_wtime();
        /* the MD loop body of src/md.c:229-247 without its output */
        for (istep = first; istep < npas + 1; istep++) {
            double ts = omp_get_wtime();
            prop_agate(istep);
            if (lverletL) check_verletlist();
            if ((rescale_allowed) && (istep < nequil) && (istep % nequilT == 0)) rescale_velocities(1);
            step_wall[istep - first] = omp_get_wtime() - ts;
            REC_THERMO(istep - first + 1);
            if (every > 0 && istep % every == 0) REC_FRAME();
        }
        double t1 = omp_get_wtime();
        put_s("wall", t1 - t0);
        put_d("step_wall", step_wall, nsteps);
        free(step_wall);
        put_d("thermo", th, 12LL * nrec);
        if (every > 0) put_d("traj", traj, 9LL * nion * iframe);
        put_xyz("r", rx, ry, rz);
        put_xyz("v", vx, vy, vz);
        put_xyz("f", fx, fy, fz);
        if (egrator == 2) {
            put_d("xi", xi, nhc_n);
            put_d("vxi", vxi, nhc_n);
        }
        put_thermo();
        free(th);
        free(traj);
    } else if (strcmp(task, "rdf") == 0) {
        /* init_rdf (src/radial_distribution.c:147-163) minus its sample_config prints:
         * default_rdf, read_rdf, alloc_rdf, then read_next_traj + get_gr for each of
         * the nconf TRAJFF configurations; dumps the integer histogram gr[bin][it][jt]
         * of the types present, and with "write" also runs write_rdf (RDFFF) */
        default_rdf();
        read_rdf(controlfn);
        alloc_rdf();
        FILE *fp = fopen("TRAJFF", "r");
        if (!fp) {
            fprintf(stderr, "no TRAJFF\n");
            return 2;
        }
        for (int ic = 0; ic < nconf; ic++) {
            read_next_traj(fp);
            get_gr();
        }
        fclose(fp);
        int *h = malloc(sizeof(int) * (size_t)nbins * ntype * ntype);
        for (int b = 0; b < nbins; b++)
            for (int it = 0; it < ntype; it++)
                for (int jt = 0; jt < ntype; jt++) h[(b * ntype + it) * ntype + jt] = gr[b][it][jt];
        put_i("gr", h, (long long)nbins * ntype * ntype);
        put_s("cutgr", cutgr);
        put_s("resg", resg);
        put_s("nbins", (double)nbins);
        put_s("nconf", (double)nconf);
        free(h);
        if (argc > 3 && strcmp(argv[3], "write") == 0) write_rdf();
    } else {
        fprintf(stderr, "unknown task %s\n", task);
        return 2;
    }
    fclose(g_out);
    return 0;
}
