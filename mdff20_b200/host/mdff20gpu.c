/* mdff20gpu.x -- the reference's program (src/mdff20.c, run_md src/md.c:192-283) with
 * every force evaluation, neighbour list and MD step on the GPU through libmdffgpu.
 *
 *   mdff20gpu.x [-p fp64|mixed] [-s reference|cg|cg-fused] [-g 0|1] [-d device] [-r RESTART] <control>
 *
 * It reads the control file and ./POSFF like mdff20.x and writes the same files:
 * OSZIFF every fprint steps, CONTFF every cprint steps and at the end, TRAJFF every
 * tprint steps from tstart, and the thermodynamic block on stdout every nprint steps.
 * With lrdf it reads nconf configurations of TRAJFF instead and writes RDFFF, the
 * pair histogram accumulated on the GPU (mdffgpu_rdf_*).
 * Defaults reproduce the reference's numerics (FP64, the reference's algo_pim);
 * -p mixed / -s cg-fused select the fast paths; -g 0 disables CUDA-graph replay.
 * Steps between two outputs that need the host run as one mdffgpu_md_steps call;
 * the per-step thermodynamic records of that call give the OSZIFF lines.
 *
 * Next to every CONTFF it writes RESTART: the engine's complete state
 * (mdffgpu_save_state) behind a small header (step, OSZIFF record count, OSZIFF and
 * TRAJFF lengths).  -r RESTART continues such a run up to npas: OSZIFF and TRAJFF are
 * cut back to their lengths at the restart step and appended to, so the files end up
 * as one uninterrupted run would have left them.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "mdffgpu.h"
#include "mdffhost.h"

#define SEP "============================================================="

static mdffgpu_ctx *g_ctx;

/* RESTART: "MDFFHRS1", int32 istep, int32 oszcall, int64 OSZIFF and TRAJFF sizes at
 * that step, uint64 engine block size, the block */
static const char RESTART_MAGIC[8] = {'M', 'D', 'F', 'F', 'H', 'R', 'S', '1'};

static void die(const char *what, const char *msg) {
    fprintf(stderr, "ERROR: %s: %s\n", what, msg ? msg : "");
    if (g_ctx) mdffgpu_destroy(g_ctx);
    exit(-1);
}

static void check(int rc, const char *what) {
    if (rc != MDFFGPU_OK) die(what, g_ctx ? mdffgpu_last_error(g_ctx) : "");
}

static void thermo_from_record(const double *rec, mdffgpu_thermo *t) {
    memset(t, 0, sizeof *t);
    t->e_kin = rec[0];
    t->u_lj = rec[1];
    t->u_bhmftd = rec[2];
    t->u_coul = rec[3];
    t->u_pol = rec[4];
    t->e_nvt = rec[5];
    t->pvir_lj = rec[6];
    t->pvir_bhmftd = rec[7];
    t->pvir_coul = rec[8];
}

static void pull_state(mdffh_run *run) {
    check(mdffgpu_get_state(g_ctx, run->rx, run->ry, run->rz, run->vx, run->vy, run->vz, run->fx, run->fy,
                            run->fz),
          "get_state");
}

static long long file_size(const char *path) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return 0;
    fseek(fp, 0, SEEK_END);
    long long n = ftell(fp);
    fclose(fp);
    return n;
}

static void write_restart(mdffh_run *run, int istep, FILE *osz) {
    size_t bytes = 0;
    check(mdffgpu_state_size(g_ctx, &bytes), "state_size");
    void *blob = malloc(bytes);
    if (!blob) die("RESTART", "out of memory");
    check(mdffgpu_save_state(g_ctx, blob, bytes), "save_state");
    fflush(osz);
    int head[2] = {istep, run->oszcall};
    long long sizes[2] = {file_size("OSZIFF"), file_size("TRAJFF")};
    unsigned long long nb = bytes;
    FILE *fp = fopen("RESTART", "wb");
    if (!fp) die("RESTART", "cannot open for writing");
    int ok = fwrite(RESTART_MAGIC, 8, 1, fp) == 1 && fwrite(head, sizeof head, 1, fp) == 1 &&
             fwrite(sizes, sizeof sizes, 1, fp) == 1 && fwrite(&nb, sizeof nb, 1, fp) == 1 &&
             fwrite(blob, bytes, 1, fp) == 1;
    if (fclose(fp) != 0 || !ok) die("RESTART", "write failed");
    free(blob);
}

/* Loads a RESTART file into the context and cuts OSZIFF and TRAJFF back to their
 * lengths at that step; returns the step. */
static int read_restart(mdffh_run *run, const char *path) {
    FILE *fp = fopen(path, "rb");
    if (!fp) die(path, "cannot open restart file");
    char magic[8];
    int head[2];
    long long sizes[2];
    unsigned long long nb = 0;
    if (fread(magic, 8, 1, fp) != 1 || memcmp(magic, RESTART_MAGIC, 8) != 0 || fread(head, sizeof head, 1, fp) != 1 ||
        fread(sizes, sizeof sizes, 1, fp) != 1 || fread(&nb, sizeof nb, 1, fp) != 1)
        die(path, "not a restart file");
    void *blob = malloc(nb ? nb : 1);
    if (!blob || fread(blob, nb, 1, fp) != 1) die(path, "truncated restart file");
    fclose(fp);
    int istep = 0;
    check(mdffgpu_load_state(g_ctx, blob, nb, &istep), "load_state");
    free(blob);
    if (istep != head[0]) die(path, "inconsistent restart file");
    run->oszcall = head[1];
    const char *files[2] = {"OSZIFF", "TRAJFF"};
    for (int k = 0; k < 2; k++) {
        if (file_size(files[k]) < sizes[k]) die(files[k], "shorter than at the restart step");
        if (access(files[k], F_OK) == 0 && truncate(files[k], sizes[k]) != 0) die(files[k], "cannot truncate");
    }
    return istep;
}

/* Does step s need the host (anything but an OSZIFF line)? */
static int host_step(const mdffh_run *run, int s, int rescale_allowed) {
    const mdffgpu_params *p = &run->p;
    if (s == run->npas) return 1;
    if (rescale_allowed && s < p->nequil && p->nequilT > 0 && s % p->nequilT == 0) return 1;
    return mdffh_iopnode(s, run->npas, run->nprint) || mdffh_iopnode(s, run->npas, run->cprint) ||
           mdffh_iopsnode(s, run->npas, run->tprint, run->tstart);
}

/* run_md (src/md.c:192-283) from step first (1, or the step after a restart). */
static void run_md(mdffh_run *run, int first) {
    const mdffgpu_params *p = &run->p;
    int egrator = (p->egrator == 0 && p->nequil > 0) ? 1 : p->egrator;   /* check_md, src/md.c:128-131 */
    int rescale_allowed = egrator == 1;
    mdffgpu_thermo t;
    if (first == 1) {
        double e_kin = mdffh_calc_kin(run);
        printf(SEP "\nproperties at t=0\n" SEP "\n\n");
        check(mdffgpu_engforce(g_ctx), "engforce");
        check(mdffgpu_get_thermo(g_ctx, &t), "get_thermo");
        t.e_kin = e_kin;
        t.e_nvt = 0.0;
        mdffh_info_thermo(run, 0, stdout, 0, &t);
    }
    if (run->npas >= first) printf(SEP "\nstarting main MD loop at step %d\n" SEP "\n\n", first);
    FILE *osz = fopen("OSZIFF", first == 1 ? "w" : "a");
    if (!osz) die("opening OSZIFF file", "");
    double *rec = malloc(12 * sizeof(double) * (size_t)(run->npas > 0 ? run->npas : 1));
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int istep = first;
    while (istep <= run->npas) {
        int last = istep;
        while (last < run->npas && !host_step(run, last, rescale_allowed)) last++;
        int nsteps = last - istep + 1;
        check(mdffgpu_md_steps(g_ctx, istep, nsteps, rec), "md_steps");
        for (int k = 0; k < nsteps - 1; k++) {   /* steps that only write OSZIFF */
            if (!mdffh_iopnode(istep + k, run->npas, run->fprint)) continue;
            thermo_from_record(rec + 12 * (size_t)k, &t);
            mdffh_info_thermo(run, 1, osz, istep + k, &t);
        }
        int s = last;   /* loop body of src/md.c:242-281 after prop_agate + check_verletlist */
        int need_state = mdffh_iopnode(s, run->npas, run->cprint) || mdffh_iopsnode(s, run->npas, run->tprint, run->tstart);
        if (rescale_allowed && s < p->nequil && p->nequilT > 0 && s % p->nequilT == 0) {
            pull_state(run);
            mdffh_rescale_velocities(run, 1);
            check(mdffgpu_set_velocities(g_ctx, run->vx, run->vy, run->vz), "set_velocities");
        }
        check(mdffgpu_get_thermo(g_ctx, &t), "get_thermo");
        if (mdffh_iopnode(s, run->npas, run->nprint)) {
            clock_gettime(CLOCK_MONOTONIC, &t1);
            double dt = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
            printf("  MD step %9d  wall time since last report %10.4f (s)\n", s, dt);
            t0 = t1;
            mdffh_info_thermo(run, 0, stdout, s, &t);
        }
        if (mdffh_iopnode(s, run->npas, run->fprint)) mdffh_info_thermo(run, 1, osz, s, &t);
        if (need_state) {
            pull_state(run);
            if (mdffh_iopsnode(s, run->npas, run->tprint, run->tstart) && mdffh_write_config(run, "TRAJFF", 'a'))
                die("TRAJFF", run->err);
            if (mdffh_iopnode(s, run->npas, run->cprint)) {
                if (mdffh_write_config(run, "CONTFF", 'w')) die("CONTFF", run->err);
                write_restart(run, s, osz);
            }
        }
        istep = last + 1;
    }
    free(rec);
    pull_state(run);
    if (mdffh_write_config(run, "CONTFF", 'w')) die("CONTFF", run->err);
    write_restart(run, istep - 1, osz);
    fclose(osz);
}

/* The lrdf branch of the reference's main (src/mdff20.c:108-110, init_rdf
 * src/radial_distribution.c:147-163): nconf configurations of TRAJFF into the pair
 * histogram on the GPU, then RDFFF. */
static void run_rdf(mdffh_run *run, const char *controlfn, int device) {
    mdffgpu_params *p = &run->p;
    if (mdffh_init_rdf(run, controlfn)) die("rdf", run->err);
    printf("radial distribution: resg = %.5f, nconf = %d, %d points in g(r), cutgr = %.5f\n", run->resg, run->nconf,
           run->nbins, run->cutgr);
    mdffgpu_rdf *acc = NULL;
    if (mdffgpu_rdf_create(p->nion, p->ntype, p->nionit, run->cutgr, run->resg, run->nbins, device, &acc) != MDFFGPU_OK)
        die("rdf_create", "bad sizes or no device");
    FILE *fp = fopen("TRAJFF", "r");
    if (!fp) die("TRAJFF", "not found");
    for (int ic = 0; ic < run->nconf; ic++) {
        if (mdffh_read_traj(run, fp)) die("TRAJFF", run->err);
        if (mdffgpu_rdf_add(acc, &p->cell[0][0], run->rx, run->ry, run->rz) != MDFFGPU_OK)
            die("rdf_add", mdffgpu_rdf_last_error(acc));
    }
    fclose(fp);
    size_t nh = (size_t)run->nbins * p->ntype * p->ntype;
    long long *pairs = malloc(sizeof(long long) * nh);
    int nconf = 0;
    if (!pairs || mdffgpu_rdf_counts(acc, pairs, &nconf) != MDFFGPU_OK) die("rdf_counts", mdffgpu_rdf_last_error(acc));
    mdffgpu_rdf_destroy(acc);
    if (mdffh_write_rdf(run, pairs, run->nconf, "RDFFF")) die("RDFFF", run->err);
    free(pairs);
    printf("write RDFFF\n");
}

static void usage(const char *prog) {
    fprintf(stderr, "Usage : %s [-p fp64|mixed] [-s reference|cg|cg-fused] [-g 0|1] [-d device] [-r RESTART] <control>\n",
            prog);
    exit(-1);
}

int main(int argc, char **argv) {
    int precision = MDFFGPU_FP64, solver = MDFFGPU_PIM_REFERENCE, graph = 1, device = 0, opt;
    const char *restart = NULL;
    while ((opt = getopt(argc, argv, "p:s:g:d:r:")) != -1) {
        if (opt == 'p')
            precision = strcmp(optarg, "mixed") == 0 ? MDFFGPU_MIXED : MDFFGPU_FP64;
        else if (opt == 's')
            solver = strcmp(optarg, "cg") == 0         ? MDFFGPU_PIM_CG
                     : strcmp(optarg, "cg-fused") == 0 ? MDFFGPU_PIM_CG_FUSED
                                                       : MDFFGPU_PIM_REFERENCE;
        else if (opt == 'g')
            graph = atoi(optarg);
        else if (opt == 'd')
            device = atoi(optarg);
        else if (opt == 'r')
            restart = optarg;
        else
            usage(argv[0]);
    }
    if (optind >= argc) usage(argv[0]);
    const char *controlfn = argv[optind];
    struct timespec start, end;
    clock_gettime(CLOCK_MONOTONIC, &start);

    static mdffh_run run;
    if (mdffh_load(&run, controlfn, "POSFF")) die("input", run.err);
    mdffgpu_params *p = &run.p;
    printf(SEP "\nmdff20gpu: %d ions, %d types, config %s\n", p->nion, p->ntype, run.configname);
    printf("cutshortrange = %-6.2f cutlongrange = %-6.2f skindiff = %-6.2f\n", p->cutshortrange, p->cutlongrange,
           p->skindiff);
    if (p->lcoulombic) printf("alphaES = %f  kES = %d %d %d\n", p->alphaES, p->kES[0], p->kES[1], p->kES[2]);
    printf("precision %s, induced-dipole solver %s, graph %d\n" SEP "\n", precision ? "mixed" : "fp64",
           solver == MDFFGPU_PIM_REFERENCE ? "reference" : (solver == MDFFGPU_PIM_CG ? "cg" : "cg-fused"), graph);
    if (run.lrdf) {   /* TRAJFF is input here: check_md keeps it (src/md.c:136) */
        run_rdf(&run, controlfn, device);
        mdffh_free(&run);
        return 0;
    }
    /* check_md (src/md.c:134-137): a requested trajectory starts from an empty file
     * (a restarted run appends to it) */
    if (!restart && run.tprint > 0 && access("TRAJFF", F_OK) == 0) remove("TRAJFF");

    check(mdffgpu_create(p, run.rx, run.ry, run.rz, run.vx, run.vy, run.vz, device, &g_ctx), "create");
    check(mdffgpu_set_precision(g_ctx, precision), "set_precision");
    check(mdffgpu_set_pim_solver(g_ctx, solver), "set_pim_solver");
    check(mdffgpu_set_graph(g_ctx, graph), "set_graph");
    if (p->lverletL) check(mdffgpu_gen_verletlist(g_ctx), "gen_verletlist");

    if (!run.lstatic) {
        int first = 1;
        if (restart) {
            first = read_restart(&run, restart) + 1;
        } else {
            mdffh_init_velocities(&run);
            check(mdffgpu_set_velocities(g_ctx, run.vx, run.vy, run.vz), "set_velocities");
        }
        run_md(&run, first);
    } else {
        mdffgpu_thermo t;
        double e_kin = mdffh_calc_kin(&run);
        printf("  static properties\n");
        check(mdffgpu_engforce(g_ctx), "engforce");
        check(mdffgpu_get_thermo(g_ctx, &t), "get_thermo");
        t.e_kin = e_kin;
        t.e_nvt = 0.0;
        check(mdffgpu_get_state(g_ctx, NULL, NULL, NULL, NULL, NULL, NULL, run.fx, run.fy, run.fz), "get_state");
        printf(SEP "\n  properties at t=0\n" SEP "\n\n");
        if (mdffh_write_config(&run, "CONTFF", 'w')) die("CONTFF", run.err);
        mdffh_info_thermo(&run, 0, stdout, 0, &t);
    }
    mdffgpu_destroy(g_ctx);
    g_ctx = NULL;
    mdffh_free(&run);
    clock_gettime(CLOCK_MONOTONIC, &end);
    printf("\n" SEP "\nElapsed time : %5.3f (s)\n", (end.tv_sec - start.tv_sec) + 1e-9 * (end.tv_nsec - start.tv_nsec));
    return 0;
}
