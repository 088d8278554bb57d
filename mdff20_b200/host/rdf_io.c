/* Radial distribution: parameters, trajectory reader and RDFFF writer of the
 * reference (src/radial_distribution.c:14-146, read_next_traj src/config.c:448-510).
 * The pair histogram itself is accumulated on the GPU (mdffgpu_rdf_*). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mdffhost.h"

int mdffh_fail(mdffh_run *run, const char *fmt, ...);
void mdffh_lattice(mdffh_run *run);
void mdffh_to_cartesian(int n, double *x, double *y, double *z, const double A[3][3]);

int mdffh_init_rdf(mdffh_run *run, const char *controlfn) {
    double wmin = run->w[0];
    for (int i = 1; i < 3; i++)
        if (run->w[i] < wmin) wmin = run->w[i];
    run->resg = 0.1;
    run->nconf = 0;
    run->cutgr = 0.5 * wmin;
    int nbins_default = (int)(run->cutgr / run->resg) + 1;
    FILE *fp = fopen(controlfn, "r");
    if (!fp) return mdffh_fail(run, "opening control file %s", controlfn);
    char tok[MDFFH_NAMELEN];
    while (fscanf(fp, "%80s", tok) == 1) {
        if (strcmp(tok, "resg") == 0) (void)!fscanf(fp, "%lf", &run->resg);
        if (strcmp(tok, "nconf") == 0) (void)!fscanf(fp, "%d", &run->nconf);
    }
    fclose(fp);
    if (!(run->resg > 0.0)) return mdffh_fail(run, "resg must be positive");
    run->nbins = run->resg >= 0.1 ? nbins_default : (int)(run->cutgr / run->resg) + 1;
    return 0;
}

int mdffh_read_traj(mdffh_run *run, FILE *fp) {
    mdffgpu_params *p = &run->p;
    int nion = 0, ntype = 0;
    char cpos[MDFFH_NAMELEN];
    if (fscanf(fp, "%d ", &nion) != 1 || nion != p->nion) return mdffh_fail(run, "TRAJFF: bad or missing frame header");
    if (fscanf(fp, "%80s ", run->configname) != 1) return mdffh_fail(run, "TRAJFF: no name");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (fscanf(fp, "%lf", &p->cell[i][j]) != 1) return mdffh_fail(run, "TRAJFF: bad cell");
    mdffh_lattice(run);
    if (fscanf(fp, "%d", &ntype) != 1 || ntype != p->ntype) return mdffh_fail(run, "TRAJFF: type count differs");
    for (int t = 0; t < ntype; t++)
        if (fscanf(fp, "%80s ", run->atypit[t]) != 1) return mdffh_fail(run, "TRAJFF: bad type names");
    for (int t = 0; t < ntype; t++)
        if (fscanf(fp, "%d", &p->nionit[t]) != 1) return mdffh_fail(run, "TRAJFF: bad ion counts");
    if (fscanf(fp, "%80s ", cpos) != 1) return mdffh_fail(run, "TRAJFF: no coordinate kind");
    for (int ia = 0; ia < nion; ia++) {
        if (fscanf(fp, "%80s ", run->atypia[ia]) != 1 ||
            fscanf(fp, " %lf %lf %lf ", &run->rx[ia], &run->ry[ia], &run->rz[ia]) != 3 ||
            fscanf(fp, " %lf %lf %lf ", &run->vx[ia], &run->vy[ia], &run->vz[ia]) != 3 ||
            fscanf(fp, " %lf %lf %lf ", &run->fx[ia], &run->fy[ia], &run->fz[ia]) != 3)
            return mdffh_fail(run, "TRAJFF: truncated ion block");
    }
    if (strcmp(cpos, "Direct") == 0 || strcmp(cpos, "D") == 0)
        mdffh_to_cartesian(nion, run->rx, run->ry, run->rz, p->cell);
    return 0;
}

int mdffh_write_rdf(mdffh_run *run, const long long *pairs, int nconf, const char *path) {
    const mdffgpu_params *p = &run->p;
    int nt = p->ntype, nb = run->nbins, npairs = nt * (nt + 1) / 2;
    FILE *fp = fopen(path, "w");
    if (!fp) return mdffh_fail(run, "opening file : %s", path);
    double *g = malloc(sizeof(double) * nt * nt);
    for (int b = 0; b < nb; b++) {
        const long long *h = pairs + (size_t)b * nt * nt;
        long long all = 0;
        for (int k = 0; k < nt * nt; k++) all += h[k];
        double rr = ((double)b + 0.5) * run->resg;
        double vol = 4 * M_PI * (run->resg * rr * rr + (pow(run->resg, 3)) / 12);
        vol = vol / run->omega;
        for (int a = 0, mp = 0; a < nt; a++)
            for (int c = 0; c < nt; c++, mp++) {
                long long cnt = h[a * nt + c] + ((a == 0 && c == 0) ? all : 0);
                g[mp] = ((double)cnt) / (double)(nconf * vol * p->nionit[a] * p->nionit[c]);
            }
        for (int mp = 0; mp < npairs; mp++) fprintf(fp, "%19.12e %19.12e ", rr, g[mp]);
        fprintf(fp, "\n");
    }
    free(g);
    fclose(fp);
    return 0;
}
