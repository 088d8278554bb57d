/* Configuration files of the reference: POSFF in, CONTFF/TRAJFF out.
 *
 * POSFF (read_config, src/config.c:347-446), whitespace-separated:
 *   nion / name / 3 rows of the cell matrix A (rows are lattice vectors) / ntype /
 *   ntype type names / ntype ion counts / "Cartesian" or "Direct" ("D") /
 *   per ion: type name, x y z, then vx vy vz when Fposff >= rvn, fx fy fz when rvf.
 * Ions come grouped by type in type order (init_config assigns types in blocks of
 * nionit, src/config.c:135-148).  Positions are wrapped into the cell as read_config
 * does (src/config.c:442-444): to fractional with B, minus nearbyint, back with A.
 *
 * CONTFF and TRAJFF (write_config, src/config.c:291-345) use the same layout with the
 * reference's fixed formats: "%19.12f " numbers, "Cartesian", per ion the name as
 * read, wrapped position, velocity and force.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mdffhost.h"

int mdffh_fail(mdffh_run *run, const char *fmt, ...);
void mdffh_lattice(mdffh_run *run);
void mdffh_to_cartesian(int n, double *x, double *y, double *z, const double A[3][3]);

#define FF "%19.12f "

/* lattice (src/cell.c:13-91): unnormalised reciprocal rows Bu_i = A_j x A_k, the volume
 * sum_i Bu_i[0] A_i[0], the face distances omega/|column i of Bu|, B = Bu/omega, and
 * the column norms Anorm[i] = |(A_0[i], A_1[i], A_2[i])|. */
void mdffh_lattice(mdffh_run *run) {
    const double(*A)[3] = run->p.cell;
    double(*B)[3] = run->B;
    const int nx[3] = {1, 2, 0}, ny[3] = {2, 0, 1};
    for (int i = 0; i < 3; i++) {
        const double *u = A[nx[i]], *v = A[ny[i]];
        B[i][0] = u[1] * v[2] - u[2] * v[1];
        B[i][1] = u[2] * v[0] - u[0] * v[2];
        B[i][2] = u[0] * v[1] - u[1] * v[0];
    }
    double omega = B[0][0] * A[0][0] + B[1][0] * A[1][0] + B[2][0] * A[2][0];
    run->omega = omega;
    run->inveOmega = 1.0 / omega;
    run->inveOmegaPU = 1.0 / (omega * run->press_unit);
    for (int i = 0; i < 3; i++)
        run->w[i] = omega / sqrt(B[0][i] * B[0][i] + B[1][i] * B[1][i] + B[2][i] * B[2][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) B[i][j] = B[i][j] * run->inveOmega;
    for (int i = 0; i < 3; i++) {
        double s = 0.0;
        for (int j = 0; j < 3; j++) s += A[j][i] * A[j][i];
        run->Anorm[i] = sqrt(s);
    }
}

/* kardir / dirkar (src/cell.c:125-161), then the minimum-image shift of replace_pbc
 * (src/pbc.c:17-23) in between: the wrap every configuration goes through. */
static void to_fractional(int n, double *x, double *y, double *z, const double B[3][3]) {
    for (int i = 0; i < n; i++) {
        double a = x[i] * B[0][0] + y[i] * B[0][1] + z[i] * B[0][2];
        double b = x[i] * B[1][0] + y[i] * B[1][1] + z[i] * B[1][2];
        double c = x[i] * B[2][0] + y[i] * B[2][1] + z[i] * B[2][2];
        x[i] = a, y[i] = b, z[i] = c;
    }
}

void mdffh_to_cartesian(int n, double *x, double *y, double *z, const double A[3][3]) {
    for (int i = 0; i < n; i++) {
        double a = x[i] * A[0][0] + y[i] * A[1][0] + z[i] * A[2][0];
        double b = x[i] * A[0][1] + y[i] * A[1][1] + z[i] * A[2][1];
        double c = x[i] * A[0][2] + y[i] * A[1][2] + z[i] * A[2][2];
        x[i] = a, y[i] = b, z[i] = c;
    }
}

static void wrap(const mdffh_run *run, int n, double *x, double *y, double *z) {
    to_fractional(n, x, y, z, (const double(*)[3])run->B);
    for (int i = 0; i < n; i++) {
        x[i] -= nearbyint(x[i]);
        y[i] -= nearbyint(y[i]);
        z[i] -= nearbyint(z[i]);
    }
    mdffh_to_cartesian(n, x, y, z, run->p.cell);
}

int mdffh_read_config(mdffh_run *run, const char *posff) {
    mdffgpu_params *p = &run->p;
    FILE *fp = fopen(posff, "r");
    if (!fp) return mdffh_fail(run, "POSFF not found: %s", posff);
    int ok = fscanf(fp, "%d", &p->nion) == 1 && fscanf(fp, "%80s", run->configname) == 1;
    for (int i = 0; ok && i < 3; i++)
        for (int j = 0; ok && j < 3; j++) ok = fscanf(fp, "%lf", &p->cell[i][j]) == 1;
    ok = ok && fscanf(fp, "%d", &p->ntype) == 1;
    if (!ok || p->nion <= 0 || p->ntype <= 0 || p->ntype > MDFFGPU_NTMAX) {
        fclose(fp);
        return mdffh_fail(run, "POSFF: bad header (nion, name, cell, ntype)");
    }
    mdffh_lattice(run);
    for (int t = 0; ok && t < p->ntype; t++) ok = fscanf(fp, "%80s", run->atypit[t]) == 1;
    int total = 0;
    for (int t = 0; ok && t < p->ntype; t++) {
        ok = fscanf(fp, "%d", &p->nionit[t]) == 1;
        total += p->nionit[t];
    }
    ok = ok && fscanf(fp, "%80s", run->cpos) == 1;
    if (!ok || total != p->nion) {
        fclose(fp);
        return mdffh_fail(run, "POSFF: bad type block (names, ions per type summing to nion, coordinates)");
    }
    int n = p->nion;
    run->atypia = calloc((size_t)n, sizeof *run->atypia);
    double **arr[] = {&run->rx, &run->ry, &run->rz, &run->vx, &run->vy, &run->vz, &run->fx, &run->fy, &run->fz};
    for (int k = 0; k < 9; k++) *arr[k] = calloc((size_t)n, sizeof(double));
    for (int ia = 0; ok && ia < n; ia++) {
        ok = fscanf(fp, "%80s ", run->atypia[ia]) == 1 &&
             fscanf(fp, "%lf %lf %lf ", &run->rx[ia], &run->ry[ia], &run->rz[ia]) == 3;
        if (ok && run->Fposff > 0) ok = fscanf(fp, "%lf %lf %lf ", &run->vx[ia], &run->vy[ia], &run->vz[ia]) == 3;
        if (ok && run->Fposff > 1) ok = fscanf(fp, "%lf %lf %lf ", &run->fx[ia], &run->fy[ia], &run->fz[ia]) == 3;
    }
    fclose(fp);
    if (!ok) return mdffh_fail(run, "POSFF: truncated ion block (Fposff %d)", run->Fposff);
    if (strcmp(run->cpos, "Direct") == 0 || strcmp(run->cpos, "D") == 0)
        mdffh_to_cartesian(n, run->rx, run->ry, run->rz, p->cell);
    wrap(run, n, run->rx, run->ry, run->rz);
    return 0;
}

int mdffh_write_config(mdffh_run *run, const char *filename, char mode) {
    const mdffgpu_params *p = &run->p;
    int n = p->nion;
    double *x = malloc(3 * (size_t)n * sizeof(double)), *y = x + n, *z = y + n;
    if (!x) return mdffh_fail(run, "write_config: out of memory");
    memcpy(x, run->rx, n * sizeof(double));
    memcpy(y, run->ry, n * sizeof(double));
    memcpy(z, run->rz, n * sizeof(double));
    wrap(run, n, x, y, z);
    const char m[2] = {mode, 0};
    FILE *fp = fopen(filename, m);
    if (!fp) {
        free(x);
        return mdffh_fail(run, "opening file : %s", filename);
    }
    fprintf(fp, "%d \n", n);
    fprintf(fp, "%s \n", run->configname);
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) fprintf(fp, FF, p->cell[i][j]);
        fprintf(fp, " \n");
    }
    fprintf(fp, "%d \n", p->ntype);
    for (int t = 0; t < p->ntype; t++) fprintf(fp, "%s ", run->atypit[t]);
    fprintf(fp, "\n");
    for (int t = 0; t < p->ntype; t++) fprintf(fp, "%d ", p->nionit[t]);
    fprintf(fp, " \n");
    fprintf(fp, "Cartesian \n");
    for (int ia = 0; ia < n; ia++) {
        fprintf(fp, "%s ", run->atypia[ia]);
        fprintf(fp, FF FF FF, x[ia], y[ia], z[ia]);
        fprintf(fp, FF FF FF, run->vx[ia], run->vy[ia], run->vz[ia]);
        fprintf(fp, FF FF FF, run->fx[ia], run->fy[ia], run->fz[ia]);
        fprintf(fp, "\n");
    }
    fclose(fp);
    free(x);
    return 0;
}
