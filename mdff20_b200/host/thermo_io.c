/* Velocities and thermodynamic output of the reference, restated.
 *
 * init_velocities / maxwellboltzmann_velocities / rescale_velocities / calc_kin
 * (src/kinetic.c:15-113, box_muller src/rand.c:19-31) and info_thermo
 * (src/thermo.c:12-122): the stdout block and the OSZIFF record.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "mdffhost.h"

#define EE "%19.12e "
#define E8 "%15.8e "
#define TT3 "%14.7e %14.7e %14.7e "

static const char OSZ_HEADER[] =
    "   step      Time/Temp   Etot/Pressure    Ekin/Pvir_nb  Utot/Pvir_coul      U_nb/Omega     U_coul/Htot\n";

/* Standard normal sample by the Box-Muller transform on two rand() draws in (0, 1]. */
static double gauss(void) {
    double u, v;
    do {
        u = (double)rand() / (double)RAND_MAX;
        v = (double)rand() / (double)RAND_MAX;
    } while (u == 0.0 || v == 0.0);
    return sqrt(-2.0 * log(u)) * cos(2.0 * M_PI * v);
}

static double mass_of(const mdffh_run *run, int ia) {
    int acc = 0;
    for (int t = 0; t < run->p.ntype; t++) {
        acc += run->p.nionit[t];
        if (ia < acc) return run->p.massit[t];
    }
    return run->p.massit[run->p.ntype - 1];
}

double mdffh_calc_kin(const mdffh_run *run) {
    double kin = 0.0;
    for (int ia = 0; ia < run->p.nion; ia++)
        kin += (run->vx[ia] * run->vx[ia] + run->vy[ia] * run->vy[ia] + run->vz[ia] * run->vz[ia]) *
               mass_of(run, ia);
    return kin * 0.5;
}

static void remove_drift(mdffh_run *run) {
    int n = run->p.nion;
    double sx = 0.0, sy = 0.0, sz = 0.0, inv = 1.0 / (double)n;
    for (int ia = 0; ia < n; ia++) sx += run->vx[ia], sy += run->vy[ia], sz += run->vz[ia];
    sx *= inv, sy *= inv, sz *= inv;
    for (int ia = 0; ia < n; ia++) run->vx[ia] -= sx, run->vy[ia] -= sy, run->vz[ia] -= sz;
}

/* temperature as held after check_md (kB T) and the time-step ratio dt / tauTberendsen
 * (tauTberendsen defaults to dt when nequil > 0, src/md.c:121). */
static double kT(const mdffh_run *run) { return run->p.temp * run->boltz_unit; }

void mdffh_rescale_velocities(mdffh_run *run, int quiet) {
    const mdffgpu_params *p = &run->p;
    double ekin = mdffh_calc_kin(run);
    double T = (2.0 * ekin) / (3.0 * (double)p->nion * run->boltz_unit);
    double tau = p->tauTberendsen;
    if (p->nequil > 0 && tau == 0.0) tau = p->dt;
    double lambda;
    if (p->egrator != 2)   /* both times in internal units, as check_md leaves them */
        lambda = sqrt(1.0 + ((p->dt * run->time_unit) / (tau * run->time_unit)) *
                                ((kT(run) / T / run->boltz_unit) - 1.0));
    else
        lambda = sqrt(1.0 + ((kT(run) / T / run->boltz_unit) - 1.0));
    for (int ia = 0; ia < p->nion; ia++) run->vx[ia] *= lambda, run->vy[ia] *= lambda, run->vz[ia] *= lambda;
    remove_drift(run);
    if (!quiet) {
        printf("initial kinetic energy info\n");
        printf("effective temperature T  = %10.4f\n", T);
        printf("wanted temperature    T0 = %10.4f\n", kT(run) / run->boltz_unit);
    }
}

void mdffh_init_velocities(mdffh_run *run) {
    double t = kT(run);
    srand(1);   /* the reference never seeds rand(): its draws start from the default seed */
    for (int ia = 0; ia < run->p.nion; ia++) {
        double s = sqrt(t * (1.0 / mass_of(run, ia)));
        run->vx[ia] = s * gauss();
        run->vy[ia] = s * gauss();
        run->vz[ia] = s * gauss();
    }
    remove_drift(run);
    mdffh_rescale_velocities(run, 0);
}

void mdffh_info_thermo(mdffh_run *run, int key, FILE *fp, int istep, const mdffgpu_thermo *t) {
    const mdffgpu_params *p = &run->p;
    double l = 3.0 * (double)p->nion;
    double temp_r = (2.0 * t->e_kin) / (l * run->boltz_unit);
    double time = (double)istep * (p->dt * run->time_unit) / run->time_unit;
    double u_vdw = t->u_lj + t->u_bhmftd;
    double u_tot = u_vdw + t->u_coul + t->u_pol;
    double e_tot = u_tot + t->e_kin;
    double h_tot = e_tot + t->e_nvt;
    double pvir_vdw = t->pvir_lj + t->pvir_bhmftd;
    double pvir_tot = pvir_vdw + t->pvir_coul;
    double pressure = pvir_tot + temp_r * run->boltz_unit * run->inveOmegaPU;
    if (key == 1) {
        if (run->oszcall % 10 == 0) {
            for (int i = 0; i < 105; i++) fputc('-', fp);
            fputc('\n', fp);
            fputs(OSZ_HEADER, fp);
            for (int i = 0; i < 105; i++) fputc('-', fp);
            fputc('\n', fp);
        }
        fprintf(fp, "%7d" E8 E8 E8 E8 E8 E8 "\n", istep, time, e_tot, t->e_kin, u_tot, u_vdw, t->u_coul);
        fprintf(fp, "%7d" E8 E8 E8 E8 E8 E8 "\n", istep, temp_r, pressure, pvir_vdw, t->pvir_coul, run->omega, h_tot);
        run->oszcall += 1;
        return;
    }
    double tau_vdw[9], tau_tot[9];
    for (int k = 0; k < 9; k++) {
        tau_vdw[k] = t->tau_lj[k] + t->tau_bhmftd[k];
        tau_tot[k] = tau_vdw[k] + t->tau_coul[k];
    }
    static const char RULE[] = "  ---------------------------------------------\n";
    fprintf(fp, "\n");
    fprintf(fp, "  Thermodynamic information                    \n");
    fputs(RULE, fp);
    fprintf(fp, "  step                  = %9d\n", istep);
    fprintf(fp, "  time                  = " EE "\n", time);
    fprintf(fp, "  Ekin                  = " EE "\n", t->e_kin);
    fprintf(fp, "  Temp                  = " EE "\n", temp_r);
    fprintf(fp, "  Utot                  = " EE "\n", u_tot);
    fprintf(fp, "  Uvdw                  = " EE "\n", u_vdw);
    fprintf(fp, "  Ucoul                 = " EE "\n", t->u_coul);
    fprintf(fp, "  Upol                  = " EE "\n", t->u_pol);
    fprintf(fp, "  Pressure              = " EE "\n", pressure);
    fprintf(fp, "  Pvirvdw               = " EE "\n", pvir_vdw);
    fprintf(fp, "  Pvircoul              = " EE "\n", t->pvir_coul);
    fprintf(fp, "  volume                = " EE "\n", run->omega);
    fprintf(fp, "  a cell                = " EE "\n", run->Anorm[0]);
    fprintf(fp, "  b cell                = " EE "\n", run->Anorm[1]);
    fprintf(fp, "  c cell                = " EE "\n", run->Anorm[2]);
    fputs(RULE, fp);
    fprintf(fp, "  Etot                  = " EE "\n", e_tot);
    fprintf(fp, "  Htot                  = " EE "\n", h_tot);
    fprintf(fp, "\n");
    const double *blocks[3] = {tau_vdw, t->tau_coul, tau_tot};
    static const char *const titles[3] = {"  non_bonded stress tensor :                   \n",
                                          "  electrostatic stress tensor :                \n",
                                          "  total stress tensor :                \n"};
    int split = (p->lnmlj || p->lbhmft || p->lbhmftd) && p->lcoulombic && run->lpstress;
    for (int b = split ? 0 : 2; b < 3; b++) {
        const double *tau = blocks[b];
        double iso = 0.0;
        fputs(RULE, fp);
        fputs(titles[b], fp);
        fputs(RULE, fp);
        for (int i = 0; i < 3; i++) {
            fprintf(fp, "  " TT3 "\n", tau[3 * i], tau[3 * i + 1], tau[3 * i + 2]);
            iso += tau[4 * i];
        }
        fputs(RULE, fp);
        fprintf(fp, "  iso = " E8 "(" E8 ")\n", iso * (1.0 / 3.0), iso * (1.0 / (3.0 * (double)p->nion)));
        fputc('\n', fp);
    }
}

int mdffh_oszi_append(mdffh_run *run, const char *path, int istep, const mdffgpu_thermo *t) {
    FILE *fp = fopen(path, "a");
    if (!fp) {
        snprintf(run->err, sizeof run->err, "opening %s", path);
        return -1;
    }
    mdffh_info_thermo(run, 1, fp, istep, t);
    fclose(fp);
    return 0;
}
