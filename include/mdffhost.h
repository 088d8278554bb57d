/* mdffhost.h -- the reference's input/output layer, restated in C for a drop-in host.
 *
 * libmdffhost (mdff20_b200/host/) reads the reference's two inputs and writes its
 * output files in the reference's formats, so that mdff20gpu.x (the C host program
 * over libmdffgpu) takes the same working directory as the reference executable
 * mdff20.x and leaves the same files behind:
 *
 *   control file  keyword scans of init_global (src/global.c:13-60, 85-107),
 *                 init_md (src/md.c:29-154), init_field (src/field.c:31-183, 313-335),
 *                 read_nmlj/default_nmlj (src/nmlj.c:39-119), read_bhmftd
 *                 (src/bhmftd.c:26-90), read_pim/default_pim (src/pim.c:28-85)
 *   POSFF         read_config (src/config.c:347-446), including its wrap
 *   CONTFF/TRAJFF write_config (src/config.c:291-345)
 *   OSZIFF        info_thermo key 1 (src/thermo.c:111-122)
 *   stdout        info_thermo key 0 (src/thermo.c:36-109)
 *
 * Every scan re-reads the whole control file as whitespace-separated tokens with the
 * C library's fscanf, as each reference module does, so a control file is read the
 * same way token for token (comments are ordinary tokens that match no keyword).
 * Calls return 0 on success and -1 on a bad input; the message is in run->err.  The
 * reference prints an error and exits in the same situations.
 */
#ifndef MDFFHOST_H
#define MDFFHOST_H

#include <stdio.h>
#include "mdffgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MDFFH_NAMELEN 81 /* MAX_LEN + 1 (src/constants.h:4) */

typedef struct mdffh_run {
    mdffgpu_params p;                  /* what the parsers leave in the reference globals */
    /* global (src/global.h) */
    int Fposff;                        /* 0 rnn, 1 rvn, 2 rvf (src/global.c:88-91) */
    int lstatic, lrdf, lpstress, lsymmetric;
    /* md (src/md.h) */
    int npas, nprint, fprint, cprint, tstart, tprint;
    double timesca_baro;
    /* field (src/field.h) */
    int lautoES;
    double epsw;
    int nmass, nqch, ndip, nqua, npol;  /* per-type keyword counts (src/field.c:34-39) */
    /* units: src/constants.c:8-18, or reduced_units (src/constants.c:38-45) */
    double boltz_unit, time_unit, press_unit, coul_unit;
    /* the cell: lattice (src/cell.c:13-91) */
    double B[3][3], omega, inveOmega, inveOmegaPU, w[3], Anorm[3];
    /* POSFF */
    char configname[MDFFH_NAMELEN];
    char cpos[MDFFH_NAMELEN];          /* "Cartesian" or "Direct"/"D" */
    char atypit[MDFFGPU_NTMAX][MDFFH_NAMELEN];
    char (*atypia)[MDFFH_NAMELEN];     /* per-ion type name as read (written back by CONTFF) */
    double *rx, *ry, *rz, *vx, *vy, *vz, *fx, *fy, *fz;
    /* radial distribution (src/radial_distribution.h): resolution, cut-off, bins,
     * configurations to read from TRAJFF */
    double resg, cutgr;
    int nbins, nconf;
    /* output state */
    int oszcall;                       /* OSZIFF records written (src/io.c:58) */
    char err[256];
} mdffh_run;

/* The four set-up calls of the reference's main (src/mdff20.c:74-80), in that order:
 * init_global, read_config (POSFF, wrapped into the cell), init_md, init_field
 * (set_autoES included when lautoES).  posff may be NULL: "POSFF". */
int mdffh_load(mdffh_run *run, const char *controlfn, const char *posff);
void mdffh_free(mdffh_run *run);

/* The steps of mdffh_load one by one. */
int mdffh_init_global(mdffh_run *run, const char *controlfn);
int mdffh_read_config(mdffh_run *run, const char *posff);
int mdffh_init_md(mdffh_run *run, const char *controlfn);
int mdffh_init_field(mdffh_run *run, const char *controlfn);

/* set_autoES (src/ewald.c:48-71): alphaES, kES and cutlongrange from epsw and the cell,
 * with the reference's integer abs() in alpha. */
void mdffh_auto_es(mdffh_run *run);

/* init_velocities (src/kinetic.c:15-28): Maxwell-Boltzmann velocities from the C
 * library's rand() (box_muller, src/rand.c:19-31), centre-of-mass motion removed, then
 * rescale_velocities(0).  The reference never seeds rand(); this call restarts it at
 * the default seed (srand(1)), so it draws the reference's numbers. */
void mdffh_init_velocities(mdffh_run *run);
/* rescale_velocities (src/kinetic.c:83-113) on run->vx..vz; quiet != 0 prints nothing. */
void mdffh_rescale_velocities(mdffh_run *run, int quiet);
/* calc_kin (src/kinetic.c:67-74) of run->vx..vz. */
double mdffh_calc_kin(const mdffh_run *run);

/* write_config (src/config.c:291-345): positions wrapped into the cell, velocities
 * and forces as held in run; mode 'w' (CONTFF) or 'a' (TRAJFF). */
int mdffh_write_config(mdffh_run *run, const char *filename, char mode);

/* info_thermo (src/thermo.c:12-122) at step istep: key 0 prints the thermodynamic
 * block to fp (stdout), key 1 appends one OSZIFF record to fp (with the header
 * every tenth record). */
void mdffh_info_thermo(mdffh_run *run, int key, FILE *fp, int istep, const mdffgpu_thermo *t);
/* info_thermo key 1 appended to the file at path (opened and closed per record). */
int mdffh_oszi_append(mdffh_run *run, const char *path, int istep, const mdffgpu_thermo *t);

/* init_rdf's parameters (src/radial_distribution.c:14-41): resg (default 0.1) and nconf
 * from the control file, cutgr = half the smallest face distance of the POSFF cell.
 * The reference sizes its histogram from the default resg before it reads resg, so
 * nbins = (int)(cutgr / 0.1) + 1 whenever resg >= 0.1; for resg < 0.1, where the
 * reference writes past its histogram, nbins = (int)(cutgr / resg) + 1. */
int mdffh_init_rdf(mdffh_run *run, const char *controlfn);
/* read_next_traj (src/config.c:448-510): the next configuration of a TRAJFF stream into
 * run (cell, positions, velocities, forces; Direct coordinates converted). */
int mdffh_read_traj(mdffh_run *run, FILE *fp);
/* write_rdf (src/radial_distribution.c:96-146) from the ordered-pair counts
 * pairs[nbins][ntype][ntype] of nconf configurations: the all-pairs count added into
 * [0][0] as get_gr does, normalised per type pair by nconf * 4 pi (resg r^2 + resg^3/12)
 * / volume * nionit[a] * nionit[b], and written as lines of ntype(ntype+1)/2 (r, g)
 * pairs taken in the order (0,0), (0,1), ... of the full type matrix, as the
 * reference's loop leaves them.  The volume is that of the last configuration read. */
int mdffh_write_rdf(mdffh_run *run, const long long *pairs, int nconf, const char *path);

/* iopnode / iopsnode (src/io.c:62-69). */
int mdffh_iopnode(int step, int npas, int every);
int mdffh_iopsnode(int step, int npas, int every, int start);

#ifdef __cplusplus
}
#endif
#endif
