"""The systems behind the golden fixtures (shared by make_golden.py and the tests).

Each case is a small seeded system the compiled reference runs in seconds.  The
fixture stores the reference's own inputs (positions after read_config's wrap,
velocities) next to its outputs, so a test rebuilds the System from here and feeds the
stored positions.

Single points use random packings; MD cases start from a jittered beta-cristobalite
cell (a random packing of these ions collapses into the Buckingham short-range
divergence within tens of steps, in the reference as in the engine).
"""
from __future__ import annotations

import numpy as np

from mdff20_b200 import synth


def lj256():
    return synth.lj_fcc(ncell=4)


def silica96(polarizable: bool, **kw):
    args = dict(rc_sr=4.5, rc_lr=5.0, skin=0.5, kmax=5, alpha=0.6, conv_tol=1e-10, extrapolate_order=0)
    args.update(kw)
    dmin = synth.PIM_DMIN if polarizable else 1.4
    return synth.silica(32, seed=11, polarizable=polarizable, dmin=dmin, **args)


def silica450(polarizable: bool, **kw):
    # L = 18.9 A, list cut 6 A: three cells per edge, so the cell-list path is used
    args = dict(rc_sr=5.0, rc_lr=5.5, skin=0.5, kmax=6, alpha=0.55, conv_tol=1e-10, extrapolate_order=0)
    args.update(kw)
    dmin = synth.PIM_DMIN if polarizable else 1.4
    return synth.silica(150, seed=12, polarizable=polarizable, dmin=dmin, **args)


def crist192(polarizable: bool, **kw):
    # 2x2x2 beta-cristobalite (64 SiO2), L = 14.26 A
    args = dict(rc_sr=5.0, rc_lr=6.0, skin=0.5, kmax=6, alpha=0.5, conv_tol=1e-10, extrapolate_order=0,
                structure="cristobalite", jitter=0.05)
    args.update(kw)
    return synth.silica(64, seed=13, polarizable=polarizable, **args)


def es_inputs(s, seed: int = 0):
    """Charges and random dipoles for multipole_ES flag tests."""
    rng = np.random.default_rng(seed)
    q = np.repeat(np.array([-1.2, 2.4]), s.nionit)
    mu = rng.normal(size=(s.nion, 3)) * 0.1
    return q, mu


# flags lq ld ldamp do_forces do_stress do_ef do_efg do_dir do_rec
ES_FLAG_SETS = [
    (1, 1, 1, 1, 1, 1, 1, 1, 1),
    (0, 1, 0, 0, 0, 1, 0, 1, 1),
    (1, 1, 0, 1, 1, 1, 1, 1, 0),
    (1, 0, 0, 1, 1, 1, 1, 0, 1),
    (1, 0, 1, 0, 0, 1, 0, 1, 1),
    (1, 1, 1, 1, 1, 0, 0, 1, 1),
]
ES_FLAG_NAMES = ["lq", "ld", "ldamp", "do_forces", "do_stress", "do_ef", "do_efg", "do_dir", "do_rec"]

CASES = {
    "lj256": lambda: lj256(),
    "silica96_rigid": lambda: silica96(False),
    "silica96_pim": lambda: silica96(True),
    "silica450_pim": lambda: silica450(True),
    "crist192_nhc": lambda: crist192(False, integrator="nvt-nhcn", temp=3000.0),
    "crist192_pim_nhc": lambda: crist192(True, integrator="nvt-nhcn", temp=2500.0),
    "crist192_pim_vv": lambda: crist192(True, integrator="nve-vv", temp=2500.0),
}
MD_CASES = (("lj256", 50), ("crist192_nhc", 30), ("crist192_pim_nhc", 10), ("crist192_pim_vv", 10))


def silica96_ko():
    """algo_pim scfkO (momentpolaSCFkO, src/pim.c:457-603) with omegakO 0.8."""
    s = silica96(True)
    s.algo_pim = "scfkO"
    s.omegakO = 0.8
    s.conv_tol_ind = 1e-9
    return s


CASES["silica96_ko"] = silica96_ko

# ASPC order 4 (the config-5 bench setting) over NHC steps started at step index 6, past the
# reference's first-steps order switch (src/pim.c:321-333)
ASPC4_FIRST, ASPC4_STEPS = 6, 10
CASES["crist192_pim_nhc_aspc4"] = lambda: crist192(True, integrator="nvt-nhcn", temp=2500.0, extrapolate_order=4)


# ---------------------------------------------------------------- C host (mdff20gpu.x)
def _with(s, **kw):
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def host_runs():
    """Runs of the reference program mdff20.x whose output files (OSZIFF, CONTFF, TRAJFF,
    the stdout thermodynamic blocks) pin the C host's: NHC with induced dipoles and ASPC,
    velocity Verlet with velocity rescaling during equilibration, LJ in reduced units, a static run and a zero-step run (the initial velocities)."""
    pim = dict(integrator="nvt-nhcn", temp=1500.0)
    return {
        "pim_nhc": _with(crist192(True, extrapolate_order=2, **pim),
                         npas=6, nprint=3, fprint=1, cprint=4, tprint=3, tstart=1),
        "rigid_equil": _with(crist192(False, integrator="nve-vv", temp=2000.0),
                             npas=6, nequil=4, nequilT=2, nprint=2, fprint=2, cprint=6, tprint=6),
        "lj_vv": _with(lj256(), tauTberendsen=0.005, npas=5, nprint=5, fprint=1, cprint=5, tprint=5, tstart=6),
        "pim_static": _with(crist192(True), lstatic=True, lpstress=True),
        "pim_init": _with(crist192(True, **pim), npas=0, nprint=1, fprint=1, cprint=1, tprint=1),
    }


def autoes_cases():
    """Systems for set_autoES (src/ewald.c:48-71): cubic and triclinic cells, two epsw."""
    a = _with(crist192(False), lautoES=True, epsw=1e-6)
    b = _with(silica450(False), lautoES=True, epsw=1e-5, cutlongrange=12.0)
    c = _with(crist192(False), lautoES=True, epsw=1e-3)
    c.cell = c.cell.copy()
    c.cell[1, 0] = 1.5
    c.cell[2, 1] = -0.75
    return {"crist192_1e-6": a, "silica450_1e-5": b, "crist192_tri_1e-3": c}
