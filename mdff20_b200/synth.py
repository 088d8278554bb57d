"""Seeded synthetic inputs for the five benchmark systems and for the parity tests.

No public dataset exists for this path; these generators ARE the workloads.  Every
generator takes a seed and uses numpy's PCG64, so the same call gives the same system.

* ``lj_fcc``      : n-m Lennard-Jones argon on an fcc lattice (reduced units), the
                    ``bin/cubic.py`` lattice of the reference.
* ``silica``      : Si:O = 1:2 placed by random sequential addition with a minimum
                    separation, at a given mass density, with the Buckingham silica
                    parameters, point charges and (optionally) O polarisability with
                    Tang-Toennies damping of the charge-dipole field.

Type order is O (type 0) then Si (type 1), as in the reference's own silica inputs
(src/control_SiO.s).  With this order the damping entries lpoldamping[O][O][O] and
lpoldamping[O][O][Si] survive the reference's table symmetrisation, which copies
[t][i][k] onto [t][k][i] with i < k winning (src/field.c:209-219).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .system import BOLTZ_UNIT, RHO_UNIT, System

MASS_O = 15.9994
MASS_SI = 28.0855
O, SI = 0, 1


def maxwell_boltzmann(masses: np.ndarray, kT: float, rng: np.random.Generator) -> np.ndarray:
    """Gaussian velocities with zero total momentum, rescaled exactly to kT.

    Same recipe as maxwellboltzmann_velocities + rescale_velocities
    (src/kinetic.c:42-64, 83-113): sigma = sqrt(kT/m), subtract the mean velocity,
    scale by sqrt(T0/T) with T = 2 E_kin / (3 N kB), subtract the mean again.
    """
    n = masses.shape[0]
    v = rng.standard_normal((n, 3)) * np.sqrt(kT / masses)[:, None]
    v -= v.mean(axis=0)
    ekin = 0.5 * float(np.sum(masses[:, None] * v * v))
    t_now = 2.0 * ekin / (3.0 * n)
    v *= math.sqrt(kT / t_now)
    v -= v.mean(axis=0)
    return v


def lj_fcc(ncell: int = 4, rho: float = 0.8442, temp: float = 0.728, seed: int = 1,
           rc: float = 2.5, skin: float = 0.3, dt: float = 0.005, npas: int = 1000,
           trunc: str = "linear") -> System:
    """Config 1: 4*ncell^3 LJ atoms, reduced units, NVE velocity Verlet."""
    n = 4 * ncell ** 3
    L = (n / rho) ** (1.0 / 3.0)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1)
    frac = (g.reshape(-1, 1, 3) + basis[None]).reshape(-1, 3) / ncell
    pos = frac * L
    rng = np.random.Generator(np.random.PCG64(seed))
    vel = maxwell_boltzmann(np.ones(n), temp, rng)
    one = np.ones((1, 1))
    return System(
        cell=np.eye(3) * L, type_names=["A"], nionit=[n], pos=pos, vel=vel, name="lj_fcc",
        mass=[1.0], lreduced=True, lnmlj=True, trunc=trunc, sigmalj=one, epslj=one,
        plj=one * 6.0, qlj=one * 12.0, cutshortrange=rc, cutlongrange=rc, skindiff=skin,
        integrator="nve-vv", dt=dt, temp=temp, npas=npas,
    )


def box_length(n_si: int, n_o: int, density: float) -> float:
    """Cubic box edge (Å) holding n_si Si + n_o O at `density` g/cm^3 (src/field.c:186-193)."""
    mass = n_si * MASS_SI + n_o * MASS_O
    return (mass * RHO_UNIT / density) ** (1.0 / 3.0)


def random_sequential_addition(types: np.ndarray, L: float, dmin: np.ndarray, rng: np.random.Generator,
                               batch: int = 2048, max_rounds: int = 100000) -> np.ndarray:
    """Random sequential addition in a cubic box: ion i (in the given order) is placed at
    the first uniform trial point that keeps dmin[type_i, type_j] (minimum image) to
    every ion placed before it.  Trials are drawn `batch` at a time per type and tested
    against the placed ions with a periodic k-d tree; inside a batch the earlier
    accepted trial wins."""
    from scipy.spatial import cKDTree

    n = types.shape[0]
    dmax = float(np.max(dmin))
    pos = np.empty((n, 3))
    placed = 0
    tree = None
    rounds = 0
    while placed < n:
        rounds += 1
        if rounds > max_rounds:
            raise RuntimeError("random sequential addition failed: box too dense")
        t = types[placed]
        # a run of consecutive ions of the same type shares one batch of trials
        run = 1
        while placed + run < n and types[placed + run] == t and run < batch:
            run += 1
        cand = rng.random((batch, 3)) * L
        ok = np.ones(batch, bool)
        if tree is not None:
            kq = min(32, placed)
            dist, idx = tree.query(cand, k=kq, distance_upper_bound=dmax)
            dist = dist.reshape(batch, kq)
            idx = idx.reshape(batch, kq)
            valid = idx < placed
            lim = np.where(valid, dmin[t][types[np.minimum(idx, placed - 1)]], 0.0)
            ok = ~np.any(valid & (dist < lim), axis=1)
        cand = cand[ok]
        acc = []
        d_tt2 = dmin[t, t] ** 2
        for k in range(cand.shape[0]):
            if len(acc) == run:
                break
            if acc:
                d = cand[k] - cand[acc]
                d -= L * np.round(d / L)
                if np.any(np.einsum("ij,ij->i", d, d) < d_tt2):
                    continue
            acc.append(k)
        m = len(acc)
        if m:
            pos[placed:placed + m] = cand[acc]
            placed += m
            tree = cKDTree(np.mod(pos[:placed], L), boxsize=L)
    return pos


def cristobalite(ncell: int, density: float = 2.20, jitter: float = 0.0,
                 rng: Optional[np.random.Generator] = None):
    """Ideal beta-cristobalite supercell (ncell^3 cubic cells of 8 SiO2), scaled to the
    given density: Si on a diamond lattice, O halfway along every Si-Si bond.  Returns
    (positions grouped O then Si, box edge); `jitter` adds seeded Gaussian displacements."""
    fcc = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    bonds = np.array([[.25, .25, .25], [.25, -.25, -.25], [-.25, .25, -.25], [-.25, -.25, .25]])
    si_cell = np.concatenate([fcc, fcc + 0.25])
    o_cell = (fcc[:, None, :] + bonds[None, :, :] * 0.5).reshape(-1, 3)
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 1, 3)
    si = (g + si_cell[None]).reshape(-1, 3)
    o = (g + o_cell[None]).reshape(-1, 3)
    L = box_length(si.shape[0], o.shape[0], density)
    a = L / ncell
    pos = np.concatenate([o, si]) * a
    if jitter > 0.0:
        pos = pos + rng.standard_normal(pos.shape) * jitter
    pos -= L * np.round(pos / L)
    return pos, L


def silica(n_si: int, seed: int, density: float = 2.20, dmin=1.4,
           polarizable: bool = False, rc_sr: float = 7.0, rc_lr: float = 10.0,
           alpha: float = 0.32, kmax: int = 12, skin: float = 1.0,
           integrator: str = "nvt-nhcn", temp: float = 3000.0, dt: float = 0.001,
           npas: int = 1000, nhc_n: int = 3, timesca_thermo: float = 0.1,
           conv_tol: float = 1e-6, extrapolate_order: int = 0,
           damping: bool = True, velocities: bool = True, L: Optional[float] = None,
           structure: str = "random", jitter: float = 0.05) -> System:
    """Configs 2, 3 and 5: silica with Buckingham short range and Ewald electrostatics.

    Buckingham (BHMFT without damping, D=0) Si-O A=18003.7572 eV, B=4.87318 1/Å,
    C=133.5381 eV Å^6; O-O A=1388.7730, B=2.76, C=175.0; Si-Si zero.  q_Si=+2.4,
    q_O=-1.2.  With ``polarizable``, alpha_O = 1 Å^3 (isotropic), alpha_Si = 0 and the
    charge->dipole field on O is Tang-Toennies damped, f_4(b r) with b=2, c=1.
    ``dmin`` is one minimum separation for all pairs or a (2,2) table by type.
    ``structure`` "random": random sequential addition; "cristobalite": beta-cristobalite
    supercell (n_si = 8 m^3) with seeded Gaussian displacements of rms `jitter` Å.
    """
    n_o = 2 * n_si
    n = n_si + n_o
    rng = np.random.Generator(np.random.PCG64(seed))
    if structure == "cristobalite":
        m = round((n_si / 8) ** (1.0 / 3.0))
        if 8 * m ** 3 != n_si:
            raise ValueError("cristobalite needs n_si = 8 m^3")
        pos, L = cristobalite(m, density, jitter, rng)
    else:
        if L is None:
            L = box_length(n_si, n_o, density)
        types = np.array([O] * n_o + [SI] * n_si)
        dm = np.full((2, 2), float(dmin)) if np.isscalar(dmin) else np.asarray(dmin, float)
        # placement order alternates the species in runs of 64 ions so neither fills the box first
        order = np.concatenate([np.concatenate([np.arange(n_o)[k * 128:(k + 1) * 128],
                                                n_o + np.arange(n_si)[k * 64:(k + 1) * 64]])
                                for k in range((n_si + 63) // 64)])
        pos = np.empty((n, 3))
        pos[order] = random_sequential_addition(types[order], L, dm, rng)
        pos -= L * np.round(pos / L)      # centre on the origin like the reference's POSFF files
    masses = np.array([MASS_O] * n_o + [MASS_SI] * n_si)
    vel = maxwell_boltzmann(masses, temp * BOLTZ_UNIT, rng) if velocities else None
    A = np.zeros((2, 2)); B = np.zeros((2, 2)); C = np.zeros((2, 2)); D = np.zeros((2, 2))
    A[O, O] = 1388.7730; B[O, O] = 2.76; C[O, O] = 175.0
    A[O, SI] = A[SI, O] = 18003.7572; B[O, SI] = B[SI, O] = 4.87318; C[O, SI] = C[SI, O] = 133.5381
    s = System(
        cell=np.eye(3) * L, type_names=["O", "Si"], nionit=[n_o, n_si], pos=pos, vel=vel,
        name=f"silica{n}", mass=[MASS_O, MASS_SI], lbhmft=True, Abhmftd=A, Bbhmftd=B,
        Cbhmftd=C, Dbhmftd=D, BDbhmftd=np.zeros((2, 2)), cutshortrange=rc_sr,
        cutlongrange=rc_lr, skindiff=skin, lcoulombic=True, qit=[-1.2, 2.4],
        alphaES=alpha, kES=(kmax, kmax, kmax), lautoES=False, epsw=1e-6,
        integrator=integrator, temp=temp, dt=dt, npas=npas, nhc_n=nhc_n, nhc_mults=2,
        nhc_yosh_order=3, timesca_thermo=timesca_thermo,
        conv_tol_ind=conv_tol, algo_pim="scf", algo_extrapolate_dipole="aspc",
        extrapolate_order=extrapolate_order, min_scf_pim_iter=3, max_scf_pim_iter=200,
    )
    if polarizable:
        pol = np.zeros((2, 3, 3))
        pol[O] = np.eye(3) * 1.0
        s.polit = pol
        if damping:
            s.poldamp = [(O, O, O, 2.0, 1.0, 4), (O, O, SI, 2.0, 1.0, 4)]
    return s


# ----------------------------------------------------------------------------------
# the five benchmark systems
def config1() -> System:
    return lj_fcc(ncell=4, rho=0.8442, temp=0.728, seed=1)


def config2() -> System:
    return silica(1000, seed=2, polarizable=False, kmax=12, temp=3000.0, npas=1000)


# Minimum separations (Å, O/Si by type) for the polarisable systems.  With one 1.4 Å
# minimum for every pair, random O-O contacts make alpha*T exceed 1 and the induced-dipole
# problem has no bounded solution (the polarisation catastrophe); these values keep
# O-O and Si-Si contacts at distances found in dense silica.
PIM_DMIN = np.array([[2.3, 1.5], [1.5, 2.8]])


def config3() -> System:
    s = silica(2000, seed=3, polarizable=True, kmax=14, integrator="nve-vv", temp=0.0,
               conv_tol=1e-8, velocities=False, dmin=PIM_DMIN)
    s.lstatic = True
    return s


def config5(structure: str = "cristobalite", cells: int = 10) -> System:
    """N = 24000 polarisable silica, NHC (chain 3) at 2500 K, 1 Å skin, SCF to 1e-6 with
    ASPC order 4.  MD starts from a 10^3 beta-cristobalite supercell at 2.20 g/cm^3
    (L = 71.3 Å) with 0.05 Å seeded displacements: a random packing of these ions falls
    into the Buckingham short-range divergence within tens of steps.  `cells` < 10: the
    same model on a cells^3 supercell (24 cells^3 ions), the small case of profiles."""
    return silica(8 * cells ** 3, seed=6, polarizable=True, kmax=14, temp=2500.0, npas=10000,
                  conv_tol=1e-6, extrapolate_order=4, dmin=PIM_DMIN, structure=structure)
