"""Host-side description of one mdff20 system: cell, ions, force field and MD settings.

It mirrors the reference's two inputs, the keyword control file and the POSFF
configuration, and writes both in the reference's formats:

* POSFF (read by ``read_config``, src/config.c:347-446): nion, a name, the three
  lattice vectors as rows of A (``simuCell.A[i][j]``, src/config.c:376-380), ntype, the
  type names, ions per type, ``Cartesian``/``Direct``, then one line per ion with the
  type name, position and, for Fposff rvn/rvf, velocity and force (src/config.c:412-421).
  Ions must come grouped by type in type order, as ``init_config`` assigns types in
  blocks of ``nionit`` (src/config.c:135-148).
* the control file, a whitespace-token keyword scan done once per module
  (src/global.c:13-60, src/md.c:29-98, src/field.c:31-183, src/nmlj.c:39-107,
  src/bhmftd.c:26-90, src/pim.c:28-69).  Per-type keys (massit, qit, dipit, polit) are
  positional in type order (src/field.c:67-108); pair tables are read as upper
  triangles (src/nmlj.c:51-59, src/bhmftd.c:39-47).

The same object feeds the CUDA engine through the C-ABI (``mdff20_b200.engine``).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# constants of src/constants.c:8-18
BOLTZ_UNIT = 8.61734229648141e-05
TIME_UNIT = 98.2269514139276
PRESS_UNIT = 0.00624150964712042
RHO_UNIT = 1.660538782
COUL_UNIT = 14.3996441494161

INTEGRATORS = ("nve-lf", "nve-vv", "nvt-nhcn")   # src/md.c:102-104
TRUNC_TYPES = ("no", "linear", "quadratic")        # src/nmlj.c:128-130
ALGO_PIM = ("scf", "scfkO")                        # src/pim.c:74-75
ALGO_EXTRAPOLATE = ("poly", "aspc")                # src/pim.c:77-78


def _upper(t: np.ndarray) -> List[float]:
    n = t.shape[0]
    return [float(t[i, j]) for i in range(n) for j in range(n) if j >= i]


@dataclass
class System:
    """One configuration plus its force field, in the reference's units (eV, Å, amu, ps, K)."""

    cell: np.ndarray                      # (3,3) rows are lattice vectors a, b, c
    type_names: List[str]
    nionit: List[int]
    pos: np.ndarray                       # (N,3) Cartesian, grouped by type
    vel: Optional[np.ndarray] = None      # (N,3) internal velocity units
    name: str = "mdff20_b200"
    mass: List[float] = field(default_factory=list)
    # ---- global (src/global.c:366-377 defaults)
    lverletL: bool = True
    skindiff: float = 0.15
    cutshortrange: float = 0.0
    cutlongrange: float = 0.0
    lstatic: bool = False
    lreduced: bool = False
    lpstress: bool = False
    # ---- short range
    lnmlj: bool = False
    lbhmft: bool = False
    lbhmftd: bool = False
    trunc: str = "no"
    sigmalj: Optional[np.ndarray] = None
    epslj: Optional[np.ndarray] = None
    plj: Optional[np.ndarray] = None
    qlj: Optional[np.ndarray] = None
    Abhmftd: Optional[np.ndarray] = None
    Bbhmftd: Optional[np.ndarray] = None
    Cbhmftd: Optional[np.ndarray] = None
    Dbhmftd: Optional[np.ndarray] = None
    BDbhmftd: Optional[np.ndarray] = None
    # ---- electrostatics
    lcoulombic: bool = False
    qit: List[float] = field(default_factory=list)
    dipit: Optional[np.ndarray] = None    # (ntype,3)
    polit: Optional[np.ndarray] = None    # (ntype,3,3)
    # damping: list of (type, it, jt, b, c, k) meaning lpoldamping[type][it][jt]=true
    poldamp: List[tuple] = field(default_factory=list)
    alphaES: float = 0.0
    kES: tuple = (0, 0, 0)
    lautoES: bool = False
    epsw: float = 0.0
    # ---- pim (src/pim.c:72-85 defaults)
    algo_pim: str = "scf"
    algo_extrapolate_dipole: str = "poly"
    conv_tol_ind: float = 1e-6
    extrapolate_order: int = 0
    min_scf_pim_iter: int = 3
    max_scf_pim_iter: int = 100
    omegakO: float = 0.0
    # ---- md (src/md.c:100-118 defaults)
    integrator: str = "nve-vv"
    dt: float = 0.001
    temp: float = 0.0
    npas: int = 0
    # output periods of run_md (src/md.c:242-281); tprint 0: no trajectory
    nprint: int = 1000000
    fprint: int = 1000000
    cprint: int = 1000000
    tprint: int = 0
    tstart: int = 0
    nhc_n: int = 3
    nhc_mults: int = 1
    nhc_yosh_order: int = 1
    timesca_thermo: float = 0.0
    tauTberendsen: float = 0.0
    nequil: int = 0
    nequilT: int = 1

    # ------------------------------------------------------------------ helpers
    @property
    def nion(self) -> int:
        return int(self.pos.shape[0])

    @property
    def ntype(self) -> int:
        return len(self.type_names)

    def typia(self) -> np.ndarray:
        return np.repeat(np.arange(self.ntype, dtype=np.int32), self.nionit)

    def copy(self) -> "System":
        return dataclasses.replace(
            self, pos=self.pos.copy(), vel=None if self.vel is None else self.vel.copy()
        )

    def volume(self) -> float:
        return float(abs(np.linalg.det(self.cell)))

    def nk(self) -> int:
        """Number of k-vectors of the half k-box, src/kspace.c:21."""
        kx, ky, kz = self.kES
        return kz + ky * (2 * kz + 1) + kx * (2 * ky + 1) * (2 * kz + 1)

    # ------------------------------------------------------------------ writers
    def posff_text(self, with_velocities: bool = True) -> str:
        lines = [f"{self.nion}", self.name]
        for i in range(3):
            lines.append(" ".join(f"{self.cell[i, j]:.17e}" for j in range(3)))
        lines.append(f"{self.ntype}")
        lines.append(" ".join(self.type_names))
        lines.append(" ".join(str(n) for n in self.nionit))
        lines.append("Cartesian")
        names = np.repeat(np.array(self.type_names, dtype=object), self.nionit)
        vel = self.vel if (with_velocities and self.vel is not None) else np.zeros_like(self.pos)
        for i in range(self.nion):
            p = self.pos[i]
            v = vel[i]
            lines.append(
                f"{names[i]} {p[0]:.17e} {p[1]:.17e} {p[2]:.17e} "
                f"{v[0]:.17e} {v[1]:.17e} {v[2]:.17e} 0.0 0.0 0.0"
            )
        return "\n".join(lines) + "\n"

    def control_text(self) -> str:
        b = lambda x: "true" if x else "false"
        L = []
        L += ["Fposff rvf", f"lverletL {b(self.lverletL)}", f"skindiff {self.skindiff!r}",
              f"cutshortrange {self.cutshortrange!r}", f"cutlongrange {self.cutlongrange!r}",
              f"lstatic {b(self.lstatic)}", f"lreduced {b(self.lreduced)}", f"lpstress {b(self.lpstress)}"]
        L += [f"integrator {self.integrator}", f"dt {self.dt!r}", f"temp {self.temp!r}",
              f"npas {self.npas}", f"nprint {self.nprint}", f"fprint {self.fprint}", f"cprint {self.cprint}",
              f"tprint {self.tprint}", f"tstart {self.tstart}",
              f"nequil {self.nequil}", f"nequilT {self.nequilT}", f"tauTberendsen {self.tauTberendsen!r}",
              f"nhc_n {self.nhc_n}", f"nhc_mults {self.nhc_mults}", f"nhc_yosh_order {self.nhc_yosh_order}",
              f"timesca_thermo {self.timesca_thermo!r}"]
        L += [f"lnmlj {b(self.lnmlj)}", f"lbhmft {b(self.lbhmft)}", f"lbhmftd {b(self.lbhmftd)}",
              f"lcoulombic {b(self.lcoulombic)}"]
        for m in self.mass:
            L.append(f"massit {m!r}")
        if self.lnmlj:
            L.append(f"trunc {self.trunc}")
            for key in ("sigmalj", "epslj", "plj", "qlj"):
                t = getattr(self, key)
                if t is not None:
                    L.append(key + " " + " ".join(repr(v) for v in _upper(np.asarray(t, float))))
        if self.lbhmft or self.lbhmftd:
            for key in ("Abhmftd", "Bbhmftd", "Cbhmftd", "Dbhmftd", "BDbhmftd"):
                t = getattr(self, key)
                if t is not None:
                    L.append(key + " " + " ".join(repr(v) for v in _upper(np.asarray(t, float))))
        if self.lcoulombic:
            for q in self.qit:
                L.append(f"qit {q!r}")
            if self.dipit is not None:
                for d in np.asarray(self.dipit, float):
                    L.append("dipit " + " ".join(repr(float(x)) for x in d))
            if self.polit is not None:
                for p in np.asarray(self.polit, float):
                    L.append("polit " + " ".join(repr(float(x)) for x in p.reshape(9)))
            for (t, i, j, bb, cc, kk) in self.poldamp:
                L.append(f"lpoldamping {t} {i} {j} true")
                L.append(f"pol_damp_b {t} {i} {j} {bb!r}")
                L.append(f"pol_damp_c {t} {i} {j} {cc!r}")
                L.append(f"pol_damp_k {t} {i} {j} {int(kk)}")
            L.append(f"lautoES {b(self.lautoES)}")
            L.append(f"epsw {self.epsw!r}")
            L.append(f"alphaES {self.alphaES!r}")
            L.append("kES {} {} {}".format(*self.kES))
            L += [f"algo_pim {self.algo_pim}", f"algo_extrapolate_dipole {self.algo_extrapolate_dipole}",
                  f"conv_tol_ind {self.conv_tol_ind!r}", f"extrapolate_order {self.extrapolate_order}",
                  f"min_scf_pim_iter {self.min_scf_pim_iter}", f"max_scf_pim_iter {self.max_scf_pim_iter}",
                  f"omegakO {self.omegakO!r}"]
        return "\n".join(L) + "\n"

    def write(self, directory: str, control_name: str = "control.s") -> str:
        import os

        with open(os.path.join(directory, "POSFF"), "w") as fp:
            fp.write(self.posff_text())
        path = os.path.join(directory, control_name)
        with open(path, "w") as fp:
            fp.write(self.control_text())
        return path
