"""ctypes front end of the C restatement (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, as the checker.  ``params_from_system`` fills the C parameter block from a
``mdff20_b200.system.System`` exactly as the reference's parsers would fill its
globals from the control file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
NT = 16

D = C.c_double
I = C.c_int


class OrcParams(C.Structure):
    _fields_ = [
        ("nion", I), ("ntype", I), ("nionit", I * NT), ("massit", D * NT), ("cell", D * 9),
        ("lreduced", I), ("lverletL", I), ("skindiff", D), ("cutshortrange", D), ("cutlongrange", D),
        ("lnmlj", I), ("trunctype", I), ("sigmalj", D * (NT * NT)), ("epslj", D * (NT * NT)),
        ("plj", D * (NT * NT)), ("qlj", D * (NT * NT)), ("lbhmft", I), ("lbhmftd", I),
        ("Abhmftd", D * (NT * NT)), ("Bbhmftd", D * (NT * NT)), ("Cbhmftd", D * (NT * NT)),
        ("Dbhmftd", D * (NT * NT)), ("BDbhmftd", D * (NT * NT)), ("lcoulombic", I), ("qit", D * NT),
        ("dipit", D * (NT * 3)), ("polit", D * (NT * 9)), ("lpoldamping", I * (NT ** 3)),
        ("pol_damp_b", D * (NT ** 3)), ("pol_damp_c", D * (NT ** 3)), ("pol_damp_k", I * (NT ** 3)),
        ("alphaES", D), ("kES", I * 3), ("algo_pim", I), ("algo_extrapolate_dipole", I),
        ("extrapolate_order", I), ("min_scf_pim_iter", I), ("max_scf_pim_iter", I),
        ("conv_tol_ind", D), ("omegakO", D), ("egrator", I), ("nhc_n", I), ("nhc_mults", I),
        ("nhc_yosh_order", I), ("nequil", I), ("nequilT", I), ("dt", D), ("temp", D),
        ("timesca_thermo", D), ("tauTberendsen", D),
    ]


class OrcThermo(C.Structure):
    _fields_ = [
        ("e_kin", D), ("e_nvt", D), ("u_lj", D), ("u_bhmftd", D), ("u_coul", D), ("u_pol", D),
        ("pvir_lj", D), ("pvir_bhmftd", D), ("pvir_coul", D), ("tau_lj", D * 9),
        ("tau_bhmftd", D * 9), ("tau_coul", D * 9), ("utail", D), ("ptail", D), ("scf_rmsd", D),
        ("scf_iter", I), ("nlist_builds", I),
    ]


def fill_params(P, s) -> None:
    """Fill a parameter block (OrcParams or the engine's identical layout) from a System."""
    from mdff20_b200.system import ALGO_EXTRAPOLATE, ALGO_PIM, INTEGRATORS, TRUNC_TYPES

    nt = s.ntype
    P.nion = s.nion
    P.ntype = nt
    for i in range(nt):
        P.nionit[i] = int(s.nionit[i])
        P.massit[i] = float(s.mass[i]) if s.mass else 1.0
    for k, v in enumerate(np.asarray(s.cell, float).reshape(9)):
        P.cell[k] = float(v)
    P.lreduced = int(s.lreduced)
    P.lverletL = int(s.lverletL)
    P.skindiff = s.skindiff
    P.cutshortrange = s.cutshortrange
    P.cutlongrange = s.cutlongrange
    P.lnmlj = int(s.lnmlj)
    P.trunctype = TRUNC_TYPES.index(s.trunc)

    def tab(name, arr, default=0.0):
        dst = getattr(P, name)
        a = np.full((nt, nt), default) if arr is None else np.asarray(arr, float)
        for i in range(nt):
            for j in range(nt):
                dst[i * NT + j] = float(a[i, j])

    if s.lnmlj:
        # default_nmlj, src/nmlj.c:110-119
        tab("sigmalj", s.sigmalj, 3.405)
        tab("epslj", s.epslj, 0.010323576)
        tab("plj", s.plj, 6.0)
        tab("qlj", s.qlj, 12.0)
    P.lbhmft = int(s.lbhmft)
    P.lbhmftd = int(s.lbhmftd)
    for name in ("Abhmftd", "Bbhmftd", "Cbhmftd", "Dbhmftd", "BDbhmftd"):
        tab(name, getattr(s, name))
    P.lcoulombic = int(s.lcoulombic)
    if s.lcoulombic:
        for i, q in enumerate(s.qit):
            P.qit[i] = float(q)
        if s.dipit is not None:
            d = np.asarray(s.dipit, float)
            for i in range(nt):
                for k in range(3):
                    P.dipit[i * 3 + k] = float(d[i, k])
        if s.polit is not None:
            p = np.asarray(s.polit, float).reshape(nt, 9)
            for i in range(nt):
                for k in range(9):
                    P.polit[i * 9 + k] = float(p[i, k])
        for (t, i, j, b, c, k) in s.poldamp:
            idx = (t * NT + i) * NT + j
            P.lpoldamping[idx] = 1
            P.pol_damp_b[idx] = float(b)
            P.pol_damp_c[idx] = float(c)
            P.pol_damp_k[idx] = int(k)
    P.alphaES = s.alphaES
    for k in range(3):
        P.kES[k] = int(s.kES[k])
    P.algo_pim = ALGO_PIM.index(s.algo_pim)
    P.algo_extrapolate_dipole = ALGO_EXTRAPOLATE.index(s.algo_extrapolate_dipole)
    P.extrapolate_order = s.extrapolate_order
    P.min_scf_pim_iter = s.min_scf_pim_iter
    P.max_scf_pim_iter = s.max_scf_pim_iter
    P.conv_tol_ind = s.conv_tol_ind
    P.omegakO = s.omegakO
    P.egrator = INTEGRATORS.index(s.integrator)
    P.nhc_n = s.nhc_n
    P.nhc_mults = s.nhc_mults
    P.nhc_yosh_order = s.nhc_yosh_order
    P.nequil = s.nequil
    P.nequilT = s.nequilT
    P.dt = s.dt
    P.temp = s.temp
    P.timesca_thermo = s.timesca_thermo
    P.tauTberendsen = s.tauTberendsen


def wrapped_positions(s) -> np.ndarray:
    """Positions as read_config leaves them (src/config.c:442-444): fractional wrap by
    nearbyint, then back to Cartesian, with the reference's operation order."""
    from mdff20_b200.cellmath import wrap_positions

    return wrap_positions(s.cell, s.pos)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "restate"], check=True, stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(OrcParams), dp, dp]
        L.orc_destroy.argtypes = [vp]
        for name, args in [("orc_set_positions", [vp, dp]), ("orc_set_velocities", [vp, dp]),
                           ("orc_get_state", [vp, dp, dp, dp]), ("orc_get_dipoles", [vp, dp]),
                           ("orc_set_dipole_history", [vp, dp]), ("orc_get_dipole_history", [vp, dp]),
                           ("orc_set_nhc", [vp, dp, dp]), ("orc_get_nhc", [vp, dp, dp]),
                           ("orc_set_istep", [vp, I]), ("orc_get_thermo", [vp, C.POINTER(OrcThermo)])]:
            getattr(L, name).argtypes = args
            getattr(L, name).restype = None
        for name, args in [("orc_gen_verletlist", [vp]), ("orc_check_verletlist", [vp]),
                           ("orc_get_verletlist", [vp, I, ip, ip, I]), ("orc_engforce", [vp]),
                           ("orc_multipole_es", [vp, dp, dp, I, D, dp, dp, dp, dp, dp, dp]),
                           ("orc_md_step", [vp, I]), ("orc_md", [vp, I, dp]), ("orc_md_from", [vp, I, I, dp]), ("orc_nion", [vp]),
                           ("orc_nk", [vp])]:
            getattr(L, name).argtypes = args
            getattr(L, name).restype = C.c_int
        L.orc_gr.argtypes = [I, dp, dp, ip, I, D, D, I, C.POINTER(C.c_longlong)]
        L.orc_gr.restype = None
        _lib = L
    return _lib


def gr_counts(frames, nionit, cutgr: float, resg: float, nbins: int) -> np.ndarray:
    """get_gr (src/radial_distribution.c:180-230) over frames [(cell (3,3), pos (N,3))]:
    ordered-pair counts hist[nbins][nt][nt] (without the reference's all-pairs tally in
    [0][0])."""
    L = lib()
    nt = len(nionit)
    typ = np.ascontiguousarray(np.repeat(np.arange(nt, dtype=np.int32), nionit))
    hist = np.zeros((nbins, nt, nt), dtype=np.int64)
    for cell, pos in frames:
        cell = np.ascontiguousarray(cell, float)
        pos = np.ascontiguousarray(pos, float)
        L.orc_gr(len(typ), _dp(cell), _dp(pos), typ.ctypes.data_as(C.POINTER(C.c_int)), nt, float(cutgr),
                 float(resg), int(nbins), hist.ctypes.data_as(C.POINTER(C.c_longlong)))
    return hist


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


ES_FLAGS = dict(lq=1, ld=2, ldamp=4, do_forces=8, do_stress=16, do_ef=32, do_efg=64, do_dir=128, do_rec=256)


class Oracle:
    """One system held by the C restatement."""

    def __init__(self, s, wrap: bool = True):
        self.L = lib()
        self.P = OrcParams()
        fill_params(self.P, s)
        pos = wrapped_positions(s) if wrap else np.ascontiguousarray(s.pos, float)
        self._pos = np.ascontiguousarray(pos, float)
        vel = None if s.vel is None else np.ascontiguousarray(s.vel, float)
        self.n = s.nion
        self.h = self.L.orc_create(C.byref(self.P), _dp(self._pos), _dp(vel) if vel is not None else None)

    def __del__(self):
        try:
            if self.h:
                self.L.orc_destroy(self.h)
        except Exception:
            pass

    def set_positions(self, pos):
        self._pos = np.ascontiguousarray(pos, float)
        self.L.orc_set_positions(self.h, _dp(self._pos))

    def set_velocities(self, vel):
        v = np.ascontiguousarray(vel, float)
        self.L.orc_set_velocities(self.h, _dp(v))

    # ---------------------------------------------------------------- lists
    def gen_verletlist(self):
        rc = self.L.orc_gen_verletlist(self.h)
        if rc:
            raise RuntimeError(f"orc_gen_verletlist failed {rc}")

    def verletlist(self, which: int):
        point = np.zeros(self.n + 1, np.int32)
        cap = 500 * self.n
        lst = np.zeros(cap, np.int32)
        cnt = self.L.orc_get_verletlist(self.h, which, _ip(point), _ip(lst), cap)
        if cnt < 0:
            raise RuntimeError("verlet list unavailable")
        return point, lst[:cnt].copy()

    def check_verletlist(self) -> bool:
        return bool(self.L.orc_check_verletlist(self.h))

    # ---------------------------------------------------------------- forces
    def engforce(self):
        rc = self.L.orc_engforce(self.h)
        if rc:
            raise RuntimeError(f"orc_engforce failed {rc}")

    def state(self):
        pos = np.zeros((self.n, 3)); vel = np.zeros((self.n, 3)); f = np.zeros((self.n, 3))
        self.L.orc_get_state(self.h, _dp(pos), _dp(vel), _dp(f))
        return pos, vel, f

    def forces(self):
        return self.state()[2]

    def thermo(self) -> dict:
        t = OrcThermo()
        self.L.orc_get_thermo(self.h, C.byref(t))
        out = {k: getattr(t, k) for k, _ in OrcThermo._fields_}
        for k in ("tau_lj", "tau_bhmftd", "tau_coul"):
            out[k] = np.array(out[k][:]).reshape(3, 3)
        return out

    def dipoles(self):
        mu = np.zeros((self.n, 3))
        self.L.orc_get_dipoles(self.h, _dp(mu))
        return mu

    def set_dipole_history(self, h):
        h = np.ascontiguousarray(h, float).reshape(self.n, 6, 3)
        self.L.orc_set_dipole_history(self.h, _dp(h))

    def dipole_history(self):
        h = np.zeros((self.n, 6, 3))
        self.L.orc_get_dipole_history(self.h, _dp(h))
        return h

    def set_istep(self, istep: int):
        self.L.orc_set_istep(self.h, istep)

    def multipole_es(self, q, mu, alpha: float = 0.0, **flags):
        q = np.ascontiguousarray(q, float)
        mu = np.ascontiguousarray(mu, float).reshape(self.n, 3)
        fl = 0
        for k, v in flags.items():
            if v:
                fl |= ES_FLAGS[k]
        u = np.zeros(1); pv = np.zeros(1); tau = np.zeros(9)
        ef = np.zeros((self.n, 3)); efg = np.zeros((self.n, 9)); f = np.zeros((self.n, 3))
        rc = self.L.orc_multipole_es(self.h, _dp(q), _dp(mu), fl, alpha, _dp(u), _dp(pv), _dp(tau), _dp(ef),
                                     _dp(efg), _dp(f))
        if rc:
            raise RuntimeError(f"orc_multipole_es failed {rc}")
        return dict(u=u[0], pvir=pv[0], tau=tau.reshape(3, 3), ef=ef, efg=efg.reshape(self.n, 3, 3), f=f)

    # ---------------------------------------------------------------- md
    def md(self, nsteps: int, first: int = 1):
        """Forces at t = 0, then nsteps steps with step indices first, first + 1, ..."""
        th = np.zeros((nsteps + 1, 12))
        rc = self.L.orc_md_from(self.h, first, nsteps, _dp(th))
        if rc:
            raise RuntimeError(f"orc_md failed {rc}")
        return th

    def md_step(self, istep: int):
        rc = self.L.orc_md_step(self.h, istep)
        if rc:
            raise RuntimeError(f"orc_md_step failed {rc}")

    def set_nhc(self, xi, vxi):
        xi = np.ascontiguousarray(xi, float); vxi = np.ascontiguousarray(vxi, float)
        self.L.orc_set_nhc(self.h, _dp(xi), _dp(vxi))

    def nhc(self):
        xi = np.zeros(16); vxi = np.zeros(16)
        self.L.orc_get_nhc(self.h, _dp(xi), _dp(vxi))
        k = int(self.P.nhc_n)
        return xi[:k], vxi[:k]
