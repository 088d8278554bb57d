"""Python binding of libmdffhost.so (include/mdffhost.h): the reference's input and
output files.

``load_inputs(control, posff)`` reads a control file and a POSFF exactly as the
reference's parsers do (init_global, read_config, init_md, init_field,
src/mdff20.c:74-80) and returns the parsed run (``HostRun``, the C struct) together
with a ``System`` built from it, so a reference input directory can drive the engine
from Python.  ``write_config`` and ``oszi_record`` produce the reference's CONTFF/TRAJFF
and OSZIFF text.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from .engine import NT, Params, Thermo
from .system import ALGO_EXTRAPOLATE, ALGO_PIM, INTEGRATORS, TRUNC_TYPES, System

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdffhost.so")
NAMELEN = 81
D, I = C.c_double, C.c_int


class HostRun(C.Structure):
    """mdffh_run of include/mdffhost.h."""

    _fields_ = [
        ("p", Params), ("Fposff", I), ("lstatic", I), ("lrdf", I), ("lpstress", I), ("lsymmetric", I),
        ("npas", I), ("nprint", I), ("fprint", I), ("cprint", I), ("tstart", I), ("tprint", I),
        ("timesca_baro", D), ("lautoES", I), ("epsw", D), ("nmass", I), ("nqch", I), ("ndip", I),
        ("nqua", I), ("npol", I), ("boltz_unit", D), ("time_unit", D), ("press_unit", D), ("coul_unit", D),
        ("B", D * 9), ("omega", D), ("inveOmega", D), ("inveOmegaPU", D), ("w", D * 3), ("Anorm", D * 3),
        ("configname", C.c_char * NAMELEN), ("cpos", C.c_char * NAMELEN),
        ("atypit", (C.c_char * NAMELEN) * NT), ("atypia", C.c_void_p),
        ("rx", C.POINTER(D)), ("ry", C.POINTER(D)), ("rz", C.POINTER(D)),
        ("vx", C.POINTER(D)), ("vy", C.POINTER(D)), ("vz", C.POINTER(D)),
        ("fx", C.POINTER(D)), ("fy", C.POINTER(D)), ("fz", C.POINTER(D)),
        ("resg", D), ("cutgr", D), ("nbins", I), ("nconf", I),
        ("oszcall", I), ("err", C.c_char * 256),
    ]

    def xyz(self, which: str) -> np.ndarray:
        """(nion, 3) copy of positions ("r"), velocities ("v") or forces ("f")."""
        n = self.p.nion
        cols = [getattr(self, which + a) for a in "xyz"]
        return np.stack([np.ctypeslib.as_array(c, (n,)).copy() for c in cols], axis=1)

    def set_xyz(self, which: str, a: np.ndarray) -> None:
        n = self.p.nion
        a = np.asarray(a, float).reshape(n, 3)
        for k, c in enumerate("xyz"):
            np.ctypeslib.as_array(getattr(self, which + c), (n,))[:] = a[:, k]


_lib = None


def load_library(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built: run `make -C mdff20_b200`")
    L = C.CDLL(path)
    rp = C.POINTER(HostRun)
    sig = {
        "mdffh_load": ([rp, C.c_char_p, C.c_char_p], I),
        "mdffh_free": ([rp], None),
        "mdffh_auto_es": ([rp], None),
        "mdffh_init_velocities": ([rp], None),
        "mdffh_rescale_velocities": ([rp, I], None),
        "mdffh_calc_kin": ([rp], D),
        "mdffh_write_config": ([rp, C.c_char_p, C.c_char], I),
        "mdffh_iopnode": ([I, I, I], I),
        "mdffh_iopsnode": ([I, I, I, I], I),
        "mdffh_oszi_append": ([rp, C.c_char_p, I, C.POINTER(Thermo)], I),
        "mdffh_init_rdf": ([rp, C.c_char_p], I),
        "mdffh_read_traj": ([rp, C.c_void_p], I),
        "mdffh_write_rdf": ([rp, C.POINTER(C.c_longlong), I, C.c_char_p], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


class Inputs:
    """A parsed control file + POSFF; frees the C arrays on close()."""

    def __init__(self, control: str, posff: Optional[str] = None):
        self.lib = load_library()
        self.run = HostRun()
        rc = self.lib.mdffh_load(C.byref(self.run), control.encode(), None if posff is None else posff.encode())
        if rc != 0:
            msg = self.run.err.decode()
            self.lib.mdffh_free(C.byref(self.run))
            raise ValueError(f"reference input rejected: {msg}")

    def close(self) -> None:
        if self.lib is not None:
            self.lib.mdffh_free(C.byref(self.run))
            self.lib = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def system(self) -> System:
        """The parsed run as a System (positions wrapped as read_config leaves them)."""
        return system_from_run(self.run)

    def init_velocities(self) -> np.ndarray:
        self.lib.mdffh_init_velocities(C.byref(self.run))
        return self.run.xyz("v")

    def init_rdf(self, control: str) -> Tuple[float, float, int, int]:
        """init_rdf's parameters: (resg, cutgr, nbins, nconf)."""
        if self.lib.mdffh_init_rdf(C.byref(self.run), control.encode()) != 0:
            raise ValueError(self.run.err.decode())
        r = self.run
        return r.resg, r.cutgr, r.nbins, r.nconf

    def traj_frames(self, path: str, nconf: int):
        """The first nconf configurations of a TRAJFF file (read_next_traj), as
        [(cell (3,3), Cartesian positions (N,3))]."""
        libc = C.CDLL(None)
        libc.fopen.restype = C.c_void_p
        libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
        libc.fclose.argtypes = [C.c_void_p]
        fp = libc.fopen(path.encode(), b"r")
        if not fp:
            raise FileNotFoundError(path)
        frames = []
        try:
            for _ in range(nconf):
                if self.lib.mdffh_read_traj(C.byref(self.run), fp) != 0:
                    raise ValueError(self.run.err.decode())
                frames.append((np.array(self.run.p.cell[:], float).reshape(3, 3), self.run.xyz("r")))
        finally:
            libc.fclose(fp)
        return frames

    def write_rdf(self, pairs: np.ndarray, nconf: int, path: str) -> None:
        pairs = np.ascontiguousarray(pairs, dtype=np.int64)
        if self.lib.mdffh_write_rdf(C.byref(self.run), pairs.ctypes.data_as(C.POINTER(C.c_longlong)), int(nconf),
                                    path.encode()) != 0:
            raise OSError(self.run.err.decode())

    def write_config(self, path: str, mode: str = "w") -> None:
        if self.lib.mdffh_write_config(C.byref(self.run), path.encode(), mode.encode()) != 0:
            raise OSError(self.run.err.decode())


def _table(flat, nt: int) -> np.ndarray:
    return np.array([[flat[i * NT + j] for j in range(nt)] for i in range(nt)], float)


def system_from_run(r: HostRun) -> System:
    p = r.p
    nt = p.ntype
    sym = lambda t: np.triu(t) + np.triu(t, 1).T   # init_nmlj / init_bhmftd copy it <= jt down
    s = System(
        cell=np.array(p.cell[:], float).reshape(3, 3),
        type_names=[r.atypit[t].value.decode() for t in range(nt)],
        nionit=[p.nionit[t] for t in range(nt)],
        pos=r.xyz("r"), vel=r.xyz("v"), name=r.configname.decode(),
        mass=[p.massit[t] for t in range(nt)] if r.nmass else [],
        lverletL=bool(p.lverletL), skindiff=p.skindiff, cutshortrange=p.cutshortrange,
        cutlongrange=p.cutlongrange, lstatic=bool(r.lstatic), lreduced=bool(p.lreduced),
        lpstress=bool(r.lpstress), lnmlj=bool(p.lnmlj), lbhmft=bool(p.lbhmft), lbhmftd=bool(p.lbhmftd),
        trunc=TRUNC_TYPES[p.trunctype], lcoulombic=bool(p.lcoulombic),
        alphaES=p.alphaES, kES=tuple(p.kES[:]), lautoES=False, epsw=r.epsw,
        algo_pim=ALGO_PIM[p.algo_pim], algo_extrapolate_dipole=ALGO_EXTRAPOLATE[p.algo_extrapolate_dipole],
        conv_tol_ind=p.conv_tol_ind, extrapolate_order=p.extrapolate_order,
        min_scf_pim_iter=p.min_scf_pim_iter, max_scf_pim_iter=p.max_scf_pim_iter, omegakO=p.omegakO,
        integrator=INTEGRATORS[p.egrator], dt=p.dt, temp=p.temp, npas=r.npas,
        nprint=r.nprint, fprint=r.fprint, cprint=r.cprint, tprint=r.tprint, tstart=r.tstart,
        nhc_n=p.nhc_n, nhc_mults=p.nhc_mults, nhc_yosh_order=p.nhc_yosh_order,
        timesca_thermo=p.timesca_thermo, tauTberendsen=p.tauTberendsen, nequil=p.nequil, nequilT=p.nequilT,
    )
    if p.lnmlj:
        for key in ("sigmalj", "epslj", "plj", "qlj"):
            setattr(s, key, sym(_table(getattr(p, key), nt)))
    if p.lbhmft or p.lbhmftd:
        for key in ("Abhmftd", "Bbhmftd", "Cbhmftd", "Dbhmftd", "BDbhmftd"):
            setattr(s, key, sym(_table(getattr(p, key), nt)))
    if p.lcoulombic:
        s.qit = [p.qit[t] for t in range(nt)]
        s.dipit = np.array(p.dipit[:], float).reshape(NT, 3)[:nt].copy()
        s.polit = np.array(p.polit[:], float).reshape(NT, 3, 3)[:nt].copy()
        for t in range(nt):
            for i in range(nt):
                for j in range(nt):
                    k = (t * NT + i) * NT + j
                    if p.lpoldamping[k]:
                        s.poldamp.append((t, i, j, p.pol_damp_b[k], p.pol_damp_c[k], p.pol_damp_k[k]))
    return s


def load_inputs(control: str, posff: Optional[str] = None) -> Tuple[System, HostRun]:
    """Parse a reference input pair; returns (System, parsed HostRun copy)."""
    with Inputs(control, posff) as inp:
        s = inp.system()
        run = HostRun.from_buffer_copy(inp.run)
    run.atypia = None
    for c in "xyz":
        for w in "rvf":
            setattr(run, w + c, C.POINTER(D)())
    return s, run


def oszi_text(run_like: HostRun, records) -> str:
    """OSZIFF text for a sequence of (istep, Thermo) records, through info_thermo key 1."""
    lib = load_library()
    import tempfile
    r = HostRun.from_buffer_copy(run_like)
    r.oszcall = 0
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "OSZIFF")
        open(path, "w").close()
        for istep, t in records:
            if lib.mdffh_oszi_append(C.byref(r), path.encode(), int(istep), C.byref(t)) != 0:
                raise OSError(r.err.decode())
        with open(path) as fp:
            return fp.read()
