"""Python binding of the C ABI (include/mdffgpu.h) of libmdffgpu.so.

``Engine`` holds one system resident on one GPU.  Its methods map one to one onto the
C entry points, which in turn replace the reference's hot-path functions
(gen_pbc_verletlist, check_verletlist, engforce, engforce_nmlj_pbc,
engforce_bhmftd_pbc, multipole_ES, get_dipoles, prop_agate and the run_md loop body).
There is no CPU fallback: without the built library or a CUDA device every call
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .system import ALGO_EXTRAPOLATE, ALGO_PIM, INTEGRATORS, TRUNC_TYPES, System

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdffgpu.so")
NT = 16

D = C.c_double
I = C.c_int

STATUS = {
    0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_LIST_OVERFLOW", 4: "ERR_SCF", 5: "ERR_NONFINITE",
    6: "ERR_STATE", 7: "ERR_NOMEM", 8: "ERR_CELL", 9: "ERR_TIMEOUT",
}
FP64, MIXED = 0, 1
PIM_REFERENCE, PIM_CG, PIM_CG_FUSED = 0, 1, 2
ES_FLAGS = dict(lq=1, ld=2, ldamp=4, do_forces=8, do_stress=16, do_ef=32, do_efg=64, do_dir=128, do_rec=256)


class MdffgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    """mdffgpu_params of include/mdffgpu.h."""

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


class Thermo(C.Structure):
    """mdffgpu_thermo of include/mdffgpu.h."""

    _fields_ = [
        ("e_kin", D), ("e_nvt", D), ("u_lj", D), ("u_bhmftd", D), ("u_coul", D), ("u_pol", D),
        ("pvir_lj", D), ("pvir_bhmftd", D), ("pvir_coul", D), ("tau_lj", D * 9),
        ("tau_bhmftd", D * 9), ("tau_coul", D * 9), ("utail", D), ("ptail", D), ("scf_rmsd", D),
        ("scf_iter", I), ("nlist_builds", I),
    ]


def params_from_system(s: System) -> Params:
    """The parameter block the reference's parsers would leave in its globals."""
    P = Params()
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

    if s.lnmlj:  # default_nmlj, src/nmlj.c:110-119
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
    if s.lcoulombic and s.lautoES:   # init_field runs set_autoES (src/field.c:330-331)
        from .cellmath import auto_es

        P.alphaES, kes, P.cutlongrange = auto_es(s.cell, s.cutlongrange, s.epsw)
        for k in range(3):
            P.kES[k] = kes[k]
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
    return P


EXPORTS = (
    "mdffgpu_create", "mdffgpu_destroy", "mdffgpu_last_error", "mdffgpu_set_precision",
    "mdffgpu_set_pim_solver", "mdffgpu_tune_launch", "mdffgpu_set_graph", "mdffgpu_set_positions", "mdffgpu_set_velocities",
    "mdffgpu_get_state",
    "mdffgpu_set_dipole_history", "mdffgpu_get_dipole_history", "mdffgpu_set_nhc", "mdffgpu_get_nhc",
    "mdffgpu_get_thermo", "mdffgpu_gen_verletlist", "mdffgpu_check_verletlist", "mdffgpu_get_verletlist",
    "mdffgpu_engforce", "mdffgpu_engforce_nmlj", "mdffgpu_engforce_bhmftd", "mdffgpu_multipole_es",
    "mdffgpu_get_dipoles", "mdffgpu_prop_agate", "mdffgpu_md_steps", "mdffgpu_md_steps_host", "mdffgpu_launch_count",
    "mdffgpu_stream", "mdffgpu_fma_peak", "mdffgpu_profile", "mdffgpu_profile_result",
    "mdffgpu_build_lists_noalloc", "mdffgpu_fit_set_params", "mdffgpu_force_match", "mdffgpu_fit_batch",
    "mdffgpu_fit_plan_create", "mdffgpu_fit_plan_eval", "mdffgpu_fit_plan_destroy", "mdffgpu_fit_plan_last_error",
    "mdffgpu_state_size", "mdffgpu_save_state", "mdffgpu_load_state",
    "mdffgpu_rdf_create", "mdffgpu_rdf_destroy", "mdffgpu_rdf_last_error", "mdffgpu_rdf_reset", "mdffgpu_rdf_add",
    "mdffgpu_rdf_add_ctx", "mdffgpu_rdf_counts",
)
FIT_NPARAM = 12

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libmdffgpu.so (or the build named by MDFFGPU_LIBRARY) and declare every
    exported function.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("MDFFGPU_LIBRARY", path)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built: run `make -C mdff20_b200` (or __graft_entry__.build())")
    L = C.CDLL(path)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    vpp = C.POINTER(C.c_void_p)
    sig = {
        "mdffgpu_create": [C.POINTER(Params), dp, dp, dp, dp, dp, dp, I, vpp],
        "mdffgpu_destroy": [vp],
        "mdffgpu_set_precision": [vp, I],
        "mdffgpu_set_pim_solver": [vp, I],
        "mdffgpu_set_graph": [vp, I],
        "mdffgpu_tune_launch": [vp, I, ip, dp],
        "mdffgpu_set_positions": [vp, dp, dp, dp],
        "mdffgpu_set_velocities": [vp, dp, dp, dp],
        "mdffgpu_get_state": [vp, dp, dp, dp, dp, dp, dp, dp, dp, dp],
        "mdffgpu_set_dipole_history": [vp, dp],
        "mdffgpu_get_dipole_history": [vp, dp],
        "mdffgpu_set_nhc": [vp, dp, dp],
        "mdffgpu_get_nhc": [vp, dp, dp],
        "mdffgpu_get_thermo": [vp, C.POINTER(Thermo)],
        "mdffgpu_state_size": [vp, C.POINTER(C.c_size_t)],
        "mdffgpu_save_state": [vp, vp, C.c_size_t],
        "mdffgpu_load_state": [vp, vp, C.c_size_t, ip],
        "mdffgpu_rdf_create": [I, I, ip, D, D, I, I, vpp],
        "mdffgpu_rdf_destroy": [vp],
        "mdffgpu_rdf_reset": [vp],
        "mdffgpu_rdf_add": [vp, dp, dp, dp, dp],
        "mdffgpu_rdf_add_ctx": [vp, vp],
        "mdffgpu_rdf_counts": [vp, C.POINTER(C.c_longlong), ip],
        "mdffgpu_gen_verletlist": [vp],
        "mdffgpu_check_verletlist": [vp, ip],
        "mdffgpu_get_verletlist": [vp, I, ip, ip, I, ip],
        "mdffgpu_engforce": [vp],
        "mdffgpu_engforce_nmlj": [vp, dp, dp, dp],
        "mdffgpu_engforce_bhmftd": [vp, dp, dp, dp],
        "mdffgpu_multipole_es": [vp, dp, dp, I, D, dp, dp, dp, dp, dp, dp],
        "mdffgpu_get_dipoles": [vp, dp, dp],
        "mdffgpu_prop_agate": [vp, I],
        "mdffgpu_md_steps": [vp, I, I, dp],
        "mdffgpu_md_steps_host": [vp, I, I, C.POINTER(dp), dp, C.POINTER(dp)],
        "mdffgpu_fit_set_params": [vp, I, I, dp],
        "mdffgpu_force_match": [vp, I, I, dp, dp, dp, D, dp],
        "mdffgpu_fit_batch": [vpp, I, I, I, dp, C.POINTER(dp), D, I, dp],
        "mdffgpu_fit_plan_create": [vpp, I, I, I, C.POINTER(dp), D, vpp],
        "mdffgpu_fit_plan_eval": [vp, dp, dp],
        "mdffgpu_fit_plan_destroy": [vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.mdffgpu_last_error.argtypes = [vp]
    L.mdffgpu_last_error.restype = C.c_char_p
    L.mdffgpu_launch_count.argtypes = [vp]
    L.mdffgpu_launch_count.restype = C.c_longlong
    L.mdffgpu_stream.argtypes = [vp]
    L.mdffgpu_stream.restype = C.c_void_p
    L.mdffgpu_fma_peak.argtypes = [I, I, dp]
    L.mdffgpu_fma_peak.restype = C.c_int
    L.mdffgpu_profile.argtypes = [vp, C.c_char_p]
    L.mdffgpu_profile.restype = C.c_int
    L.mdffgpu_profile_result.argtypes = [vp, dp, C.POINTER(C.c_longlong), dp]
    L.mdffgpu_profile_result.restype = C.c_int
    L.mdffgpu_build_lists_noalloc.argtypes = [vp, I, dp, D, D, I, vp, vp, I, vp, vp, vp, ip]
    L.mdffgpu_build_lists_noalloc.restype = C.c_int
    L.mdffgpu_rdf_last_error.argtypes = [vp]
    L.mdffgpu_rdf_last_error.restype = C.c_char_p
    L.mdffgpu_fit_plan_last_error.argtypes = [vp]
    L.mdffgpu_fit_plan_last_error.restype = C.c_char_p
    _lib = L
    return L


def fma_peak_tflops(device: int, precision: int = FP64) -> float:
    """Measured FMA-pipe throughput (TFLOP/s) of `device` for FP64 or FP32."""
    L = load_library()
    out = C.c_double(0.0)
    rc = L.mdffgpu_fma_peak(device, precision, C.byref(out))
    if rc != 0:
        raise MdffgpuError(rc, "mdffgpu_fma_peak failed")
    return out.value


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


def _soa_arg(x, n):
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous and x.size == n):
        raise ValueError("per-component arrays must be contiguous float64 of length n")
    return x


def _soa(x):
    x = np.ascontiguousarray(x, float)
    return (np.ascontiguousarray(x[:, 0]), np.ascontiguousarray(x[:, 1]), np.ascontiguousarray(x[:, 2]))


class Engine:
    """One system on one GPU (an mdffgpu context)."""

    def __init__(self, system: System, positions=None, velocities=None, device: int = -1,
                 precision: int = FP64, pim_solver: int = PIM_REFERENCE):
        self.L = load_library()
        self.system = system
        self.n = system.nion
        self.P = params_from_system(system)
        pos = np.asarray(system.pos if positions is None else positions, float)
        vel = system.vel if velocities is None else velocities
        rx, ry, rz = _soa(pos)
        if vel is not None:
            vx, vy, vz = _soa(vel)
        else:
            vx = vy = vz = None
        h = C.c_void_p()
        rc = self.L.mdffgpu_create(C.byref(self.P), _dp(rx), _dp(ry), _dp(rz), _dp(vx), _dp(vy), _dp(vz),
                                   device, C.byref(h))
        if rc != 0:
            raise MdffgpuError(rc, "mdffgpu_create failed")
        self.h = h
        self._check(self.L.mdffgpu_set_precision(self.h, precision))
        self._check(self.L.mdffgpu_set_pim_solver(self.h, pim_solver))

    def tune_launch(self, reps: int = 10) -> dict:
        """Time the mixed k-space launch shapes on this system and keep the fastest
        (mdffgpu_tune_launch)."""
        ch = np.zeros(4, np.int32)
        ms = C.c_double(0.0)
        self._check(self.L.mdffgpu_tune_launch(self.h, reps, _ip(ch), C.byref(ms)))
        return {"tensor_core_rho_pass": bool(ch[3]), "tensor_core_ion_pass": bool(ch[0]), "rho_chunks": int(ch[1]),
                "ion_tc_slices": int(ch[2]), "field_pass_ms": ms.value}

    def set_graph(self, on: bool):
        """Replay MD steps as CUDA graphs (default on); off issues every kernel."""
        self._check(self.L.mdffgpu_set_graph(self.h, 1 if on else 0))

    def close(self):
        if getattr(self, "h", None):
            self.L.mdffgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != 0:
            msg = self.L.mdffgpu_last_error(self.h)
            raise MdffgpuError(rc, msg.decode() if msg else "")

    # ------------------------------------------------------------ state
    def set_positions(self, pos):
        rx, ry, rz = _soa(pos)
        self._check(self.L.mdffgpu_set_positions(self.h, _dp(rx), _dp(ry), _dp(rz)))

    def set_velocities(self, vel):
        vx, vy, vz = _soa(vel)
        self._check(self.L.mdffgpu_set_velocities(self.h, _dp(vx), _dp(vy), _dp(vz)))

    def state(self):
        a = [np.zeros(self.n) for _ in range(9)]
        self._check(self.L.mdffgpu_get_state(self.h, *[_dp(x) for x in a]))
        return np.stack(a[0:3], 1), np.stack(a[3:6], 1), np.stack(a[6:9], 1)

    # the reference's per-component arrays as they are (contiguous float64 of length n,
    # e.g. page-locked buffers): no conversion on the Python side
    def set_positions_soa(self, rx, ry, rz):
        self._check(self.L.mdffgpu_set_positions(self.h, *[_dp(_soa_arg(x, self.n)) for x in (rx, ry, rz)]))

    def set_velocities_soa(self, vx, vy, vz):
        self._check(self.L.mdffgpu_set_velocities(self.h, *[_dp(_soa_arg(x, self.n)) for x in (vx, vy, vz)]))

    def state_soa(self, *out):
        """Positions, velocities and forces into nine given arrays (rx .. fz)."""
        if len(out) != 9:
            raise ValueError("state_soa takes nine arrays")
        self._check(self.L.mdffgpu_get_state(self.h, *[_dp(_soa_arg(x, self.n)) for x in out]))

    def forces(self):
        return self.state()[2]

    def thermo(self) -> dict:
        t = Thermo()
        self._check(self.L.mdffgpu_get_thermo(self.h, C.byref(t)))
        out = {k: getattr(t, k) for k, _ in Thermo._fields_}
        for k in ("tau_lj", "tau_bhmftd", "tau_coul"):
            out[k] = np.array(out[k][:]).reshape(3, 3)
        return out

    def set_dipole_history(self, h):
        h = np.ascontiguousarray(h, float).reshape(self.n, 6, 3)
        self._check(self.L.mdffgpu_set_dipole_history(self.h, _dp(h)))

    def dipole_history(self):
        h = np.zeros((self.n, 6, 3))
        self._check(self.L.mdffgpu_get_dipole_history(self.h, _dp(h)))
        return h

    def set_nhc(self, xi, vxi):
        xi = np.ascontiguousarray(xi, float)
        vxi = np.ascontiguousarray(vxi, float)
        self._check(self.L.mdffgpu_set_nhc(self.h, _dp(xi), _dp(vxi)))

    def nhc(self):
        k = int(self.P.nhc_n)
        xi = np.zeros(max(k, 1))
        vxi = np.zeros(max(k, 1))
        self._check(self.L.mdffgpu_get_nhc(self.h, _dp(xi), _dp(vxi)))
        return xi[:k], vxi[:k]

    def save_state(self) -> bytes:
        """The complete MD state after the last step (mdffgpu_save_state)."""
        nb = C.c_size_t(0)
        self._check(self.L.mdffgpu_state_size(self.h, C.byref(nb)))
        buf = C.create_string_buffer(nb.value)
        self._check(self.L.mdffgpu_save_state(self.h, buf, nb))
        return buf.raw

    def load_state(self, blob: bytes) -> int:
        """Restore a saved state; returns the step it was saved after."""
        step = C.c_int(0)
        buf = C.create_string_buffer(blob, len(blob))
        self._check(self.L.mdffgpu_load_state(self.h, buf, C.c_size_t(len(blob)), C.byref(step)))
        return step.value

    # ------------------------------------------------------------ lists
    def gen_verletlist(self):
        self._check(self.L.mdffgpu_gen_verletlist(self.h))

    def check_verletlist(self) -> bool:
        r = C.c_int(0)
        self._check(self.L.mdffgpu_check_verletlist(self.h, C.byref(r)))
        return bool(r.value)

    def verletlist(self, which: int):
        point = np.zeros(self.n + 1, np.int32)
        cnt = C.c_int(0)
        self._check(self.L.mdffgpu_get_verletlist(self.h, which, _ip(point), None, 0, C.byref(cnt)))
        lst = np.zeros(max(cnt.value, 1), np.int32)
        self._check(self.L.mdffgpu_get_verletlist(self.h, which, _ip(point), _ip(lst), cnt.value, C.byref(cnt)))
        return point, lst[:cnt.value]

    # ------------------------------------------------------------ forces
    def engforce(self):
        self._check(self.L.mdffgpu_engforce(self.h))

    def engforce_nmlj(self):
        u = np.zeros(1); pv = np.zeros(1); tau = np.zeros(9)
        self._check(self.L.mdffgpu_engforce_nmlj(self.h, _dp(u), _dp(pv), _dp(tau)))
        return u[0], pv[0], tau.reshape(3, 3)

    def engforce_bhmftd(self):
        u = np.zeros(1); pv = np.zeros(1); tau = np.zeros(9)
        self._check(self.L.mdffgpu_engforce_bhmftd(self.h, _dp(u), _dp(pv), _dp(tau)))
        return u[0], pv[0], tau.reshape(3, 3)

    def multipole_es(self, q, mu, alpha: float = 0.0, **flags):
        q = np.ascontiguousarray(q, float)
        mu = np.ascontiguousarray(mu, float).reshape(self.n, 3)
        fl = 0
        for k, v in flags.items():
            if v:
                fl |= ES_FLAGS[k]
        u = np.zeros(1); pv = np.zeros(1); tau = np.zeros(9)
        ef = np.zeros((self.n, 3)); efg = np.zeros((self.n, 9)); f = np.zeros((self.n, 3))
        self._check(self.L.mdffgpu_multipole_es(self.h, _dp(q), _dp(mu), fl, alpha, _dp(u), _dp(pv), _dp(tau),
                                                _dp(ef), _dp(efg), _dp(f)))
        return dict(u=u[0], pvir=pv[0], tau=tau.reshape(3, 3), ef=ef, efg=efg.reshape(self.n, 3, 3), f=f)

    def get_dipoles(self):
        mu = np.zeros((self.n, 3)); up = np.zeros(1)
        self._check(self.L.mdffgpu_get_dipoles(self.h, _dp(mu), _dp(up)))
        return mu, up[0]

    # ------------------------------------------------------------ md
    def prop_agate(self, istep: int):
        self._check(self.L.mdffgpu_prop_agate(self.h, istep))

    def md_steps(self, first: int, nsteps: int, record: bool = True):
        th = np.zeros((nsteps, 12)) if record else None
        self._check(self.L.mdffgpu_md_steps(self.h, first, nsteps, _dp(th)))
        return th

    def md_steps_host(self, first: int, nsteps: int, inp=None, out=None, record: bool = True):
        """md_steps with the state on the host in the reference's per-component layout:
        inp (rx ry rz vx vy vz; entries may be None) is copied in first, out (rx ry rz vx
        vy vz fx fy fz; entries may be None) receives the state after the last step.
        Arrays are contiguous float64 of length n (page-locked ones are copied by DMA)."""
        def ptrs(arrs, k):
            if arrs is None:
                return None
            if len(arrs) != k:
                raise ValueError(f"md_steps_host takes {k} arrays here")
            return (C.POINTER(C.c_double) * k)(*[None if x is None else _dp(_soa_arg(x, self.n)) for x in arrs])
        pin, pout = ptrs(inp, 6), ptrs(out, 9)
        th = np.zeros((nsteps, 12)) if record else None
        self._check(self.L.mdffgpu_md_steps_host(self.h, first, nsteps, pin, _dp(th), pout))
        return th

    def launch_count(self) -> int:
        return int(self.L.mdffgpu_launch_count(self.h))

    def profile(self, kernel):
        """Start timing every launch of `kernel` (None stops)."""
        self._check(self.L.mdffgpu_profile(self.h, kernel.encode() if kernel else None))

    def profile_result(self):
        ms = C.c_double(0.0); cnt = C.c_longlong(0); fl = C.c_double(0.0)
        self._check(self.L.mdffgpu_profile_result(self.h, C.byref(ms), C.byref(cnt), C.byref(fl)))
        return ms.value, cnt.value, fl.value

    def stream_handle(self) -> int:
        """The cudaStream_t of this context (for CUDA events around calls)."""
        return int(self.L.mdffgpu_stream(self.h) or 0)

    # ---------------------------------------------------------------- force matching
    def fit_set_params(self, tSi: int, tO: int, theta):
        th = np.ascontiguousarray(np.asarray(theta, float))
        assert th.shape == (FIT_NPARAM,)
        self._check(self.L.mdffgpu_fit_set_params(self.h, tSi, tO, _dp(th)))

    def force_match(self, tSi: int, tO: int, f_target, scale: float):
        """(sum |F - F_t|^2, dL/dtheta) for L = scale/2 sum |F - F_t|^2 at the current parameters."""
        fx, fy, fz = _soa(np.asarray(f_target, float))
        res = np.zeros(1 + FIT_NPARAM)
        self._check(self.L.mdffgpu_force_match(self.h, tSi, tO, _dp(fx), _dp(fy), _dp(fz), scale, _dp(res)))
        return float(res[0]), res[1:].copy()


class FitPlan:
    """mdffgpu_fit_plan: force matching over a set of contexts with each configuration's
    evaluation recorded once as a CUDA graph (device-side CG loops, theta in one device
    buffer), replayed per evaluation."""

    def __init__(self, engines, tSi: int, tO: int, targets, scale: float):
        self.L = load_library()
        n = len(engines)
        self._engines = list(engines)   # the contexts must outlive the plan
        self._ctx = (C.c_void_p * n)(*[e.h.value for e in engines])
        self._tgt_arrays = [np.ascontiguousarray(np.asarray(t, float).reshape(-1, 3)) for t in targets]
        tg = (C.POINTER(C.c_double) * n)(*[t.ctypes.data_as(C.POINTER(C.c_double)) for t in self._tgt_arrays])
        h = C.c_void_p()
        rc = self.L.mdffgpu_fit_plan_create(self._ctx, n, tSi, tO, tg, scale, C.byref(h))
        if rc != 0:
            raise MdffgpuError(rc, "mdffgpu_fit_plan_create failed")
        self.h = h

    def eval(self, theta):
        """(sum of |F - F_t|^2 over every configuration, the summed gradient)."""
        th = np.ascontiguousarray(np.asarray(theta, float))
        assert th.shape == (FIT_NPARAM,)
        res = np.zeros(1 + FIT_NPARAM)
        rc = self.L.mdffgpu_fit_plan_eval(self.h, _dp(th), _dp(res))
        if rc != 0:
            msg = self.L.mdffgpu_fit_plan_last_error(self.h)
            raise MdffgpuError(rc, msg.decode() if msg else "mdffgpu_fit_plan_eval failed")
        return float(res[0]), res[1:].copy()

    def close(self):
        if getattr(self, "h", None):
            self.L.mdffgpu_fit_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
