"""Batched force matching of the polarisable silica model with adjoint gradients.

The workload of the fit tools of the reference (bin/ drives the mdff20 executable on
perturbed inputs and compares forces): many independent configurations, one force-
matching loss and its gradient with respect to the force-field parameters

    theta = (A, B, C of Si-O, A, B, C of O-O, q_Si (q_O = -q_Si/2), alpha_O, b, c,
             D of Si-O, D of O-O)

with L(theta) = sum_c sum_i |F_i(theta) - F_i^target|^2 / (3 N_total).  The forces come
from the CUDA engine at the converged induced dipoles; the gradient from one adjoint
induced-dipole solve per configuration (mdffgpu_force_match, mdffgpu_fit_batch).

* ``ewald_tune``: the Ewald splitting alpha, the real-space cutoff and kmax of each
  configuration, chosen for a fixed accuracy at the lowest estimated cost.
* ``config4``: the seeded set of configurations (ion counts uniform over 96..1536 in
  steps of 96, Si:O = 1:2, 2.2 g/cm^3) with their tuned Ewald parameters.
* ``ForceMatchBatch``: engines for a set of configurations, loss and gradient at theta.
* ``ForceMatchLoss``: torch.autograd.Function over ForceMatchBatch.
"""
from __future__ import annotations

import copy
import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import synth
from .system import System

PARAM_NAMES = ("A_SiO", "B_SiO", "C_SiO", "A_OO", "B_OO", "C_OO", "q_Si", "alpha_O", "b", "c", "D_SiO", "D_OO")
NPARAM = len(PARAM_NAMES)
O_TYPE, SI_TYPE = synth.O, synth.SI
NUMBER_DENSITY = 0.066151   # silica ions per A^3 at 2.2 g/cm^3


# ---------------------------------------------------------------------------- parameters
def theta_of(s: System) -> np.ndarray:
    """The parameter vector of a polarisable silica System (types O = 0, Si = 1)."""
    o, si = O_TYPE, SI_TYPE
    damp = [d for d in s.poldamp]
    b = damp[0][3] if damp else 0.0
    c = damp[0][4] if damp else 0.0
    return np.array([s.Abhmftd[si, o], s.Bbhmftd[si, o], s.Cbhmftd[si, o],
                     s.Abhmftd[o, o], s.Bbhmftd[o, o], s.Cbhmftd[o, o],
                     s.qit[si], s.polit[o][0, 0], b, c,
                     s.Dbhmftd[si, o], s.Dbhmftd[o, o]], float)


def with_theta(s: System, theta) -> System:
    """A copy of `s` carrying the parameters `theta` (host side, e.g. for the oracle)."""
    t = [float(x) for x in np.asarray(theta, float)]
    o, si = O_TYPE, SI_TYPE
    s2 = copy.deepcopy(s)
    for arr, k in ((s2.Abhmftd, 0), (s2.Bbhmftd, 1), (s2.Cbhmftd, 2)):
        arr[si, o] = arr[o, si] = t[k]
        arr[o, o] = t[3 + k]
    s2.Dbhmftd = np.array(s2.Dbhmftd, float)
    s2.Dbhmftd[si, o] = s2.Dbhmftd[o, si] = t[10]
    s2.Dbhmftd[o, o] = t[11]
    s2.qit = list(s2.qit)
    s2.qit[si] = t[6]
    s2.qit[o] = -0.5 * t[6]
    s2.polit = np.array(s2.polit, float)
    s2.polit[o] = np.eye(3) * t[7]
    s2.poldamp = [(d[0], d[1], d[2], t[8], t[9], d[5]) for d in s2.poldamp]
    return s2


def fd_step(theta, k: int, rel: float = 1e-5) -> float:
    """Central-difference step of parameter k: rel |theta_k|, or for a parameter at zero
    (the C8 dispersion D of the Buckingham configurations) rel times a typical magnitude
    (D ~ 1e3 eV A^8)."""
    t = abs(float(theta[k]))
    return rel * (t if t > 0.0 else 1e3)


def perturbed_theta(theta0, seed: int = 5, frac: float = 0.05) -> np.ndarray:
    """theta0 with every component scaled by 1 + frac or 1 - frac (seeded signs)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sign = rng.choice([-1.0, 1.0], size=len(theta0))
    return np.asarray(theta0, float) * (1.0 + frac * sign)


# ---------------------------------------------------------------------------- autotuner
@dataclass
class EwaldChoice:
    alpha: float
    rc: float        # real-space cutoff, A
    kmax: int
    cost: float      # estimated flops per force evaluation


def _erfc_root(eps: float) -> float:
    """x with erfc(x) = eps (bisection)."""
    lo, hi = 0.0, 10.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if math.erfc(mid) > eps:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def ewald_tune(L: float, n: int, eps: float = 1e-6, rc_max: float = 10.0, skin: float = 0.5,
               pair_flops: float = 300.0, kspace_flops: float = 35.0) -> EwaldChoice:
    """Ewald parameters of a cubic box of side L holding n ions at accuracy eps.

    For a real-space cutoff rc the splitting parameter makes the real-space truncation
    erfc(alpha rc) = eps, and kmax is the smallest integer with
    exp(-(pi kmax / (alpha L))^2) <= eps (the reciprocal-space truncation).  The
    estimated cost of one force evaluation, pair_flops per real-space pair within rc
    plus kspace_flops per (ion, k) of the half k-box, is minimised over rc in
    [3 A, min(rc_max, L/2 - skin)] (minimum image)."""
    rho = n / L ** 3
    xr = _erfc_root(eps)
    xk = math.sqrt(-math.log(eps))
    rc_hi = min(rc_max, 0.5 * L - skin)
    if rc_hi < 3.0:
        raise ValueError("box too small for the minimum-image real-space sum")
    best = None
    for rc in np.arange(3.0, rc_hi + 1e-9, 0.05):
        alpha = xr / rc
        kmax = max(1, math.ceil(alpha * L * xk / math.pi))
        nk = kmax + kmax * (2 * kmax + 1) + kmax * (2 * kmax + 1) ** 2
        cost = n * (pair_flops * 0.5 * rho * 4.0 / 3.0 * math.pi * rc ** 3 + kspace_flops * nk)
        if best is None or cost < best.cost:
            best = EwaldChoice(alpha=float(alpha), rc=float(rc), kmax=int(kmax), cost=float(cost))
    return best


def ewald_converged(L: float, rc: float, eps: float = 1e-12) -> EwaldChoice:
    """Ewald parameters at the real-space cutoff rc whose truncation errors are below eps
    (default 1e-12): the converged sum a tuned choice at the same rc is measured against.
    (The cutoff itself is kept: the reference applies the Tang-Toennies damping
    correction -(1 - f_k(b r)) T to the pairs inside it only, src/ewald.c:536-539 and
    :567-600, so with damping the sum depends on rc whatever alpha and kmax.)"""
    alpha = _erfc_root(eps) / rc
    kmax = max(1, math.ceil(alpha * L * math.sqrt(-math.log(eps)) / math.pi))
    return EwaldChoice(alpha=float(alpha), rc=float(rc), kmax=int(kmax), cost=float("nan"))


def with_ewald(s: System, ch: EwaldChoice) -> System:
    """A copy of `s` with the Ewald splitting, real-space cutoff and kmax of `ch`."""
    s2 = copy.deepcopy(s)
    s2.alphaES = ch.alpha
    s2.cutlongrange = ch.rc
    s2.kES = (ch.kmax, ch.kmax, ch.kmax)
    return s2


# ---------------------------------------------------------------------------- config 4
def config4_sizes(nconf: int = 512, seed: int = 4) -> List[int]:
    rng = np.random.Generator(np.random.PCG64(seed))
    return [96 * int(k) for k in rng.integers(1, 17, size=nconf)]


def config4_one(c: int, n: int, seed: int = 4, eps: float = 1e-6, conv_tol: float = 1e-8) -> System:
    """Configuration number c (n ions) of the batched force-matching set."""
    n_si = n // 3
    L = (n / NUMBER_DENSITY) ** (1.0 / 3.0)
    ch = ewald_tune(L, n, eps=eps)
    rc_sr = min(7.0, ch.rc)
    s = synth.silica(n_si, seed=seed * 100003 + c, polarizable=True, rc_sr=rc_sr, rc_lr=ch.rc, skin=0.5,
                     alpha=ch.alpha, kmax=ch.kmax, integrator="nve-vv", temp=0.0, velocities=False,
                     conv_tol=conv_tol, dmin=synth.PIM_DMIN, L=L)
    s.lstatic = True
    s.name = f"fit{c}_{n}"
    return s


def _one(args):
    return config4_one(*args)


def config4(nconf: int = 512, seed: int = 4, eps: float = 1e-6, conv_tol: float = 1e-8,
            sizes: Optional[Sequence[int]] = None, indices: Optional[Sequence[int]] = None,
            workers: int = 1) -> List[System]:
    """The batched force-matching set: polarisable silica configurations (config 3's
    model) of seeded sizes, random sequential placement with the PIM minimum
    separations, each with its tuned Ewald parameters (single points, skin 0.5 A).
    indices: which configurations of the set (default all); workers > 1 builds them in
    that many spawned processes."""
    sizes = list(sizes) if sizes is not None else config4_sizes(nconf, seed)
    idx = list(indices) if indices is not None else list(range(len(sizes)))
    jobs = [(c, sizes[c], seed, eps, conv_tol) for c in idx]
    if workers > 1 and len(jobs) > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_one, jobs, chunksize=max(1, len(jobs) // (4 * workers))))
    return [_one(j) for j in jobs]


# ---------------------------------------------------------------------------- sharding
def shard(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Configuration indices per rank: size-balanced greedy bins (largest first to the
    least-loaded rank; cost ~ ions), each bin in ascending order."""
    load = [0.0] * world
    bins: List[List[int]] = [[] for _ in range(world)]
    for c in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        bins[r].append(c)
        load[r] += sizes[c]
    return [sorted(b) for b in bins]


def allreduce_loss_grad(loss: float, grad, group=None):
    """Sum (loss, grad) over the ranks of a torch.distributed group (one all-reduce of
    1 + NPARAM doubles: the only exchange of the sharded fit)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([loss] + list(np.asarray(grad, float)), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    v = t.cpu().numpy()
    return float(v[0]), v[1:].copy()


# ---------------------------------------------------------------------------- batch
class ForceMatchBatch:
    """Engines for a list of configurations; loss and adjoint gradient at theta.

    recorded (default): every configuration's evaluation is recorded once as a CUDA graph
    (mdffgpu_fit_plan) and replayed per evaluation, all configurations in flight at once;
    otherwise mdffgpu_fit_batch drives the contexts from `threads` host threads."""

    def __init__(self, systems: Sequence[System], targets: Optional[Sequence[np.ndarray]], device: int = -1,
                 precision: int = 0, threads: int = 8, ntot: Optional[int] = None, recorded: bool = True):
        """ntot: ions of the whole fit when these systems are one shard of it (the loss is
        normalised by 3 ntot), default the ions of these systems."""
        self.recorded = recorded
        self._plan = None
        from .engine import PIM_CG, Engine, load_library
        from .cellmath import wrap_positions
        self.L = load_library()
        self.systems = list(systems)
        self.engines = []
        for s in self.systems:
            e = Engine(s, positions=wrap_positions(s.cell, s.pos), device=device, precision=precision,
                       pim_solver=PIM_CG)
            e.gen_verletlist()
            self.engines.append(e)
        self.ntot = ntot if ntot is not None else sum(s.nion for s in self.systems)
        self.scale = 2.0 / (3.0 * self.ntot)
        self.threads = threads
        n = len(self.engines)
        self._ctx = (C.c_void_p * n)(*[e.h.value for e in self.engines])
        if targets is None:   # set later (set_targets), e.g. from forces() of this batch
            targets = [np.zeros((s.nion, 3)) for s in self.systems]
        self.set_targets(targets)

    def set_precision(self, precision: int):
        for e in self.engines:
            e._check(e.L.mdffgpu_set_precision(e.h, precision))

    def loss_grad(self, theta) -> tuple:
        """(L, dL/dtheta) of L = sum |F - F_t|^2 / (3 N_total)."""
        th = np.ascontiguousarray(np.asarray(theta, float))
        if self.recorded:
            if self._plan is None:
                from .engine import FitPlan
                self._plan = FitPlan(self.engines, SI_TYPE, O_TYPE, self.targets, self.scale)
            sq, grad = self._plan.eval(th)
            return 0.5 * self.scale * sq, grad
        res = np.zeros(1 + NPARAM)
        rc = self.L.mdffgpu_fit_batch(self._ctx, len(self.engines), SI_TYPE, O_TYPE,
                                      th.ctypes.data_as(C.POINTER(C.c_double)), self._tgt, self.scale,
                                      self.threads, res.ctypes.data_as(C.POINTER(C.c_double)))
        if rc != 0:
            from .engine import MdffgpuError
            raise MdffgpuError(rc, "mdffgpu_fit_batch failed")
        return 0.5 * self.scale * res[0], res[1:].copy()

    def set_targets(self, targets: Sequence[np.ndarray]):
        if getattr(self, "_plan", None) is not None:   # the plan holds the old targets on the device
            self._plan.close()
            self._plan = None
        self.targets = [np.ascontiguousarray(np.asarray(t, float).reshape(-1, 3)) for t in targets]
        n = len(self.engines)
        self._tgt = (C.POINTER(C.c_double) * n)(*[t.ctypes.data_as(C.POINTER(C.c_double))
                                                  for t in self.targets])

    def forces(self, theta) -> List[np.ndarray]:
        out = []
        for e in self.engines:
            e.fit_set_params(SI_TYPE, O_TYPE, theta)
            e.engforce()
            out.append(e.forces())
        return out

    def close(self):
        if self._plan is not None:
            self._plan.close()
            self._plan = None
        for e in self.engines:
            e.close()
        self.engines = []


def target_forces(systems: Sequence[System], theta_t, device: int = -1) -> List[np.ndarray]:
    """FP64 forces of every configuration at the parameters theta_t (the fit targets)."""
    from .engine import PIM_CG, Engine
    from .cellmath import wrap_positions
    out = []
    for s in systems:
        e = Engine(s, positions=wrap_positions(s.cell, s.pos), device=device, pim_solver=PIM_CG)
        e.gen_verletlist()
        e.fit_set_params(SI_TYPE, O_TYPE, theta_t)
        e.engforce()
        out.append(e.forces())
        e.close()
    return out


try:
    import torch

    class ForceMatchLoss(torch.autograd.Function):
        """L(theta) of a ForceMatchBatch; backward returns the adjoint gradient."""

        @staticmethod
        def forward(ctx, theta, batch: ForceMatchBatch):
            loss, grad = batch.loss_grad(theta.detach().cpu().double().numpy())
            ctx.save_for_backward(torch.as_tensor(grad, dtype=theta.dtype, device=theta.device))
            return torch.as_tensor(loss, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad, None
except ImportError:   # torch is optional for the C-ABI users
    ForceMatchLoss = None
