"""Radial distribution function on the GPU: the reference's lrdf mode
(src/radial_distribution.c) through the C ABI (mdffgpu_rdf_*).

``RDF`` accumulates the pair histogram of get_gr (src/radial_distribution.c:180-230)
over configurations, given as host arrays (``add``) or as the current positions of an
``Engine`` (``add_engine``, without leaving the device).  ``g_of_r`` turns the counts
into g(r) per ordered type pair; ``rdfff_text`` writes them the way write_rdf
(src/radial_distribution.c:96-146) lays out RDFFF, including its quirks (the all-pairs
tally folded into the first type pair, the first ntype(ntype+1)/2 entries of the full
type matrix).  There is no CPU path: without the library or a device every call raises.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence, Tuple

import numpy as np

from .cellmath import lattice
from .engine import MdffgpuError, load_library


def reference_grid(cell, resg: float = 0.1) -> Tuple[float, int]:
    """init_rdf's cut-off and bin count (src/radial_distribution.c:37-42): cutgr is half
    the smallest face distance; the reference counts bins with the default resolution 0.1
    before it reads resg, so that count holds for resg >= 0.1 (for a finer resg, where the
    reference overruns its histogram, the bins are counted with resg itself)."""
    _, _, w = lattice(np.asarray(cell, float))
    cutgr = 0.5 * float(min(w))
    return cutgr, int(cutgr / (0.1 if resg >= 0.1 else resg)) + 1


class RDF:
    """Pair-histogram accumulator on one GPU (mdffgpu_rdf_create)."""

    def __init__(self, nionit: Sequence[int], cutgr: float, resg: float = 0.1, nbins: int = 0, device: int = 0):
        self.L = load_library()
        self.nionit = [int(x) for x in nionit]
        self.nt = len(self.nionit)
        self.n = sum(self.nionit)
        self.cutgr, self.resg = float(cutgr), float(resg)
        self.nbins = int(nbins) if nbins else int(self.cutgr / self.resg) + 1
        arr = (C.c_int * self.nt)(*self.nionit)
        h = C.c_void_p()
        rc = self.L.mdffgpu_rdf_create(self.n, self.nt, arr, self.cutgr, self.resg, self.nbins, int(device),
                                       C.byref(h))
        if rc != 0:
            raise MdffgpuError(rc, "mdffgpu_rdf_create failed")
        self.h = h

    def _check(self, rc: int):
        if rc != 0:
            msg = self.L.mdffgpu_rdf_last_error(self.h)
            raise MdffgpuError(rc, msg.decode() if msg else "")

    def add(self, cell, pos) -> None:
        """One configuration: cell rows (3,3) and Cartesian positions (N,3), ions in type blocks."""
        cell = np.ascontiguousarray(cell, float).reshape(9)
        pos = np.asarray(pos, float).reshape(self.n, 3)
        x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.L.mdffgpu_rdf_add(self.h, dp(cell), dp(x), dp(y), dp(z)))

    def add_engine(self, engine) -> None:
        """The current positions of an Engine holding the same ions, on its device."""
        self._check(self.L.mdffgpu_rdf_add_ctx(self.h, engine.h))

    def counts(self) -> Tuple[np.ndarray, int]:
        """Ordered-pair counts (nbins, nt, nt) and the number of configurations added."""
        out = np.zeros((self.nbins, self.nt, self.nt), dtype=np.int64)
        nconf = C.c_int(0)
        self._check(self.L.mdffgpu_rdf_counts(self.h, out.ctypes.data_as(C.POINTER(C.c_longlong)), C.byref(nconf)))
        return out, nconf.value

    def reset(self) -> None:
        self._check(self.L.mdffgpu_rdf_reset(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.mdffgpu_rdf_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _shell_volume(resg: float, rr: float) -> float:
    # 4 pi (resg r^2 + resg^3 / 12): the shell volume used by write_rdf
    return 4 * math.pi * (resg * rr * rr + (math.pow(resg, 3)) / 12)


def g_of_r(counts: np.ndarray, nconf: int, resg: float, volume: float, nionit) -> Tuple[np.ndarray, np.ndarray]:
    """Bin centres and g(r) per ordered type pair, (nbins,), (nbins, nt, nt): counts over
    nconf * (shell volume / cell volume) * N_a * N_b."""
    nb = counts.shape[0]
    rr = (np.arange(nb) + 0.5) * resg
    vol = np.array([_shell_volume(resg, r) for r in rr]) / volume
    na = np.asarray(nionit, float)
    g = counts / (nconf * vol[:, None, None] * na[None, :, None] * na[None, None, :])
    return rr, g


def rdfff_text(counts: np.ndarray, nconf: int, resg: float, volume: float, nionit) -> str:
    """RDFFF as write_rdf (src/radial_distribution.c:96-146) writes it from these counts."""
    nb, nt, _ = counts.shape
    npairs = nt * (nt + 1) // 2
    lines = []
    for b in range(nb):
        h = counts[b].astype(np.int64)
        rr = (float(b) + 0.5) * resg
        vol = _shell_volume(resg, rr)
        vol = vol / volume
        vals = []
        for a in range(nt):
            for c in range(nt):
                cnt = int(h[a, c]) + (int(h.sum()) if a == 0 and c == 0 else 0)
                vals.append(float(cnt) / float(nconf * vol * nionit[a] * nionit[c]))
        lines.append("".join("%19.12e %19.12e " % (rr, vals[mp]) for mp in range(npairs)) + "\n")
    return "".join(lines)
