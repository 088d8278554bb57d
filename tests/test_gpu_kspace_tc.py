"""The tensor-core rho(k) pass (kspace_tc.cu: tcgen05 TF32 products of split operands,
selected with MDFFGPU_RHO_TC=1) against the CUDA-core FP32 pass and the FP64 engine:
forces, energies and induced dipoles of a full mixed-precision force evaluation (fused
CG: every rho pass of the induced-dipole solve, over the polarisable ions, and the
charge and total-moment passes over every ion go through it) for the N=24000 bench
system (kmax 14: 29 of the 32 MMA columns), a small polarisable system (kmax 5, one
64-row tile), a 450-ion system whose ion count is not a multiple of the 16-ion stage, a
rigid-ion system (charges only); both ion passes beside it; and graph-replayed MD
steps; and a triclinic cell with an unequal k box.  Bars: forces within 1e-5 RMS of FP64
and within 2x (+1e-6) of the CUDA-core pass's error, energies within 1e-5."""
import os

import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.engine import MIXED, PIM_CG, PIM_CG_FUSED, Engine
from oracle.oracle import wrapped_positions
from tests.golden import cases
from tests.helpers import rms_rel

pytestmark = pytest.mark.gpu


class _Env:
    """Environment switches for the engines created inside the block."""

    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update(self.kv)

    def __exit__(self, *exc):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _forces(s, pos, rho_tc, ion_tc=True, **kw):
    with _Env(MDFFGPU_RHO_TC="1" if rho_tc else "0", MDFFGPU_ION_TC="1" if ion_tc else "0"):
        e = Engine(s, positions=pos, **kw)
        e.gen_verletlist()
        e.engforce()
        out = e.forces(), e.thermo(), e.dipole_history()[:, 0, :]
        e.close()
    return out


def _silica450_triclinic():
    """The 450-ion system sheared into a triclinic cell (positions carried along in
    fractional coordinates) with an unequal k box (kmax 5, 6, 7): the phase-table offsets
    and E0 | E1 prefixes of the tensor-core passes in their general form."""
    s = cases.silica450(True)
    frac = s.pos @ np.linalg.inv(s.cell)
    cell = s.cell.copy()
    cell[1, 0] = 1.2
    cell[2, 1] = -0.9
    s.cell = cell
    s.pos = frac @ cell
    s.kES = (5, 6, 7)
    return s


SYSTEMS = {
    "config5": lambda: synth.config5(),
    "silica96": lambda: cases.silica96(True),
    "silica450": lambda: cases.silica450(True),
    "silica96_rigid": lambda: cases.silica96(False),
    "silica450_triclinic": _silica450_triclinic,
}


@pytest.mark.parametrize("which", list(SYSTEMS))
def test_tensor_core_rho_matches(which):
    s = SYSTEMS[which]()
    pos = wrapped_positions(s)
    f64, t64, m64 = _forces(s, pos, False, pim_solver=PIM_CG)
    ftc, ttc, mtc = _forces(s, pos, True, pim_solver=PIM_CG_FUSED, precision=MIXED)
    fcc, tcc, mcc = _forces(s, pos, False, pim_solver=PIM_CG_FUSED, precision=MIXED)
    e_tc, e_cc = rms_rel(ftc, f64), rms_rel(fcc, f64)
    print(f"{which}: force error with the tensor-core rho pass {e_tc:.2e}, CUDA-core pass {e_cc:.2e}")
    assert e_tc < 1e-5 and e_tc < 2 * e_cc + 1e-6, (e_tc, e_cc)
    for k in ("u_coul", "u_pol"):
        assert abs(ttc[k] - t64[k]) < 1e-5 * max(1.0, abs(t64[k])), k
    pol = np.abs(m64).sum(axis=1) > 0   # the induced dipoles (none in the rigid-ion system)
    if pol.any():
        assert rms_rel(mtc[pol], m64[pol]) < 1e-4


def test_tensor_core_rho_with_cuda_core_ion_pass():
    """The tensor-core rho pass beside the CUDA-core ion pass (the other pairing)."""
    s = cases.silica450(True)
    pos = wrapped_positions(s)
    f64, _, _ = _forces(s, pos, False, pim_solver=PIM_CG)
    f, _, _ = _forces(s, pos, True, ion_tc=False, pim_solver=PIM_CG_FUSED, precision=MIXED)
    assert rms_rel(f, f64) < 1e-5


def test_tensor_core_rho_md_steps():
    """Graph-replayed NHC steps with the tensor-core rho pass track the CUDA-core pass's
    (the per-stage tables follow the positions every step)."""
    g = cases.CASES["crist192_pim_nhc_aspc4"]()
    pos = wrapped_positions(g)
    runs = []
    for tc in (True, False):
        with _Env(MDFFGPU_RHO_TC="1" if tc else "0"):
            e = Engine(g, positions=pos, pim_solver=PIM_CG_FUSED, precision=MIXED)
            e.gen_verletlist()
            e.engforce()
            th = e.md_steps(1, 20)
            runs.append((th, e.forces()))
            e.close()
    (ta, fa), (tb, fb) = runs
    assert np.isfinite(ta).all()
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(tb[:, col]).max()))
        assert np.abs(ta[:, col] - tb[:, col]).max() < 1e-5 * scale, col
    assert rms_rel(fa, fb) < 1e-5
