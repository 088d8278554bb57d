"""The tensor-core ion pass (tcgen05 TF32 products of split operands, kspace_ion_tc.cu,
selected with MDFFGPU_ION_TC=1) against the CUDA-core FP32 pass and the FP64 engine:
forces of a full mixed-precision force evaluation (fused CG: the field passes of the
induced-dipole solve over the polarisable ions and the force pass over every ion go
through it) for the N=24000 bench system (kmax 14), a small system (kmax 5) and a
rigid-ion system (charges only); and graph-replayed MD steps."""
import os

import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.engine import MIXED, PIM_CG, PIM_CG_FUSED, Engine
from oracle.oracle import wrapped_positions
from tests.golden import cases
from tests.helpers import load_golden, rms_rel

pytestmark = pytest.mark.gpu


class _IonTc:
    """MDFFGPU_ION_TC for the engines created inside the block."""

    def __init__(self, on: bool):
        self.on = on

    def __enter__(self):
        self.old = os.environ.get("MDFFGPU_ION_TC")
        os.environ["MDFFGPU_ION_TC"] = "1" if self.on else "0"

    def __exit__(self, *exc):
        if self.old is None:
            os.environ.pop("MDFFGPU_ION_TC", None)
        else:
            os.environ["MDFFGPU_ION_TC"] = self.old


def _forces(s, pos, tc, **kw):
    with _IonTc(tc):
        e = Engine(s, positions=pos, **kw)
        e.gen_verletlist()
        e.engforce()
        out = e.forces(), e.thermo(), e.dipole_history()[:, 0, :]
        e.close()
    return out


@pytest.mark.parametrize("which", ["config5", "silica96", "silica96_rigid"])
def test_tensor_core_ion_pass_matches(which):
    if which == "config5":
        s = synth.config5()
    else:
        s = cases.silica96(which == "silica96")
    pos = wrapped_positions(s)
    f64, t64, m64 = _forces(s, pos, False, pim_solver=PIM_CG)
    ftc, ttc, mtc = _forces(s, pos, True, pim_solver=PIM_CG_FUSED, precision=MIXED)
    fcc, tcc, mcc = _forces(s, pos, False, pim_solver=PIM_CG_FUSED, precision=MIXED)
    e_tc, e_cc = rms_rel(ftc, f64), rms_rel(fcc, f64)
    print(f"{which}: force error with the tensor-core ion pass {e_tc:.2e}, CUDA-core pass {e_cc:.2e}")
    assert e_tc < 1e-5 and e_tc < 2 * e_cc + 1e-6, (e_tc, e_cc)
    assert rms_rel(ftc, fcc) < 1e-5
    for k in ("u_coul", "u_pol", "pvir_coul"):
        assert abs(ttc[k] - t64[k]) < 1e-5 * max(1.0, abs(t64[k])), k
    if which != "silica96_rigid":
        # induced dipoles over the polarisable ions (they come first): the solvers stop at
        # the SCF tolerance and the FP32 fields carry ~1e-6 of the dipoles, so RMS |d mu|
        # within 5 x tol x alpha_O (alpha_O = 1 A^3) + 1e-5 RMS |mu|
        pol = s.nionit[0]
        dmu = mtc[:pol] - m64[:pol]
        rms = lambda x: float(np.sqrt(np.mean(np.sum(x ** 2, 1))))
        assert rms(dmu) < 5.0 * s.conv_tol_ind + 1e-5 * rms(m64[:pol]), (rms(dmu), rms(m64[:pol]))


def test_tensor_core_ion_pass_md_steps():
    """Graph-replayed mixed MD steps with the tensor-core ion pass: the trajectory of
    the CUDA-core pass to the mixed force bar."""
    g = load_golden("crist192_pim_nhc")
    s = cases.CASES["crist192_pim_nhc"]()
    s.vel = g["vel"].reshape(-1, 3)
    p0 = g["r_in"].reshape(-1, 3)
    runs = []
    for tc in (True, False):
        with _IonTc(tc):
            e = Engine(s, positions=p0, pim_solver=PIM_CG_FUSED, precision=MIXED)
            e.gen_verletlist()
            e.engforce()
            th = e.md_steps(1, 8)
            runs.append((th, e.forces()))
            e.close()
    (ta, fa), (tb, fb) = runs
    assert np.isfinite(ta).all()
    for col in (0, 3, 4, 5):
        scale = max(1.0, float(np.abs(tb[:, col]).max()))
        assert np.abs(ta[:, col] - tb[:, col]).max() < 1e-5 * scale, col
    assert rms_rel(fa, fb) < 1e-5


def test_launch_tuner_keeps_results():
    """mdffgpu_tune_launch times the k-space launch shapes on the system and keeps the
    fastest; the forces afterwards are the mixed path's within its bar, whichever shape
    won, and the system's state is unchanged."""
    s = cases.silica450(True)
    pos = wrapped_positions(s)
    f64, _, _ = _forces(s, pos, False, pim_solver=PIM_CG)
    e = Engine(s, positions=pos, pim_solver=PIM_CG_FUSED, precision=MIXED)
    e.gen_verletlist()
    e.engforce()
    r0 = e.state()[0].copy()
    t = e.tune_launch(3)
    assert t["field_pass_ms"] > 0.0
    assert (t["rho_chunks"] == 0) == t["tensor_core_rho_pass"] and t["rho_chunks"] >= 0
    assert np.array_equal(e.state()[0], r0)
    e.engforce()
    assert rms_rel(e.forces(), f64) < 1e-5
    th = e.md_steps(1, 6)
    assert np.isfinite(th).all()
    e.close()
