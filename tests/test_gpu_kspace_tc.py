"""The tensor-core rho(k) pass (tcgen05 TF32 products of split operands, selected with
MDFFGPU_KSPACE_TC=1) against the CUDA-core FP32 pass and the FP64 engine: forces of a full mixed-precision
force evaluation (fused CG: every rho pass of the induced-dipole solve goes through it)
for the N=24000 bench system (kmax 14: 29 of the 32 MMA columns) and for a small system
(kmax 5)."""
import os

import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.engine import MIXED, PIM_CG, PIM_CG_FUSED, Engine
from oracle.oracle import wrapped_positions
from tests.golden import cases

pytestmark = pytest.mark.gpu


def _rms_rel(a, b):
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1))) / np.sqrt(np.mean(np.sum(b ** 2, axis=1))))


def forces(s, pos, tc, **kw):
    old = os.environ.get("MDFFGPU_KSPACE_TC")
    os.environ["MDFFGPU_KSPACE_TC"] = "1" if tc else "0"
    try:
        e = Engine(s, positions=pos, **kw)
        e.gen_verletlist()
        e.engforce()
        f, th = e.forces(), e.thermo()
        e.close()
    finally:
        if old is None:
            os.environ.pop("MDFFGPU_KSPACE_TC", None)
        else:
            os.environ["MDFFGPU_KSPACE_TC"] = old
    return f, th


@pytest.mark.parametrize("which", ["config5", "silica96"])
def test_tensor_core_rho_matches(which):
    s = synth.config5() if which == "config5" else cases.silica96(True)   # kmax 14 / 5
    pos = wrapped_positions(s)
    f64, t64 = forces(s, pos, False, pim_solver=PIM_CG)
    ftc, ttc = forces(s, pos, True, pim_solver=PIM_CG_FUSED, precision=MIXED)
    fcc, _ = forces(s, pos, False, pim_solver=PIM_CG_FUSED, precision=MIXED)
    e_tc, e_cc = _rms_rel(ftc, f64), _rms_rel(fcc, f64)
    print(f"{which}: force error with the tensor-core rho pass {e_tc:.2e}, CUDA-core pass {e_cc:.2e}")
    assert e_tc < 1e-5 and e_tc < 2 * e_cc + 1e-6, (e_tc, e_cc)
    for k in ("u_coul", "u_pol"):
        assert abs(ttc[k] - t64[k]) < 1e-5 * max(1.0, abs(t64[k])), k
