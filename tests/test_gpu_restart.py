"""Exact restart: a context loaded from mdffgpu_save_state continues the saved run bit
for bit (ASPC history, Nose-Hoover chain, list-build positions and step count carried),
through list rebuilds, in the reference solver, the FP64 CG and the mixed fused-CG graph
path.  The reference's own restart file (CONTFF) loses that state."""
import numpy as np
import pytest

from mdff20_b200.engine import FP64, MIXED, PIM_CG, PIM_CG_FUSED, PIM_REFERENCE, Engine, MdffgpuError
from tests.golden import cases
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu

MODES = {
    "reference_aspc_nhc": dict(pim_solver=PIM_REFERENCE, precision=FP64),
    "cg_fp64": dict(pim_solver=PIM_CG, precision=FP64),
    "fused_mixed_graph": dict(pim_solver=PIM_CG_FUSED, precision=MIXED),
}


def system(skin=0.1, integrator="nvt-nhcn"):
    g = load_golden("crist192_pim_nhc")
    s = cases.crist192(True, integrator=integrator, temp=2500.0, extrapolate_order=3, skin=skin)
    s.vel = g["vel"].reshape(-1, 3)
    return s, g["r_in"].reshape(-1, 3)


def start(s, pos, **kw):
    e = Engine(s, positions=pos, **kw)
    e.gen_verletlist()
    e.engforce()
    return e


@pytest.mark.parametrize("mode", sorted(MODES))
def test_restart_is_bit_exact(mode):
    s, pos = system()
    kw = MODES[mode]
    a = start(s, pos, **kw)
    ta = a.md_steps(1, 14)
    sa = a.state()
    a.close()
    assert ta[13, 9] > ta[6, 9], "the window after the restart should contain a list rebuild"

    b = start(s, pos, **kw)
    b.md_steps(1, 6)
    blob = b.save_state()
    b.close()

    c = Engine(s, positions=pos + 0.3, **kw)   # whatever it starts from is replaced
    assert c.load_state(blob) == 6
    tc = c.md_steps(7, 8)
    sc = c.state()
    again = c.save_state()
    c.close()
    assert np.array_equal(tc, ta[6:]), np.abs(tc - ta[6:]).max()
    for x, y in zip(sc, sa):
        assert np.array_equal(x, y)
    assert len(again) == len(blob)


def test_restart_rejects_other_system():
    s, pos = system()
    b = start(s, pos)
    blob = b.save_state()
    b.close()
    other, _ = system(integrator="nve-vv")
    c = Engine(other, positions=pos)
    with pytest.raises(MdffgpuError) as ex:
        c.load_state(blob)
    assert ex.value.code == 1
    with pytest.raises(MdffgpuError):
        c.load_state(blob[:-8])
    c.close()
