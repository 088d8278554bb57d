"""The launch-overlap machinery of an MD step changes no result.

Side-stream branches (short-range pairs, pair preparation, the real-space passes beside
the k-space ones) and programmatic dependent launch move no arithmetic between kernels and
reorder no reduction, so MD steps -- recorded graphs and kernel-by-kernel -- are
bit-identical with them on and off (MDFFGPU_SIDE_STREAMS, MDFFGPU_PDL, read when a context
is created).  The list rebuild of a recorded step is an IF node whose condition the list
check sets on the device; with a skin small enough to rebuild every few steps the graph
steps reproduce the kernel-by-kernel ones exactly."""
import os

import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.cellmath import wrap_positions
from mdff20_b200.engine import FP64, MIXED, PIM_CG_FUSED, Engine
from tests.golden import cases
from tests.helpers import load_golden

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


def _crist192():
    g = load_golden("crist192_pim_nhc")
    s = cases.CASES["crist192_pim_nhc"]()
    s.vel = g["vel"].reshape(-1, 3)
    return s, g["r_in"].reshape(-1, 3)


def _run(s, pos, precision, nsteps, graph=True, **env):
    with _Env(**env):
        e = Engine(s, positions=pos, pim_solver=PIM_CG_FUSED, precision=precision)
    try:
        e.set_graph(graph)
        e.gen_verletlist()
        e.engforce()
        th = e.md_steps(1, nsteps)
        return th, e.state(), e.forces()
    finally:
        e.close()


def _same(a, b):
    assert np.array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)
    assert np.array_equal(a[2], b[2])


SWITCHES = (dict(MDFFGPU_SIDE_STREAMS="0"), dict(MDFFGPU_PDL="0"),
            dict(MDFFGPU_SIDE_STREAMS="0", MDFFGPU_PDL="0"))


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_overlap_switches_bit_identical(precision):
    s, p0 = _crist192()
    base = _run(s, p0, precision, 10)
    for env in SWITCHES:
        _same(base, _run(s, p0, precision, 10, **env))


def test_overlap_switches_bit_identical_tensor_cores():
    """The bench model on 5184 ions: both k-space passes on the tensor cores (their
    default from 4096 ions), the CG's real-space field on its own branch while the loop
    body is recorded."""
    s = synth.config5(cells=6)
    p0 = wrap_positions(s.cell, s.pos)
    base = _run(s, p0, MIXED, 8)
    for env in SWITCHES[::2]:
        _same(base, _run(s, p0, MIXED, 8, **env))


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_rebuild_if_node_matches_eager(precision):
    s, p0 = _crist192()
    s.skindiff = 0.02   # rebuilds every few steps at 2500 K
    eager = _run(s, p0, precision, 14, graph=False)
    graph = _run(s, p0, precision, 14, graph=True)
    _same(eager, graph)
    nbuilds = graph[0][:, 9]
    # the graph replays start at step extrapolate_order + 1; rebuilds must happen there
    assert nbuilds[-1] - nbuilds[s.extrapolate_order + 1] >= 3


def test_md_steps_host_equals_separate_calls():
    """mdffgpu_md_steps_host (state in, steps, state out, one call) gives what
    set_positions + set_velocities + md_steps + get_state give, bit for bit; NULL input
    components keep the device's values."""
    s, p0 = _crist192()
    n = len(p0)
    rng = np.random.default_rng(3)
    a = Engine(s, positions=p0, pim_solver=PIM_CG_FUSED, precision=MIXED)
    b = Engine(s, positions=p0, pim_solver=PIM_CG_FUSED, precision=MIXED)
    try:
        for e in (a, b):
            e.gen_verletlist()
            e.engforce()
            e.md_steps(1, 6)
        pos = a.state()[0] + rng.normal(scale=1e-3, size=(n, 3))
        vel = a.state()[1] * 1.01
        comp = [np.ascontiguousarray(x[:, k]) for x in (pos, vel) for k in range(3)]
        # separate calls
        a.set_positions_soa(*comp[0:3])
        a.set_velocities_soa(*comp[3:6])
        ta = a.md_steps(7, 3)
        oa = [np.empty(n) for _ in range(9)]
        a.state_soa(*oa)
        # one call
        ob = [np.empty(n) for _ in range(9)]
        tb = b.md_steps_host(7, 3, comp, ob)
        assert np.array_equal(ta, tb)
        for x, y in zip(oa, ob):
            assert np.array_equal(x, y)
        # None entries: velocities kept, out entries skipped
        ta = a.md_steps(10, 1)
        oa2 = [np.empty(n) for _ in range(9)]
        a.state_soa(*oa2)
        ob2 = [np.empty(n) if k in (0, 4, 8) else None for k in range(9)]
        tb = b.md_steps_host(10, 1, [None] * 6, ob2)
        assert np.array_equal(ta, tb)
        for k in (0, 4, 8):
            assert np.array_equal(oa2[k], ob2[k])
    finally:
        a.close()
        b.close()
