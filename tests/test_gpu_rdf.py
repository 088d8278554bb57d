"""The GPU pair histogram (mdffgpu_rdf_*) against the reference's get_gr and the
oracle: integer counts identical, for the reference's own histograms, a 3000-ion
triclinic system, a histogram too large for shared memory, device-resident positions of
an Engine, and the C host's lrdf mode writing RDFFF."""
import os
import subprocess

import numpy as np
import pytest

from mdff20_b200 import cellmath, rdf, synth
from mdff20_b200.engine import Engine
from oracle import oracle
from tests.helpers import ROOT
from tests.test_rdf import CASES, case_dir, golden, load_case, unfold

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "mdff20_b200", "mdff20gpu.x")


@pytest.mark.parametrize("case", CASES)
def test_counts_match_reference(case, tmp_path):
    g = golden(case)
    inp, (resg, cutgr, nbins, nconf), nionit, frames = load_case(case, tmp_path)
    inp.close()
    with rdf.RDF(nionit, cutgr, resg, nbins) as acc:
        for cell, pos in frames:
            acc.add(cell, pos)
        h, n = acc.counts()
    assert n == nconf
    np.testing.assert_array_equal(h, unfold(g["gr"]))


def big_system():
    s = synth.silica(1000, seed=31, rc_sr=7.0, rc_lr=8.0, kmax=6)
    s.cell = s.cell.copy()
    s.cell[1, 0], s.cell[2, 1] = 2.5, -1.5
    rng = np.random.Generator(np.random.PCG64(32))
    base = cellmath.wrap_positions(s.cell, s.pos)
    return s, [base, base + rng.normal(scale=0.2, size=base.shape)]


@pytest.mark.parametrize("resg", [0.1, 0.002])
def test_counts_match_oracle_large(resg):
    """3000 ions, triclinic; resg 0.002 makes ~8900 bins x 4 type pairs, more than the
    shared-memory histogram holds, so the counts go straight to global memory."""
    s, frames = big_system()
    cutgr, nbins = rdf.reference_grid(s.cell, resg)
    want = oracle.gr_counts([(s.cell, f) for f in frames], s.nionit, cutgr, resg, nbins)
    with rdf.RDF(s.nionit, cutgr, resg, nbins) as acc:
        for f in frames:
            acc.add(s.cell, f)
        h, n = acc.counts()
        acc.reset()
        acc.add(s.cell, frames[0])
        h0, n0 = acc.counts()
    assert n == 2 and n0 == 1 and want.sum() > 1e6
    np.testing.assert_array_equal(h, want)
    np.testing.assert_array_equal(h0, oracle.gr_counts([(s.cell, frames[0])], s.nionit, cutgr, resg, nbins))


def test_engine_positions_on_device():
    s, frames = big_system()
    cutgr, nbins = rdf.reference_grid(s.cell)
    e = Engine(s, positions=frames[1])
    with rdf.RDF(s.nionit, cutgr, 0.1, nbins) as a, rdf.RDF(s.nionit, cutgr, 0.1, nbins) as b:
        a.add_engine(e)
        b.add(s.cell, frames[1])
        np.testing.assert_array_equal(a.counts()[0], b.counts()[0])
    e.close()


@pytest.mark.parametrize("case", CASES)
def test_host_program_rdf_mode(case, tmp_path):
    """mdff20gpu.x with lrdf reads TRAJFF and writes RDFFF from the GPU histogram: the
    text write_rdf gives for the reference's counts."""
    g = golden(case)
    inp, (resg, cutgr, nbins, nconf), nionit, frames = load_case(case, tmp_path)
    volume = inp.run.omega
    inp.close()
    p = subprocess.run([EXE, "control.s"], cwd=tmp_path, capture_output=True, timeout=600)
    assert p.returncode == 0, p.stderr.decode()[-2000:]
    assert open(tmp_path / "RDFFF").read() == rdf.rdfff_text(unfold(g["gr"]), nconf, resg, volume, nionit)
    assert os.path.exists(tmp_path / "TRAJFF")   # input, left in place
