"""CPU tests of the radial-distribution pieces: the oracle's get_gr and the C host's
TRAJFF reader, parameters and RDFFF writer, against the reference's own histograms
(tests/golden/rdf/, from the compiled reference's get_gr)."""
import os
import shutil

import numpy as np
import pytest

from mdff20_b200 import host, rdf
from oracle import oracle
from tests.helpers import GOLDEN

RDF_GOLDEN = os.path.join(GOLDEN, "rdf")
CASES = ("pim", "tri")


def case_dir(case, tmp_path):
    """control.s, POSFF and TRAJFF of a case in tmp_path."""
    src = os.path.join(RDF_GOLDEN, case)
    shutil.copy(os.path.join(src, "control.s"), tmp_path / "control.s")
    other = src if case == "tri" else os.path.join(GOLDEN, "host", "pim_nhc")
    for f in ("POSFF", "TRAJFF"):
        shutil.copy(os.path.join(other, f), tmp_path / f)
    return str(tmp_path / "control.s"), str(tmp_path / "POSFF"), str(tmp_path / "TRAJFF")


def golden(case):
    with np.load(os.path.join(RDF_GOLDEN, case, "gr.npz")) as z:
        return {k: z[k] for k in z.files}


def unfold(gr):
    """The reference's gr with its all-pairs tally taken out of [0][0]."""
    u = gr.copy()
    u[:, 0, 0] -= gr.sum(axis=(1, 2)) // 2
    return u


def load_case(case, tmp_path):
    ctl, pos, traj = case_dir(case, tmp_path)
    inp = host.Inputs(ctl, pos)
    resg, cutgr, nbins, nconf = inp.init_rdf(ctl)
    nionit = [inp.run.p.nionit[t] for t in range(inp.run.p.ntype)]
    cell0 = np.array(inp.run.p.cell[:], float).reshape(3, 3)   # POSFF's cell, before the frames
    assert rdf.reference_grid(cell0, resg) == (cutgr, nbins)
    frames = inp.traj_frames(traj, nconf)
    return inp, (resg, cutgr, nbins, nconf), nionit, frames


@pytest.mark.parametrize("case", CASES)
def test_parameters_and_oracle_match_reference(case, tmp_path):
    g = golden(case)
    inp, (resg, cutgr, nbins, nconf), nionit, frames = load_case(case, tmp_path)
    with inp:
        assert (resg, cutgr, nbins, nconf) == (g["resg"][0], g["cutgr"][0], g["nbins"][0], g["nconf"][0])
        h = oracle.gr_counts(frames, nionit, cutgr, resg, nbins)
    assert h.sum() > 0
    np.testing.assert_array_equal(h, unfold(g["gr"]))


@pytest.mark.parametrize("case", CASES)
def test_rdfff_writer(case, tmp_path):
    """The C writer and the Python restatement of write_rdf give the same text, with the
    reference's layout: ntype(ntype+1)/2 (r, g) pairs per line."""
    g = golden(case)
    inp, (resg, cutgr, nbins, nconf), nionit, frames = load_case(case, tmp_path)
    counts = unfold(g["gr"])
    with inp:
        out = str(tmp_path / "RDFFF")
        inp.write_rdf(counts, nconf, out)
        volume = inp.run.omega
    text = open(out).read()
    assert text == rdf.rdfff_text(counts, nconf, resg, volume, nionit)
    lines = text.splitlines()
    assert len(lines) == nbins and len(lines[0].split()) == 2 * 3
    # g(r) proper, and the reference's first column = g_00 plus all pairs over N_0^2
    r, gr = rdf.g_of_r(counts, nconf, resg, volume, nionit)
    b = int(np.argmax(counts[:, 0, 0]))
    all_over_n00 = gr[b, 0, 0] * counts[b].sum() / counts[b, 0, 0]
    assert np.isclose(float(lines[b].split()[1]), gr[b, 0, 0] + all_over_n00, rtol=1e-10)
    assert np.isclose(float(lines[b].split()[0]), r[b])
