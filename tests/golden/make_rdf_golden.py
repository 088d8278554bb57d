"""Regenerates tests/golden/rdf/: pair histograms of the reference's get_gr.

    make -C oracle ref && python tests/golden/make_rdf_golden.py

The reference's lrdf mode (src/mdff20.c:108-110) cannot write RDFFF here: write_rdf
(src/radial_distribution.c:96-146) indexes its output array with a variable that is
not yet set and the program faults.  The reference harness task "rdf" therefore runs
init_rdf's own steps (default_rdf, read_rdf, alloc_rdf, read_next_traj + get_gr per
TRAJFF configuration) and dumps the integer histogram gr[bin][it][jt], which is what
RDFFF is computed from.

Cases:
  pim  the two TRAJFF frames of tests/golden/host/pim_nhc (192 ions, cubic cell),
       default resg 0.1
  tri  two frames of 96 ions in a triclinic cell written here, resg 0.25 (coarser
       than the default: the reference sizes the histogram with resg 0.1)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mdff20_b200 import cellmath  # noqa: E402
from oracle import ref  # noqa: E402
from tests.golden import cases  # noqa: E402

OUT = os.path.join(HERE, "rdf")
HOST = os.path.join(HERE, "host")


def traj_text(s, frames) -> str:
    """TRAJFF frames in write_config's layout (src/config.c:311-338)."""
    names = np.repeat(np.array(s.type_names, dtype=object), s.nionit)
    out = []
    for pos in frames:
        out.append(f"{s.nion} \n{s.name} \n")
        for i in range(3):
            out.append("".join(f"{v:19.12f} " for v in s.cell[i]) + " \n")
        out.append(f"{s.ntype} \n" + "".join(f"{t} " for t in s.type_names) + "\n")
        out.append("".join(f"{k} " for k in s.nionit) + " \nCartesian \n")
        for i in range(s.nion):
            out.append(f"{names[i]} " + "".join(f"{v:19.12f} " for v in pos[i]) + "".join(
                f"{0.0:19.12f} " for _ in range(6)) + "\n")
    return "".join(out)


def harness_gr(wd):
    exe = ref.harness_path("fix")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run([exe, "control.s", "rdf"], cwd=wd, env=env, capture_output=True, timeout=600)
    if p.returncode != 0:
        raise RuntimeError(p.stderr.decode()[-2000:])
    r = ref.read_records(os.path.join(wd, "out.bin"))
    nb = int(r["nbins"][0])
    return r, nb


def make(name, control_text, posff_src, traj_src_or_text):
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    wd = tempfile.mkdtemp(prefix="mdffrdf_")
    try:
        with open(os.path.join(wd, "control.s"), "w") as fp:
            fp.write(control_text)
        shutil.copy(posff_src, os.path.join(wd, "POSFF"))
        if os.path.exists(traj_src_or_text):
            shutil.copy(traj_src_or_text, os.path.join(wd, "TRAJFF"))
        else:
            with open(os.path.join(wd, "TRAJFF"), "w") as fp:
                fp.write(traj_src_or_text)
            shutil.copy(os.path.join(wd, "TRAJFF"), os.path.join(d, "TRAJFF"))
            shutil.copy(os.path.join(wd, "POSFF"), os.path.join(d, "POSFF"))
        shutil.copy(os.path.join(wd, "control.s"), os.path.join(d, "control.s"))
        r, nb = harness_gr(wd)
        nt = int(round((r["gr"].size / nb) ** 0.5))
        np.savez_compressed(os.path.join(d, "gr.npz"), gr=r["gr"].reshape(nb, nt, nt).astype(np.int64),
                            cutgr=r["cutgr"], resg=r["resg"], nbins=np.array([nb]), nconf=r["nconf"])
        print(name, nb, int(r["gr"].sum()))
    finally:
        shutil.rmtree(wd, ignore_errors=True)


def main():
    ctl = open(os.path.join(HOST, "pim_nhc", "control.s")).read() + "lrdf true\nnconf 2\n"
    make("pim", ctl, os.path.join(HOST, "pim_nhc", "POSFF"), os.path.join(HOST, "pim_nhc", "TRAJFF"))

    s = cases.silica96(False)
    s.cell = s.cell.copy()
    s.cell[1, 0] = 1.2
    s.cell[2, 0] = -0.7
    s.cell[2, 1] = 0.9
    rng = np.random.Generator(np.random.PCG64(21))
    base = cellmath.wrap_positions(s.cell, s.pos)
    frames = [base + rng.normal(scale=0.15, size=base.shape) for _ in range(2)]
    s.pos = base
    wd = tempfile.mkdtemp(prefix="mdffrdf_")
    try:
        s.write(wd)
        ctl = open(os.path.join(wd, "control.s")).read() + "lrdf true\nnconf 2\nresg 0.25\n"
        make("tri", ctl, os.path.join(wd, "POSFF"), traj_text(s, frames))
    finally:
        shutil.rmtree(wd, ignore_errors=True)


if __name__ == "__main__":
    main()
