"""Regenerates tests/golden/config3.npz and tests/golden/crist192_pim_nhc_aspc4.npz from
the compiled reference.

    make -C oracle ref && python tests/golden/make_config_golden.py [config3|aspc4]

* config3: the 6000-ion polarisable silica single point (mdff20_b200.synth.config3:
  2000 Si + 4000 O at 2.20 g/cm^3, kmax 14, rc 10 A, Buckingham rc 7 A, Tang-Toennies
  damped charge-dipole field, Jacobi SCF to rmsd 1e-8): the reference's lists sizes,
  forces, energies, stress tensors and induced dipoles.  Run with 8 OpenMP threads
  (a single-threaded -O0 run takes tens of minutes); the thread count is stored.
* aspc4: 10 NHC steps of the 192-ion polarisable cristobalite cell with ASPC order 4,
  started at step index 6 so the predictor runs at the full order from the first
  step (the reference's first-steps order switch reads coefficients it never sets
  for ions >= 1, src/pim.c:389-399).

Every number stored is an output of the reference mdff20 C code itself.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mdff20_b200 import synth  # noqa: E402
from oracle import ref  # noqa: E402
from tests.golden import cases  # noqa: E402

THERMO_KEYS = ("u_lj", "u_bhmftd", "u_coul", "u_pol", "pvir_lj", "pvir_bhmftd", "pvir_coul", "tau_lj",
               "tau_bhmftd", "tau_coul")
CONFIG3_THREADS = 8


def config3():
    s = synth.config3()
    e = ref.run(s, "engforce", threads=CONFIG3_THREADS, timeout=7200.0)
    d = {"r_in": e["r_in"], "f": e["f"], "mu_ind": e["mu_ind"], "threads": np.array([CONFIG3_THREADS])}
    d.update({k: e[k] for k in THERMO_KEYS})
    return d


def aspc4():
    s = cases.CASES["crist192_pim_nhc_aspc4"]()
    m = ref.run(s, "md", cases.ASPC4_STEPS, 0, cases.ASPC4_FIRST)
    d = dict(r_in=m["r_in"], vel=s.vel.reshape(-1), md_thermo=m["thermo"], md_r=m["r"], md_v=m["v"],
             md_f=m["f"], xi=m["xi"], vxi=m["vxi"])
    return d


def main(which):
    makers = {"config3": ("config3", config3), "aspc4": ("crist192_pim_nhc_aspc4", aspc4)}
    for key in which or list(makers):
        name, fn = makers[key]
        d = fn()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
