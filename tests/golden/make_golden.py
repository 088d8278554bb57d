"""Regenerates the golden fixtures in tests/golden/*.npz from the compiled reference.

    make -C oracle ref && python tests/golden/make_golden.py

Every number stored here is an output of the reference mdff20 C code itself (built
unmodified by oracle/Makefile and driven by oracle/ref_harness.c with
OMP_NUM_THREADS=1), on the seeded systems of tests/golden/cases.py.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from tests.golden import cases  # noqa: E402

THERMO_KEYS = ("u_lj", "u_bhmftd", "u_coul", "u_pol", "pvir_lj", "pvir_bhmftd", "pvir_coul", "tau_lj",
               "tau_bhmftd", "tau_coul")


def main():
    out = {}
    # LJ: lists, forces, 50 NVE steps
    s = cases.CASES["lj256"]()
    r = ref.run(s, "list")
    out["lj256"] = dict(r_in=r["r_in"], nb_point=r["nb_point"], nb_list=r["nb_list"], coul_point=r["coul_point"],
                        coul_list=r["coul_list"], vel=s.vel.reshape(-1))
    e = ref.run(s, "engforce")
    out["lj256"].update({"f": e["f"], **{k: e[k] for k in THERMO_KEYS}})
    m = ref.run(s, "md", 50, 0)
    out["lj256"].update(md_thermo=m["thermo"], md_r=m["r"], md_v=m["v"], md_f=m["f"])

    for name in ("silica96_rigid", "silica96_pim", "silica450_pim", "silica96_ko"):
        s = cases.CASES[name]()
        r = ref.run(s, "list")
        d = dict(r_in=r["r_in"], nb_point=r["nb_point"], nb_list=r["nb_list"], coul_point=r["coul_point"],
                 coul_list=r["coul_list"])
        e = ref.run(s, "engforce")
        d.update({"f": e["f"], **{k: e[k] for k in THERMO_KEYS}})
        if "mu_ind" in e:
            d["mu_ind"] = e["mu_ind"]
        if name == "silica96_rigid":
            q, mu = cases.es_inputs(s)
            for k, fl in enumerate(cases.ES_FLAG_SETS):
                rr = ref.run(s, "ewald", *fl, extra_files={"in_q.bin": q, "in_mu.bin": mu})
                for key in ("u", "pvir", "tau", "ef", "efg", "f"):
                    d[f"es{k}_{key}"] = rr[key]
        out[name] = d

    for name, nsteps in cases.MD_CASES[1:]:
        s = cases.CASES[name]()
        m = ref.run(s, "md", nsteps, 0)
        d = dict(r_in=m["r_in"], vel=s.vel.reshape(-1), md_thermo=m["thermo"], md_r=m["r"], md_v=m["v"],
                 md_f=m["f"])
        if "xi" in m:
            d.update(xi=m["xi"], vxi=m["vxi"])
        out[name] = d

    for name, d in out.items():
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
