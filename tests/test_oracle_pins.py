"""The oracle (C restatement in oracle/) pinned against the reference itself.

* golden fixtures: outputs of the compiled reference stored in tests/golden (always run);
* live compiled reference (oracle/_ref), when it has been built on this machine;
* the reference's only stored known answers, examples/ex2 (Lennard-Jones cluster
  energies), read from the reference checkout when it is present.
"""
import os

import numpy as np
import pytest

from tests.helpers import load_golden, rel_err
from oracle import ref
from oracle.oracle import Oracle
from tests.golden import cases

# the reference checkout: $MDFF20_REFERENCE, else a sibling directory of this repository
REFERENCE_SRC = os.environ.get("MDFF20_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(
    os.path.dirname(os.path.abspath(__file__)))), "reference"))


def _oracle_for(name, wrap_from_golden=True):
    g = load_golden(name)
    s = cases.CASES[name]()
    if "vel" in g:
        s.vel = g["vel"].reshape(-1, 3)
    s.pos = g["r_in"].reshape(-1, 3)
    return Oracle(s, wrap=False), g, s


@pytest.mark.parametrize("name", ["lj256", "silica96_rigid", "silica96_pim", "silica450_pim", "silica96_ko"])
def test_lists_bit_exact(name):
    o, g, s = _oracle_for(name)
    o.gen_verletlist()
    for which, key in ((0, "nb"), (1, "coul")):
        p, lst = o.verletlist(which)
        assert np.array_equal(p, g[f"{key}_point"])
        assert np.array_equal(lst, g[f"{key}_list"])


@pytest.mark.parametrize("name", ["lj256", "silica96_rigid", "silica96_pim", "silica450_pim", "silica96_ko"])
def test_engforce_vs_reference(name):
    o, g, s = _oracle_for(name)
    o.gen_verletlist()
    o.engforce()
    th = o.thermo()
    f = o.forces()
    # force scale: the fcc LJ lattice has (near) zero forces, so compare absolutely there
    if name == "lj256":
        assert np.abs(f - g["f"].reshape(-1, 3)).max() < 1e-12
    else:
        assert rel_err(f, g["f"].reshape(-1, 3)) < 1e-12
    for k in ("u_lj", "u_bhmftd", "u_coul", "u_pol", "pvir_lj", "pvir_bhmftd", "pvir_coul"):
        assert abs(th[k] - float(g[k][0])) <= 1e-12 * max(1.0, abs(float(g[k][0]))), k
    for k in ("tau_lj", "tau_bhmftd", "tau_coul"):
        assert np.abs(th[k].ravel() - g[k]).max() < 1e-10, k
    if "mu_ind" in g:
        assert rel_err(o.dipoles(), g["mu_ind"].reshape(-1, 3)) < 1e-11


def test_multipole_es_flags_vs_reference():
    o, g, s = _oracle_for("silica96_rigid")
    o.gen_verletlist()
    q, mu = cases.es_inputs(s)
    for k, fl in enumerate(cases.ES_FLAG_SETS):
        out = o.multipole_es(q, mu, **dict(zip(cases.ES_FLAG_NAMES, fl)))
        assert abs(out["u"] - g[f"es{k}_u"][0]) < 1e-9, fl
        assert rel_err(out["ef"], g[f"es{k}_ef"].reshape(-1, 3)) < 1e-12, fl
        assert rel_err(out["efg"].reshape(-1, 9), g[f"es{k}_efg"].reshape(-1, 9)) < 1e-12, fl
        if fl[3]:
            assert rel_err(out["f"], g[f"es{k}_f"].reshape(-1, 3)) < 1e-12, fl
        assert np.abs(out["tau"].ravel() - g[f"es{k}_tau"]).max() < 1e-10, fl


@pytest.mark.parametrize("name,nsteps", list(cases.MD_CASES))
def test_md_vs_reference(name, nsteps):
    o, g, s = _oracle_for(name)
    th = o.md(nsteps)
    ref_th = g["md_thermo"].reshape(-1, 12)
    # e_kin, u_*, e_nvt track the reference step by step; the reference perturbs its
    # positions by the kardir/dirkar round trips, so allow trajectory drift
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(ref_th[:, col]).max()))
        assert np.abs(th[:, col] - ref_th[:, col]).max() < 1e-7 * scale, col
    assert th[-1, 9] == ref_th[-1, 9]  # same number of list rebuilds
    pos, vel, f = o.state()
    assert rel_err(vel, g["md_v"].reshape(-1, 3)) < 1e-7


def test_md_aspc_order4_vs_reference():
    """ASPC order 4 (the config-5 setting): NHC steps from step index 6, where the
    predictor runs at the full order from the first step."""
    o, g, s = _oracle_for("crist192_pim_nhc_aspc4")
    th = o.md(cases.ASPC4_STEPS, first=cases.ASPC4_FIRST)
    ref_th = g["md_thermo"].reshape(-1, 12)
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(ref_th[:, col]).max()))
        assert np.abs(th[:, col] - ref_th[:, col]).max() < 1e-9 * scale, col
    pos, vel, f = o.state()
    assert rel_err(vel, g["md_v"].reshape(-1, 3)) < 1e-9
    assert rel_err(f, g["md_f"].reshape(-1, 3)) < 1e-9
    xi, vxi = o.nhc()
    assert np.allclose(xi, g["xi"], rtol=1e-8, atol=1e-14)


@pytest.mark.skipif(not ref.available("fix"), reason="compiled reference not built (make -C oracle ref)")
def test_live_reference_random_seed():
    """A fresh random rigid-ion system through both the oracle and the reference."""
    from mdff20_b200 import synth
    s = synth.silica(40, seed=101, polarizable=True, rc_sr=4.5, rc_lr=5.5, skin=0.3, kmax=4, alpha=0.7,
                     conv_tol=1e-10, dmin=synth.PIM_DMIN)
    r = ref.run(s, "engforce")
    s.pos = r["r_in"].reshape(-1, 3)
    o = Oracle(s, wrap=False)
    o.gen_verletlist()
    o.engforce()
    assert rel_err(o.forces(), r["f"].reshape(-1, 3)) < 1e-12
    assert rel_err(o.dipoles(), r["mu_ind"].reshape(-1, 3)) < 1e-11


def _ex2_cases():
    cfg = os.path.join(REFERENCE_SRC, "examples", "ex2", "config")
    if not os.path.isdir(cfg):
        return []
    return [n for n in (3, 13, 38, 55, 100, 147) if os.path.exists(os.path.join(cfg, str(n)))]


@pytest.mark.skipif(not _ex2_cases(), reason="reference examples/ex2 not present on this machine")
@pytest.mark.parametrize("nat", _ex2_cases() or [0])
def test_ex2_lj_cluster_known_answers(nat):
    """examples/ex2 (run_ex2.sh:12-34): static LJ energy of a cluster in a 100 A box with
    cutoff 100 and linear truncation, against the stored REFERENCE energies.  The values
    are read from the reference checkout at test time, not copied here."""
    from mdff20_b200.system import System
    cfg = os.path.join(REFERENCE_SRC, "examples", "ex2", "config")
    pos = np.loadtxt(os.path.join(cfg, str(nat)))
    refE = None
    with open(os.path.join(cfg, "REFERENCE")) as fp:
        for line in fp:
            t = line.split()
            if len(t) >= 2 and t[0] == str(nat):
                refE = float(t[1])
    assert refE is not None
    one = np.ones((1, 1))
    s = System(cell=np.eye(3) * 100.0, type_names=["A"], nionit=[nat], pos=pos, mass=[1.0], lnmlj=True,
               trunc="linear", sigmalj=one, epslj=one, plj=one * 6, qlj=one * 12, cutshortrange=100.0,
               cutlongrange=100.0, lstatic=True)
    o = Oracle(s)
    o.gen_verletlist()
    o.engforce()
    assert abs(o.thermo()["u_lj"] - refE) < 1e-6
