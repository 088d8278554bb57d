"""The named benchmark systems at full size, through the C ABI, against the reference.

* config 3 (6000-ion polarisable silica single point, kmax 14, SCF to 1e-8) against the
  compiled reference's own outputs (tests/golden/config3.npz, make_config_golden.py):
  FP64 with the reference's Jacobi solver and with CG, and the mixed FP32/FP64 path;
* config 5 (24000 ions, the MD bench system) in FP64 against the compiled reference
  run on all host cores;
* ASPC order 4 (config 5's predictor order) over NHC steps against the reference.

Tolerances, stated per quantity (relative measures of tests/helpers.py):

| path                          | forces       | dipoles      | energies | stress       |
|-------------------------------|--------------|--------------|----------|--------------|
| FP64, same Jacobi iterations  | 1e-10 max    | 1e-10 max    | 1e-10    | 1e-10 tensor |
| FP64 CG (stops elsewhere
  inside the 1e-8 SCF tolerance) | 1e-8 max     | 1e-7 max     | 1e-9 (u_pol,
                                                                 first order in
                                                                 the dipoles: 1e-7) | 1e-8 tensor  |
| mixed, CG to 1e-6 (config 3's
  mixed tolerance)               | 1e-5 RMS     | 1e-5 RMS     | 1e-5     | 1e-5 tensor  |
"""
import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.engine import MIXED, PIM_CG, PIM_CG_FUSED, PIM_REFERENCE, Engine
from oracle.oracle import Oracle, wrapped_positions
from tests.golden import cases
from tests.helpers import load_golden, rel_err, rms_rel, tensor_rel

pytestmark = pytest.mark.gpu

ENERGIES = ("u_bhmftd", "u_coul", "u_pol")
VIRIALS = ("pvir_bhmftd", "pvir_coul")
STRESS = ("tau_bhmftd", "tau_coul")


def _config3(conv_tol=None):
    g = load_golden("config3")
    s = synth.config3()
    s.pos = g["r_in"].reshape(-1, 3)
    if conv_tol is not None:
        s.conv_tol_ind = conv_tol
    return s, g


def _errors(e, g):
    """Every result of a single point against the reference's: forces, dipoles,
    energies, virials, stress."""
    th = e.thermo()
    f = e.forces()
    mu = e.dipole_history()[:, 0, :]
    fr, mr = g["f"].reshape(-1, 3), g["mu_ind"].reshape(-1, 3)
    out = dict(f_max=rel_err(f, fr), f_rms=rms_rel(f, fr), mu_max=rel_err(mu, mr), mu_rms=rms_rel(mu, mr))
    for k in ENERGIES + VIRIALS:
        ref = float(g[k][0])
        out[k] = abs(th[k] - ref) / abs(ref)
    for k in STRESS:
        out[k] = tensor_rel(th[k], g[k])
    out["scf_iter"] = th["scf_iter"]
    out["scf_rmsd"] = th["scf_rmsd"]
    return out


def test_config3_lists_vs_oracle():
    s, g = _config3()
    o = Oracle(s, wrap=False)
    o.gen_verletlist()
    e = Engine(s, positions=s.pos)
    e.gen_verletlist()
    for which in (0, 1):
        p1, l1 = o.verletlist(which)
        p2, l2 = e.verletlist(which)
        assert np.array_equal(p1, p2) and np.array_equal(l1, l2), which


def test_config3_fp64_reference_solver():
    """FP64 with the reference's own solver (Jacobi, src/pim.c:236-278): the same
    iterations, so every result to 1e-10."""
    s, g = _config3()
    e = Engine(s, positions=s.pos, pim_solver=PIM_REFERENCE)
    e.gen_verletlist()
    e.engforce()
    err = _errors(e, g)
    for k, v in err.items():
        if k not in ("scf_iter", "scf_rmsd"):
            assert v < 1e-10, (k, err)
    assert err["scf_rmsd"] <= s.conv_tol_ind


@pytest.mark.parametrize("solver", [PIM_CG, PIM_CG_FUSED])
def test_config3_fp64_cg(solver):
    """FP64 CG: the reference's fixed point within the 1e-8 SCF tolerance."""
    s, g = _config3()
    e = Engine(s, positions=s.pos, pim_solver=solver)
    e.gen_verletlist()
    e.engforce()
    err = _errors(e, g)
    assert err["scf_rmsd"] <= s.conv_tol_ind
    assert err["f_max"] < 1e-8, err
    assert err["mu_max"] < 1e-7, err
    for k in ENERGIES + VIRIALS:
        assert err[k] < (1e-7 if k == "u_pol" else 1e-9), (k, err)
    for k in STRESS:
        assert err[k] < 1e-8, (k, err)


def test_config3_mixed():
    """Mixed FP32/FP64 with the fused CG to config 3's mixed tolerance (1e-6) against
    the reference's FP64 results at 1e-8: forces, induced dipoles, energies, virials and
    stress each within 1e-5."""
    s, g = _config3(conv_tol=1e-6)
    e = Engine(s, positions=s.pos, pim_solver=PIM_CG_FUSED, precision=MIXED)
    e.gen_verletlist()
    e.engforce()
    err = _errors(e, g)
    assert err["f_rms"] < 1e-5, err
    assert err["mu_rms"] < 1e-5, err
    for k in ENERGIES + VIRIALS + STRESS:
        assert err[k] < 1e-5, (k, err)


def test_config5_fp64_vs_reference():
    """N = 24000 (the MD bench system), FP64 with the reference's Jacobi solver against
    the compiled reference itself (-O3 build, all host cores; the oracle restatement,
    threaded, where the reference is not built): lists bit-exact, every result of the
    single point."""
    import os

    from oracle import ref
    s = synth.config5()
    if ref.available("tim") and ref.available("fix"):
        threads = os.cpu_count() or 1
        lists = ref.run(s, "list", variant="fix", threads=threads, timeout=1800)
        r = ref.run(s, "engforce", variant="tim", threads=threads, timeout=1800)
        pos = r["r_in"].reshape(-1, 3)
        want_lists = [(lists["nb_point"], lists["nb_list"]), (lists["coul_point"], lists["coul_list"])]
        want_f, want_mu = r["f"].reshape(-1, 3), r["mu_ind"].reshape(-1, 3)
        want = {k: (float(r[k][0]) if r[k].size == 1 else r[k]) for k in ENERGIES + VIRIALS + STRESS}
    else:
        pos = wrapped_positions(s)
        o = Oracle(s)
        o.gen_verletlist()
        want_lists = [o.verletlist(0), o.verletlist(1)]
        o.engforce()
        want_f, want_mu = o.forces(), o.dipoles()
        want = o.thermo()
    e = Engine(s, positions=pos, pim_solver=PIM_REFERENCE)
    e.gen_verletlist()
    for which in (0, 1):
        p2, l2 = e.verletlist(which)
        assert np.array_equal(want_lists[which][0], p2) and np.array_equal(want_lists[which][1], l2), which
    e.engforce()
    assert rel_err(e.forces(), want_f) < 1e-10
    assert rel_err(e.dipole_history()[:, 0, :], want_mu) < 1e-10
    a = e.thermo()
    for k in ENERGIES + VIRIALS:
        assert abs(a[k] - want[k]) < 1e-10 * abs(want[k]), k
    for k in STRESS:
        assert tensor_rel(a[k], want[k]) < 1e-10, k


def test_md_aspc_order4_vs_reference():
    """ASPC order 4 with the reference's Jacobi solver, NHC steps from step index 6,
    step by step against the reference."""
    g = load_golden("crist192_pim_nhc_aspc4")
    s = cases.CASES["crist192_pim_nhc_aspc4"]()
    s.vel = g["vel"].reshape(-1, 3)
    pos = g["r_in"].reshape(-1, 3)
    e = Engine(s, positions=pos, pim_solver=PIM_REFERENCE)
    e.gen_verletlist()
    e.engforce()
    th = e.md_steps(cases.ASPC4_FIRST, cases.ASPC4_STEPS)
    ref_th = g["md_thermo"].reshape(-1, 12)[1:]
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(ref_th[:, col]).max()))
        assert np.abs(th[:, col] - ref_th[:, col]).max() < 1e-9 * scale, col
    _, vel, f = e.state()
    assert rel_err(vel, g["md_v"].reshape(-1, 3)) < 1e-9
    assert rel_err(f, g["md_f"].reshape(-1, 3)) < 1e-9
    xi, vxi = e.nhc()
    assert np.allclose(xi, g["xi"], rtol=1e-8, atol=1e-14)


@pytest.mark.parametrize("precision", [0, MIXED])
def test_md_aspc_order4_cg(precision):
    """The bench's solver (fused CG, polynomial predictor through the last five
    converged dipoles) on the same ASPC-order-4 run: the reference's trajectory within
    the SCF tolerance (FP64) or the mixed force bar."""
    g = load_golden("crist192_pim_nhc_aspc4")
    s = cases.CASES["crist192_pim_nhc_aspc4"]()
    s.vel = g["vel"].reshape(-1, 3)
    e = Engine(s, positions=g["r_in"].reshape(-1, 3), pim_solver=PIM_CG_FUSED, precision=precision)
    e.gen_verletlist()
    e.engforce()
    th = e.md_steps(cases.ASPC4_FIRST, cases.ASPC4_STEPS)
    ref_th = g["md_thermo"].reshape(-1, 12)[1:]
    tol = 1e-8 if precision == 0 else 1e-5
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(ref_th[:, col]).max()))
        assert np.abs(th[:, col] - ref_th[:, col]).max() < tol * scale, col
    assert rms_rel(e.forces(), g["md_f"].reshape(-1, 3)) < tol
