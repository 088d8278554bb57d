"""CUDA engine (libmdffgpu, FP64 path) against the reference's golden outputs and the
oracle restatement.  Everything goes through the C ABI (mdff20_b200.engine).

Tolerances (FP64 arithmetic, different summation order and k-space phase
factorisation): forces and fields 1e-11 relative to the largest component, energies
1e-11 relative, stress 1e-9 GPa absolute; neighbour lists exactly equal.
"""
import numpy as np
import pytest

from mdff20_b200 import synth
from mdff20_b200.engine import PIM_CG, PIM_CG_FUSED, Engine, MdffgpuError
from oracle.oracle import Oracle, wrapped_positions
from tests.golden import cases
from tests.helpers import load_golden, rel_err, rms_rel, tensor_rel

pytestmark = pytest.mark.gpu

SINGLE = ["lj256", "silica96_rigid", "silica96_pim", "silica450_pim", "silica96_ko"]


def _engine_for(name, **kw):
    g = load_golden(name)
    s = cases.CASES[name]()
    if "vel" in g:
        s.vel = g["vel"].reshape(-1, 3)
    pos = g["r_in"].reshape(-1, 3)
    s.pos = pos
    return Engine(s, positions=pos, **kw), g, s


@pytest.mark.parametrize("name", SINGLE)
def test_verlet_lists_bit_exact(name):
    e, g, s = _engine_for(name)
    e.gen_verletlist()
    for which, key in ((0, "nb"), (1, "coul")):
        p, lst = e.verletlist(which)
        assert np.array_equal(p, g[f"{key}_point"]), key
        assert np.array_equal(lst, g[f"{key}_list"]), key


@pytest.mark.parametrize("name", SINGLE)
def test_engforce_vs_reference(name):
    e, g, s = _engine_for(name)
    e.gen_verletlist()
    e.engforce()
    th = e.thermo()
    f = e.forces()
    if name == "lj256":  # perfect lattice: forces vanish, compare absolutely
        assert np.abs(f - g["f"].reshape(-1, 3)).max() < 1e-11
    else:
        assert rel_err(f, g["f"].reshape(-1, 3)) < 1e-11
    for k in ("u_lj", "u_bhmftd", "u_coul", "u_pol", "pvir_lj", "pvir_bhmftd", "pvir_coul"):
        ref = float(g[k][0])
        assert abs(th[k] - ref) <= 1e-11 * max(1.0, abs(ref)), (k, th[k], ref)
    for k in ("tau_lj", "tau_bhmftd", "tau_coul"):
        assert np.abs(th[k].ravel() - g[k]).max() < 1e-9, k
    if "mu_ind" in g:
        mu = e.dipole_history()[:, 0, :]
        assert rel_err(mu, g["mu_ind"].reshape(-1, 3)) < 1e-10
        assert th["scf_iter"] > 0


def test_multipole_es_flags_vs_reference():
    e, g, s = _engine_for("silica96_rigid")
    e.gen_verletlist()
    q, mu = cases.es_inputs(s)
    for k, fl in enumerate(cases.ES_FLAG_SETS):
        out = e.multipole_es(q, mu, **dict(zip(cases.ES_FLAG_NAMES, fl)))
        assert abs(out["u"] - g[f"es{k}_u"][0]) < 1e-9, fl
        assert rel_err(out["ef"], g[f"es{k}_ef"].reshape(-1, 3)) < 1e-11, fl
        assert rel_err(out["efg"].reshape(-1, 9), g[f"es{k}_efg"].reshape(-1, 9)) < 1e-11, fl
        if fl[3]:
            assert rel_err(out["f"], g[f"es{k}_f"].reshape(-1, 3)) < 1e-11, fl
        assert np.abs(out["tau"].ravel() - g[f"es{k}_tau"]).max() < 1e-9, fl


@pytest.mark.parametrize("name,nsteps", list(cases.MD_CASES))
def test_md_vs_reference(name, nsteps):
    e, g, s = _engine_for(name)
    e.gen_verletlist()
    e.engforce()
    th = e.md_steps(1, nsteps)
    ref_th = g["md_thermo"].reshape(-1, 12)[1:]
    for col in (0, 1, 2, 3, 4, 5):
        scale = max(1.0, float(np.abs(ref_th[:, col]).max()))
        assert np.abs(th[:, col] - ref_th[:, col]).max() < 1e-7 * scale, col
    assert th[-1, 9] == ref_th[-1, 9]
    pos, vel, f = e.state()
    assert rel_err(vel, g["md_v"].reshape(-1, 3)) < 1e-7
    if "xi" in g:
        xi, vxi = e.nhc()
        assert np.allclose(xi, g["xi"], rtol=1e-6, atol=1e-12)


def test_lverletL_false_matches_listed():
    """lverletL false: the reference scans every pair each call (src/nmlj.c:297-300)."""
    s = cases.silica96(True)
    pos = wrapped_positions(s)
    a = Engine(s, positions=pos)
    a.gen_verletlist()
    a.engforce()
    s2 = cases.silica96(True)
    s2.lverletL = False
    b = Engine(s2, positions=pos)
    b.engforce()
    o = Oracle(s2)
    o.engforce()
    assert rel_err(b.forces(), a.forces()) < 1e-11
    assert rel_err(b.forces(), o.forces()) < 1e-11


def test_cg_solver_converges_to_reference_fixed_point():
    g = load_golden("silica450_pim")
    s = cases.CASES["silica450_pim"]()
    pos = g["r_in"].reshape(-1, 3)
    e = Engine(s, positions=pos, pim_solver=PIM_CG)
    e.gen_verletlist()
    e.engforce()
    th = e.thermo()
    assert th["scf_iter"] < 26  # fewer matrix-vector products than the Jacobi iteration
    assert th["scf_rmsd"] <= s.conv_tol_ind
    # at conv_tol_ind = 1e-10 the two fixed points agree to ~1e-10 in the dipoles
    assert rel_err(e.dipole_history()[:, 0, :], g["mu_ind"].reshape(-1, 3)) < 1e-8
    assert rel_err(e.forces(), g["f"].reshape(-1, 3)) < 1e-9
    assert abs(th["u_coul"] - float(g["u_coul"][0])) < 1e-8 * abs(float(g["u_coul"][0]))


def test_fused_cg_matches_cg():
    """PIM_CG_FUSED (one Ewald pass for E_stat + T mu0, rho(k) carried along the CG
    iterates for the force pass) is the same CG: reference fixed point, and over MD
    steps the same trajectory as PIM_CG to rounding."""
    g = load_golden("silica450_pim")
    s = cases.CASES["silica450_pim"]()
    pos = g["r_in"].reshape(-1, 3)
    e = Engine(s, positions=pos, pim_solver=PIM_CG_FUSED)
    e.gen_verletlist()
    e.engforce()
    th = e.thermo()
    assert th["scf_rmsd"] <= s.conv_tol_ind
    assert rel_err(e.forces(), g["f"].reshape(-1, 3)) < 1e-9
    assert abs(th["u_coul"] - float(g["u_coul"][0])) < 1e-8 * abs(float(g["u_coul"][0]))
    assert abs(th["u_pol"] - float(g["u_pol"][0])) < 1e-8 * abs(float(g["u_pol"][0]))
    g2 = load_golden("crist192_pim_nhc")
    s2 = cases.CASES["crist192_pim_nhc"]()
    s2.vel = g2["vel"].reshape(-1, 3)
    p2 = g2["r_in"].reshape(-1, 3)
    a = Engine(s2, positions=p2, pim_solver=PIM_CG)
    b = Engine(s2, positions=p2, pim_solver=PIM_CG_FUSED)
    for x in (a, b):
        x.gen_verletlist()
        x.engforce()
    ta, tb = a.md_steps(1, 8), b.md_steps(1, 8)
    # both stop at the SCF tolerance (1e-9): agreement to well below it
    assert np.allclose(ta, tb, rtol=1e-8, atol=1e-8)
    assert rel_err(b.forces(), a.forces()) < 1e-8
    assert rel_err(b.state()[0], a.state()[0]) < 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_steps_match_eager(precision):
    """MD steps replayed as CUDA graphs (device-side CG loop) give exactly the results of
    the kernel-by-kernel steps, in both precisions."""
    g = load_golden("crist192_pim_nhc")
    s = cases.CASES["crist192_pim_nhc"]()
    s.vel = g["vel"].reshape(-1, 3)
    p0 = g["r_in"].reshape(-1, 3)
    runs = []
    for graph in (False, True):
        e = Engine(s, positions=p0, pim_solver=PIM_CG_FUSED, precision=precision)
        e.set_graph(graph)
        e.gen_verletlist()
        e.engforce()
        l0 = e.launch_count()
        th = e.md_steps(1, 12)
        runs.append((th, e.state(), e.launch_count() - l0))
        e.close()
    (ta, sa, la), (tb, sb, lb) = runs
    assert np.array_equal(ta, tb)
    for a, b in zip(sa, sb):
        assert np.array_equal(a, b)
    # the graph counts what it replays: the device-side CG tests (one per iteration and
    # one before) and the search-direction update after the last iteration come on top;
    # the list rebuild is an IF node whose five kernels launch only on rebuild steps,
    # where kernel-by-kernel steps launch them every step (they return at once)
    assert la - 12 * 5 <= lb <= la + 12 * 16 and lb != la


def test_graph_scf_nonconvergence_reported():
    """A CG iteration cap that cannot be met is reported as ERR_SCF from a graph step."""
    g = load_golden("crist192_pim_nhc")
    s = cases.CASES["crist192_pim_nhc"]()
    s.vel = g["vel"].reshape(-1, 3)
    s.max_scf_pim_iter = 1
    s.conv_tol_ind = 1e-14
    e = Engine(s, positions=g["r_in"].reshape(-1, 3), pim_solver=PIM_CG_FUSED)
    e.gen_verletlist()
    with pytest.raises(MdffgpuError) as ex:
        e.md_steps(1, 3)
    assert ex.value.code == 4   # MDFFGPU_ERR_SCF


def test_random_systems_vs_oracle():
    """Fresh seeds (not in the fixtures), engine vs oracle, several flag paths."""
    for seed in (201, 202):
        s = synth.silica(48, seed=seed, polarizable=True, rc_sr=4.8, rc_lr=5.6, skin=0.4, kmax=5, alpha=0.62,
                         conv_tol=1e-11, dmin=synth.PIM_DMIN)
        pos = wrapped_positions(s)
        o = Oracle(s)
        o.gen_verletlist()
        o.engforce()
        e = Engine(s, positions=pos)
        e.gen_verletlist()
        e.engforce()
        assert rel_err(e.forces(), o.forces()) < 1e-10
        a, b = e.thermo(), o.thermo()
        for k in ("u_bhmftd", "u_coul", "u_pol"):
            assert abs(a[k] - b[k]) < 1e-10 * max(1.0, abs(b[k]))


def test_config2_single_point_vs_oracle():
    """Full-size rigid-ion silica (N=3000, kmax 12, rc 10 A) against the oracle."""
    s = synth.config2()
    pos = wrapped_positions(s)
    o = Oracle(s)
    o.gen_verletlist()
    o.engforce()
    e = Engine(s, positions=pos)
    e.gen_verletlist()
    for which in (0, 1):
        p1, l1 = o.verletlist(which)
        p2, l2 = e.verletlist(which)
        assert np.array_equal(p1, p2) and np.array_equal(l1, l2)
    e.engforce()
    assert rel_err(e.forces(), o.forces()) < 1e-11
    a, b = e.thermo(), o.thermo()
    for k in ("u_bhmftd", "u_coul", "pvir_coul"):
        assert abs(a[k] - b[k]) < 1e-11 * max(1.0, abs(b[k])), k


def test_deterministic_and_newton3_full_size():
    """N=24000 PIM silica: two evaluations are bit-identical; sum of forces ~ 0."""
    s = synth.config5()
    pos = wrapped_positions(s)
    e = Engine(s, positions=pos, pim_solver=PIM_CG)
    e.gen_verletlist()
    e.engforce()
    f1 = e.forces().copy()
    e2 = Engine(s, positions=pos, pim_solver=PIM_CG)
    e2.gen_verletlist()
    e2.engforce()
    assert np.array_equal(f1, e2.forces())
    # real-space pair forces are antisymmetric; k-space forces sum to ~0 for a neutral cell
    assert np.abs(f1.sum(axis=0)).max() < 1e-6 * np.abs(f1).max() * np.sqrt(s.nion)


def test_error_paths():
    s = cases.silica96(True)
    pos = wrapped_positions(s)
    e = Engine(s, positions=pos)
    with pytest.raises(MdffgpuError) as ex:
        e.engforce()                        # no Verlet list yet
    assert ex.value.code == 6
    e.gen_verletlist()
    bad = pos.copy()
    bad[3, 0] = np.nan
    e.set_positions(bad)
    with pytest.raises(MdffgpuError) as ex:
        e.engforce()
    assert ex.value.code in (5,)
    s2 = cases.silica96(True, conv_tol=1e-14)
    s2.max_scf_pim_iter = 2
    c = Engine(s2, positions=pos, pim_solver=PIM_CG)
    c.gen_verletlist()
    with pytest.raises(MdffgpuError) as ex:
        c.engforce()
    assert ex.value.code == 4


def test_list_capacity_grows():
    """A compressed box overflows the initial list capacity; the engine grows it and
    still returns the reference pair set."""
    s = cases.silica96(False)
    pos = wrapped_positions(s)
    e = Engine(s, positions=pos)
    e.gen_verletlist()
    o = Oracle(s)
    o.gen_verletlist()
    dense = pos * 0.6   # squeeze every ion into 22% of the volume
    e.set_positions(dense)
    e.gen_verletlist()
    o.set_positions(dense)
    o.gen_verletlist()
    for which in (0, 1):
        p1, l1 = o.verletlist(which)
        p2, l2 = e.verletlist(which)
        assert np.array_equal(p1, p2) and np.array_equal(l1, l2)


# ---------------------------------------------------------------------------- mixed precision
# Mixed FP32/FP64 bars (relative): forces and induced dipoles 1e-5 RMS over ions, energies
# and virials 1e-5, stress tensors 1e-5 of their largest component.
_rms_rel = rms_rel


@pytest.mark.parametrize("name", ["silica450_pim", "silica96_rigid", "silica96_pim"])
def test_mixed_precision_errors_small(name):
    """Mixed FP32/FP64 forces, induced dipoles, energies and stress against the
    reference's FP64 results."""
    from mdff20_b200.engine import MIXED
    e, g, s = _engine_for(name, precision=MIXED)
    e.gen_verletlist()
    e.engforce()
    fr = g["f"].reshape(-1, 3)
    assert _rms_rel(e.forces(), fr) < 1e-5
    th = e.thermo()
    assert abs(th["u_coul"] - float(g["u_coul"][0])) < 1e-6 * abs(float(g["u_coul"][0]))
    for k in ("u_bhmftd", "u_pol", "pvir_coul", "pvir_bhmftd"):
        ref = float(g[k][0])
        assert abs(th[k] - ref) <= 1e-5 * max(abs(ref), 1e-12), k
    for k in ("tau_coul", "tau_bhmftd"):
        assert tensor_rel(th[k], g[k]) < 1e-5, k
    if "mu_ind" in g:
        assert _rms_rel(e.dipole_history()[:, 0, :], g["mu_ind"].reshape(-1, 3)) < 1e-5


def test_mixed_precision_force_error_full_size():
    """N=24000 PIM silica (the bench system): mixed with the fused CG (the bench's
    mixed configuration) vs the FP64 engine with the plain CG."""
    from mdff20_b200.engine import MIXED
    s = synth.config5()
    pos = wrapped_positions(s)
    ref = Engine(s, positions=pos, pim_solver=PIM_CG)
    ref.gen_verletlist()
    ref.engforce()
    mix = Engine(s, positions=pos, pim_solver=PIM_CG_FUSED, precision=MIXED)
    mix.gen_verletlist()
    mix.engforce()
    err = _rms_rel(mix.forces(), ref.forces())
    assert err < 1e-5, err
    a, b = mix.thermo(), ref.thermo()
    # energies: same 1e-5 relative bar as the forces (u_pol carries the SCF
    # convergence tolerance on top of the FP32 field error)
    for k in ("u_coul", "u_pol", "u_bhmftd", "pvir_coul", "pvir_bhmftd"):
        assert abs(a[k] - b[k]) < 1e-5 * max(1.0, abs(b[k])), k
    for k in ("tau_coul", "tau_bhmftd"):
        assert tensor_rel(a[k], b[k]) < 1e-5, k
    # the induced dipoles of this near-crystalline system are small (u_pol 42 eV over 16000
    # O), so their difference is set by the SCF tolerance both solvers stop at (residual
    # rmsd 1e-6, alpha_O = 1): RMS |d mu| over the polarisable ions within 5 x tol x alpha
    pol = s.nionit[0]
    dmu = mix.dipole_history()[:pol, 0, :] - ref.dipole_history()[:pol, 0, :]
    mu_err = float(np.sqrt(np.mean(np.sum(dmu ** 2, 1))))
    assert mu_err < 5.0 * s.conv_tol_ind * 1.0, mu_err
    th = mix.md_steps(1, 3)
    assert np.isfinite(th).all()
