"""Batched force matching, host side: the Ewald autotuner, the seeded configuration
set, parameter plumbing, the sharding of configurations over ranks (2 gloo ranks on
CPU) and the oracle's loss against the reference's (tests/golden/fit96.npz)."""
import math
import os

import numpy as np
import pytest

from mdff20_b200 import fit
from tests.helpers import load_golden


@pytest.mark.parametrize("n", [96, 480, 1536])
def test_ewald_tune_meets_accuracy(n):
    L = (n / fit.NUMBER_DENSITY) ** (1.0 / 3.0)
    ch = fit.ewald_tune(L, n, eps=1e-6)
    assert math.erfc(ch.alpha * ch.rc) <= 1.0001e-6                       # real-space truncation
    assert math.exp(-(math.pi * ch.kmax / (ch.alpha * L)) ** 2) <= 1e-6   # reciprocal truncation
    assert ch.rc <= 0.5 * L - 0.5 + 1e-9                                 # minimum image with skin
    # the choice is the cheapest of its rc grid: a neighbour cutoff is not cheaper
    for drc in (-0.3, 0.3):
        rc = ch.rc + drc
        if 3.0 <= rc <= min(10.0, 0.5 * L - 0.5):
            alpha = ch.alpha * ch.rc / rc
            kmax = math.ceil(alpha * L * math.sqrt(-math.log(1e-6)) / math.pi)
            nk = kmax + kmax * (2 * kmax + 1) + kmax * (2 * kmax + 1) ** 2
            cost = n * (300.0 * 0.5 * n / L ** 3 * 4.0 / 3.0 * math.pi * rc ** 3 + 35.0 * nk)
            assert cost >= ch.cost * (1 - 1e-12)


@pytest.mark.parametrize("c,n", [(0, 96), (1, 192)])
def test_ewald_tune_force_error_vs_converged_sum(c, n):
    """The tuned alpha and kmax of a configuration against the converged sum at the same
    real-space cutoff (oracle restatement, FP64, damped polarisable model): the relative
    RMS force error is a few times eps (measured 6.9e-6 at 96 ions, 4.9e-6 at 192 for
    eps = 1e-6); bar 1e-5."""
    from oracle.oracle import Oracle

    def forces(x):
        o = Oracle(x)
        o.gen_verletlist()
        o.engforce()
        return o.forces()

    s = fit.config4_one(c, n, conv_tol=1e-11, eps=1e-6)
    conv = fit.ewald_converged(s.cell[0, 0], s.cutlongrange)
    assert conv.alpha > s.alphaES and conv.kmax > s.kES[0]
    f, fr = forces(s), forces(fit.with_ewald(s, conv))
    err = float(np.sqrt(np.mean(np.sum((f - fr) ** 2, 1))) / np.sqrt(np.mean(np.sum(fr ** 2, 1))))
    assert err < 1e-5, err


def test_config4_sizes():
    sizes = fit.config4_sizes()
    assert len(sizes) == 512
    assert all(s % 96 == 0 and 96 <= s <= 1536 for s in sizes)
    assert len(set(sizes)) == 16
    assert 3.8e5 < sum(sizes) < 4.6e5          # about 4.2e5 ions in all
    assert sizes == fit.config4_sizes()         # seeded


def test_theta_roundtrip():
    s = fit.config4(sizes=[96])[0]
    th = fit.theta_of(s)
    assert th.shape == (fit.NPARAM,)
    t2 = fit.perturbed_theta(th)
    nz = th != 0.0
    assert np.allclose(np.abs(t2[nz] / th[nz] - 1.0), 0.05)
    assert np.all(t2[~nz] == 0.0)                 # D = 0 (no C8 term in this model) stays 0
    assert np.array_equal(fit.theta_of(fit.with_theta(s, t2)), t2)
    assert np.array_equal(fit.theta_of(s), th)   # the original is untouched


def test_shard_balanced():
    sizes = fit.config4_sizes()
    for world in (1, 2, 4, 8):
        bins = fit.shard(sizes, world)
        assert sorted(c for b in bins for c in b) == list(range(len(sizes)))
        loads = [sum(sizes[c] for c in b) for b in bins]
        assert max(loads) - min(loads) <= max(sizes)


SHARD_SIZES = [96, 192, 96, 192]
SHARD_PARAMS = (6,)   # gradient entry by central differences: q_Si


def _config_loss_grad(c, size, theta, ft, ntot):
    """One configuration's share of the fit loss L = sum |F - F_t|^2 / (3 N_total) and of
    the SHARD_PARAMS gradient entries (central differences), forces from the oracle
    restatement."""
    from oracle.oracle import Oracle
    s = fit.config4_one(c, size, conv_tol=1e-10)

    def loss(th):
        o = Oracle(fit.with_theta(s, th))
        o.gen_verletlist()
        o.engforce()
        return float(np.sum((o.forces() - ft) ** 2) / (3.0 * ntot))

    grad = np.zeros(fit.NPARAM)
    for k in SHARD_PARAMS:
        h = 1e-5 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        grad[k] = (loss(tp) - loss(tm)) / (2.0 * h)
    return loss(theta), grad


def _shard_inputs():
    from oracle.oracle import Oracle
    systems = [fit.config4_one(c, n, conv_tol=1e-10) for c, n in enumerate(SHARD_SIZES)]
    th0 = fit.theta_of(systems[0])
    tht = fit.perturbed_theta(th0)
    targets = []
    for s in systems:
        o = Oracle(fit.with_theta(s, tht))
        o.gen_verletlist()
        o.engforce()
        targets.append(o.forces())
    return th0, targets


def _rank_main(rank, world, port, th0, targets, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = fit.shard(SHARD_SIZES, world)[rank]
        ntot = sum(SHARD_SIZES)
        loss, grad = 0.0, np.zeros(fit.NPARAM)
        for c in mine:
            lc, gc = _config_loss_grad(c, SHARD_SIZES[c], th0, targets[c], ntot)
            loss += lc
            grad += gc
        tot, g = fit.allreduce_loss_grad(loss, grad)
        out[rank] = (tot, g, sorted(mine))
    finally:
        dist.destroy_process_group()


def test_sharded_loss_and_gradient_two_gloo_ranks():
    """Configurations sharded over 2 gloo ranks, each rank's per-configuration losses and
    gradient entries summed by one all-reduce: equal to the unsharded sums."""
    import torch.multiprocessing as mp
    th0, targets = _shard_inputs()
    mgr = mp.Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() % 2000)
    mp.spawn(_rank_main, args=(2, port, th0, targets, out), nprocs=2, join=True)
    ntot = sum(SHARD_SIZES)
    want_loss, want_grad = 0.0, np.zeros(fit.NPARAM)
    for c, n in enumerate(SHARD_SIZES):
        lc, gc = _config_loss_grad(c, n, th0, targets[c], ntot)
        want_loss += lc
        want_grad += gc
    assert sorted(out[0][2] + out[1][2]) == list(range(len(SHARD_SIZES)))
    assert out[0][2] and out[1][2]                     # both ranks did work
    for r in (0, 1):
        tot, g, _ = out[r]
        assert abs(tot - want_loss) <= 1e-12 * want_loss
        assert np.allclose(g, want_grad, rtol=1e-9, atol=0.0)
        assert np.all(g[list(SHARD_PARAMS)] != 0.0)


def test_oracle_loss_matches_reference_fixture():
    """The oracle restatement's forces at the fixture's parameters reproduce the
    reference's loss (FP64, SCF converged to 1e-11)."""
    from oracle.oracle import Oracle
    g = load_golden("fit96")
    s = fit.config4(sizes=[96], conv_tol=1e-11)[0]
    s.pos = g["r_in"].reshape(-1, 3)
    ft = g["f_t"].reshape(-1, 3)
    o = Oracle(fit.with_theta(s, g["theta0"]))
    o.gen_verletlist()
    o.engforce()
    f = o.forces()
    assert np.abs(f - g["f0"].reshape(-1, 3)).max() < 1e-9 * np.abs(f).max()
    loss = float(np.sum((f - ft) ** 2) / (3.0 * s.nion))
    assert abs(loss - float(g["loss0"][0])) < 1e-9 * float(g["loss0"][0])
