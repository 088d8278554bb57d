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
    assert np.allclose(np.abs(t2 / th - 1.0), 0.05)
    assert np.array_equal(fit.theta_of(fit.with_theta(s, t2)), t2)
    assert np.array_equal(fit.theta_of(s), th)   # the original is untouched


def test_shard_balanced():
    sizes = fit.config4_sizes()
    for world in (1, 2, 4, 8):
        bins = fit.shard(sizes, world)
        assert sorted(c for b in bins for c in b) == list(range(len(sizes)))
        loads = [sum(sizes[c] for c in b) for b in bins]
        assert max(loads) - min(loads) <= max(sizes)


def _rank_main(rank, world, port, sizes, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = fit.shard(sizes, world)[rank]
        # stand-in partial results: a per-configuration loss and gradient
        loss = sum(float(sizes[c]) for c in mine)
        grad = np.zeros(fit.NPARAM)
        for c in mine:
            grad += np.arange(fit.NPARAM) * sizes[c] + c
        tot, g = fit.allreduce_loss_grad(loss, grad)
        out[rank] = (tot, g)
    finally:
        dist.destroy_process_group()


def test_sharded_reduction_two_gloo_ranks():
    import torch.multiprocessing as mp
    sizes = fit.config4_sizes(nconf=37, seed=11)
    mgr = mp.Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() % 2000)
    mp.spawn(_rank_main, args=(2, port, sizes, out), nprocs=2, join=True)
    want_loss = float(sum(sizes))
    want_grad = sum(np.arange(fit.NPARAM) * s + c for c, s in enumerate(sizes))
    for r in (0, 1):
        tot, g = out[r]
        assert tot == want_loss
        assert np.array_equal(g, want_grad)


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
