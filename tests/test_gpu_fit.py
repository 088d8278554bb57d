"""Force-matching loss and adjoint gradient on the GPU (through the C ABI) against the
reference's FP64 forces and finite-difference gradient (tests/golden/fit96.npz), against
finite differences of the GPU loss itself, batched vs single evaluations, the
torch.autograd wrapper and the mixed-precision engine."""
import numpy as np
import pytest

from mdff20_b200 import fit
from mdff20_b200.engine import MIXED, PIM_CG, Engine
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), 1e-30)))


def test_gradient_vs_reference_finite_differences():
    g = load_golden("fit96")
    s = fit.config4(sizes=[96], conv_tol=1e-11)[0]
    pos = g["r_in"].reshape(-1, 3)
    e = Engine(s, positions=pos, pim_solver=PIM_CG)
    e.gen_verletlist()
    e.fit_set_params(fit.SI_TYPE, fit.O_TYPE, g["theta0"])
    scale = 2.0 / (3.0 * s.nion)
    sq, grad = e.force_match(fit.SI_TYPE, fit.O_TYPE, g["f_t"].reshape(-1, 3), scale)
    assert np.abs(e.forces() - g["f0"].reshape(-1, 3)).max() < 1e-8
    loss = 0.5 * scale * sq
    assert abs(loss - float(g["loss0"][0])) < 1e-8 * float(g["loss0"][0])
    # the reference gradient is a central difference (step 1e-5 relative): 1e-4 bar
    assert _rel(grad, g["grad_fd"]) < 1e-4, (grad, g["grad_fd"])
    e.close()


def test_gradient_vs_gpu_finite_differences():
    systems = fit.config4(sizes=[96, 192], conv_tol=1e-11)
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(systems, fit.perturbed_theta(th0))
    b = fit.ForceMatchBatch(systems, targets, threads=2)
    _, grad = b.loss_grad(th0)
    for k in range(fit.NPARAM):
        h = fit.fd_step(th0, k)
        tp, tm = th0.copy(), th0.copy()
        tp[k] += h
        tm[k] -= h
        gfd = (b.loss_grad(tp)[0] - b.loss_grad(tm)[0]) / (2.0 * h)
        assert abs(grad[k] - gfd) <= 1e-4 * abs(gfd), (fit.PARAM_NAMES[k], grad[k], gfd)
    b.close()


def test_batch_is_the_sum_of_single_evaluations():
    systems = fit.config4(sizes=[96, 288, 192])
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(systems, fit.perturbed_theta(th0, seed=9))
    b = fit.ForceMatchBatch(systems, targets, threads=3)
    loss, grad = b.loss_grad(th0)
    sq, gs = 0.0, np.zeros(fit.NPARAM)
    for e, t in zip(b.engines, targets):
        e.fit_set_params(fit.SI_TYPE, fit.O_TYPE, th0)
        a, g = e.force_match(fit.SI_TYPE, fit.O_TYPE, t, b.scale)
        sq += a
        gs += g
    assert abs(loss - 0.5 * b.scale * sq) <= 1e-12 * loss
    assert _rel(grad, gs) < 1e-10
    b.close()


def test_torch_autograd_wrapper():
    import torch
    systems = fit.config4(sizes=[96, 192], conv_tol=1e-10)
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(systems, fit.perturbed_theta(th0))
    b = fit.ForceMatchBatch(systems, targets, threads=2)
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    loss = fit.ForceMatchLoss.apply(theta, b)
    loss.backward()
    _, grad = b.loss_grad(th0)
    assert np.allclose(theta.grad.numpy(), grad, rtol=1e-12, atol=0.0)
    # directional derivative along a mixed direction against a central difference
    v = np.array([1.0, 1e-4, 1.0, 1.0, 1e-4, 1.0, 1e-4, 1e-4, 1e-4, 1e-4, 0.0, 0.0]) * th0 * 1e-5
    v[10:] = 1e-2   # the C8 dispersion (zero in this model): an absolute step
    d_fd = (b.loss_grad(th0 + v)[0] - b.loss_grad(th0 - v)[0]) / 2.0
    assert abs(float(np.dot(grad, v)) - d_fd) <= 1e-4 * abs(d_fd)
    b.close()


def test_mixed_precision_gradient_close_to_fp64():
    systems = fit.config4(sizes=[192, 480], conv_tol=1e-8)
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(systems, fit.perturbed_theta(th0))
    ref = fit.ForceMatchBatch(systems, targets, threads=2)
    mix = fit.ForceMatchBatch(systems, targets, threads=2, precision=MIXED)
    l64, g64 = ref.loss_grad(th0)
    l32, g32 = mix.loss_grad(th0)
    assert abs(l32 - l64) < 1e-4 * l64
    assert np.max(np.abs(g32 - g64)) < 1e-4 * np.max(np.abs(g64))
    ref.close()
    mix.close()


@pytest.mark.parametrize("precision", [0, MIXED])
def test_recorded_plan_matches_host_driven_batch(precision):
    """mdffgpu_fit_plan (each configuration's evaluation recorded once as a CUDA graph,
    theta from a device buffer, both CG loops device-controlled) against the host-driven
    batch, over several theta values replayed through the same graphs."""
    systems = fit.config4(sizes=[96, 288, 192, 384], conv_tol=1e-9)
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(systems, fit.perturbed_theta(th0, seed=7))
    rec = fit.ForceMatchBatch(systems, targets, precision=precision)
    host = fit.ForceMatchBatch(systems, targets, precision=precision, threads=4, recorded=False)
    rng = np.random.default_rng(3)
    for k in range(3):
        th = th0 * (1.0 + 0.02 * rng.standard_normal(fit.NPARAM)) if k else th0
        l1, g1 = rec.loss_grad(th)
        l2, g2 = host.loss_grad(th)
        assert abs(l1 - l2) <= 1e-9 * l2, (k, l1, l2)
        assert np.max(np.abs(g1 - g2)) <= 1e-8 * np.max(np.abs(g2)), (k, g1, g2)
    # after the replays a context holds the last theta on the device and in its host
    # copies: a single evaluation without setting theta agrees with the host-driven one
    a = rec.engines[1].force_match(fit.SI_TYPE, fit.O_TYPE, targets[1], rec.scale)
    b = host.engines[1].force_match(fit.SI_TYPE, fit.O_TYPE, targets[1], host.scale)
    assert abs(a[0] - b[0]) <= 1e-9 * b[0]
    assert np.max(np.abs(a[1] - b[1])) <= 1e-8 * np.max(np.abs(b[1]))
    rec.close()
    host.close()


def test_recorded_plan_reports_nonconvergence():
    """An iteration cap the induced-dipole CG cannot meet comes back as ERR_SCF from a
    replayed evaluation, with the configuration named."""
    from mdff20_b200.engine import MdffgpuError
    systems = fit.config4(sizes=[96, 192], conv_tol=1e-10)
    systems[1].max_scf_pim_iter = 1
    th0 = fit.theta_of(systems[0])
    targets = fit.target_forces(fit.config4(sizes=[96, 192]), fit.perturbed_theta(th0))
    b = fit.ForceMatchBatch(systems, targets)
    with pytest.raises(MdffgpuError) as ex:
        b.loss_grad(th0)
    assert ex.value.code == 4 and "configuration 1" in str(ex.value)
    b.close()
