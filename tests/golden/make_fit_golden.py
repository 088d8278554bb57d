"""Regenerates tests/golden/fit96.npz: the force-matching loss and its FP64 reference
gradient from the compiled reference.

    make -C oracle ref && python tests/golden/make_fit_golden.py

One seeded 96-ion configuration of the batched fit (mdff20_b200.fit.config4 with the SCF
converged to 1e-11): the reference's forces at the perturbed parameters are the
targets, L(theta) = sum |F(theta) - F_t|^2 / (3 N) from the reference's forces, and the
gradient is the central finite difference of that L (relative steps 1e-5; for the C8
dispersion D, which is zero in this model, fit.fd_step's absolute step), every force
an output of the reference mdff20 C code (OMP_NUM_THREADS=1).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mdff20_b200 import fit  # noqa: E402
from oracle import ref  # noqa: E402

STEP = 1e-5


def fit96():
    return fit.config4(sizes=[96], conv_tol=1e-11)[0]


def main():
    s = fit96()
    th0 = fit.theta_of(s)
    tht = fit.perturbed_theta(th0)
    rt = ref.run(fit.with_theta(s, tht), "engforce")
    ft = rt["f"].reshape(-1, 3)

    def loss(th):
        r = ref.run(fit.with_theta(s, th), "engforce")
        f = r["f"].reshape(-1, 3)
        return float(np.sum((f - ft) ** 2) / (3.0 * s.nion)), r

    l0, r0 = loss(th0)
    grad = np.zeros(fit.NPARAM)
    for k in range(fit.NPARAM):
        h = fit.fd_step(th0, k, STEP)
        tp = th0.copy()
        tp[k] += h
        tm = th0.copy()
        tm[k] -= h
        grad[k] = (loss(tp)[0] - loss(tm)[0]) / (2.0 * h)
    np.savez(os.path.join(HERE, "fit96.npz"), r_in=r0["r_in"], theta0=th0, theta_t=tht, f_t=ft.ravel(),
             f0=r0["f"], loss0=np.array([l0]), grad_fd=grad, step=np.array([STEP]))
    print("fit96: loss", l0, "grad", grad)


if __name__ == "__main__":
    main()
