"""The sum rearrangements the mixed-precision k-space kernels are built on, checked in
FP64 numpy against the direct sums over k-vectors on random ions (no GPU).

* rho pass (k_rho32, k_rho_tc): with E2[-z] = conj E2[z] = (c, -d), eight weighted sums
  per |nz| over the ions give rho(+z) and rho(-z) of a row (nx, ny).
* ion pass (k_ion32, k_ion32x2): with Y(k) = Ak rho(k) conj(exp(i k.r)), the field and
  force sums of a row are conj(w) G, conj(w) H, conj(w) K of the row phase w and three
  complex z-sums whose weights fold rho(+z) and rho(-z) over the sign of nz.
"""
import numpy as np


def _ions(rng, n):
    t = rng.random((n, 3))                    # fractional coordinates B^T r
    q = rng.normal(size=n)
    m = rng.normal(size=(n, 3))               # 2 pi B^T mu
    return t, q, m


def test_paired_rho_sums():
    rng = np.random.default_rng(7)
    t, q, m = _ions(rng, 40)
    K2 = 6
    for nx, ny in [(0, 1), (2, -3), (1, 0)]:
        b = np.exp(2j * np.pi * (nx * t[:, 0] + ny * t[:, 1]))
        c0 = nx * m[:, 0] + ny * m[:, 1]
        c1 = m[:, 2]
        B1 = (q + 1j * c0) * b
        B2 = 1j * c1 * b
        for z in range(1, K2 + 1):
            E = np.exp(2j * np.pi * z * t[:, 2])
            c, d = E.real, E.imag
            Sa, Sb = np.sum(B1.real * c), np.sum(B1.imag * d)
            Sc, Sd = np.sum(B1.real * d), np.sum(B1.imag * c)
            Ta, Tb = np.sum(B2.real * c), np.sum(B2.imag * d)
            Tc, Td = np.sum(B2.real * d), np.sum(B2.imag * c)
            plus = (Sa - Sb + z * (Ta - Tb)) + 1j * (Sc + Sd + z * (Tc + Td))
            minus = (Sa + Sb - z * (Ta + Tb)) + 1j * (Sd - Sc + z * (Tc - Td))
            for sgn, got in ((1, plus), (-1, minus)):
                n = np.array([nx, ny, sgn * z])
                direct = np.sum((q + 1j * (m @ n)) * np.exp(2j * np.pi * (t @ n)))
                assert abs(got - direct) < 1e-12 * max(1.0, abs(direct))


def test_folded_ion_sums():
    rng = np.random.default_rng(11)
    K2 = 7
    rp = rng.normal(size=K2) + 1j * rng.normal(size=K2)     # Ak rho(+z), z = 1..K2
    rn = rng.normal(size=K2) + 1j * rng.normal(size=K2)     # Ak rho(-z)
    r0 = complex(rng.normal(), rng.normal())                # Ak rho(0)
    z = np.arange(1, K2 + 1)
    a1, a2 = rp.real + rn.real, rp.imag - rn.imag
    a3, a4 = rp.imag + rn.imag, rn.real - rp.real
    for tz, th in rng.random((5, 2)):
        e = np.exp(2j * np.pi * z * tz)
        w = np.exp(2j * np.pi * th)
        c, d = e.real, e.imag
        G = complex(r0.real + np.sum(a1 * c + a2 * d), r0.imag + np.sum(a3 * c + a4 * d))
        H = complex(np.sum(z * (-a4 * c + a3 * d)), np.sum(z * (a2 * c - a1 * d)))
        K = complex(np.sum(z * z * (a1 * c + a2 * d)), np.sum(z * z * (a3 * c + a4 * d)))
        # direct: Y = Ak rho conj(exp(i k.r)) for +z, -z and z = 0
        yp = rp * np.conj(w * e)
        ym = rn * np.conj(w * np.conj(e))
        y0 = r0 * np.conj(w)
        sums = {
            "G": y0 + np.sum(yp + ym),
            "H": np.sum(z * (yp - ym)),
            "K": np.sum(z * z * (yp + ym)),
        }
        for name, folded in (("G", G), ("H", H), ("K", K)):
            got = np.conj(w) * folded
            assert abs(got - sums[name]) < 1e-12 * max(1.0, abs(sums[name])), name
