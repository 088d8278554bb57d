"""Cell geometry on the host, with the reference's operation order (no FMA in numpy).

``lattice`` follows src/cell.c:13-91, ``kardir``/``dirkar`` src/cell.c:125-161 and
``wrap_positions`` the wrap that read_config applies to every configuration it reads
(src/config.c:442-444: kardir, subtract nearbyint, dirkar).
"""
from __future__ import annotations

import numpy as np


def lattice(A: np.ndarray):
    """Reciprocal rows B (A_j x A_k / volume), the volume and the perpendicular widths.

    The volume is sum_i Bunnorm[i][0] * A[i][0] as in src/cell.c:228-231 (the triple
    product for orthorhombic cells).
    """
    A = np.asarray(A, float)
    Bu = np.array([np.cross(A[1], A[2]), np.cross(A[2], A[0]), np.cross(A[0], A[1])])
    omega = Bu[0, 0] * A[0, 0] + Bu[1, 0] * A[1, 0] + Bu[2, 0] * A[2, 0]
    w = np.array([omega / np.sqrt(Bu[0, i] ** 2 + Bu[1, i] ** 2 + Bu[2, i] ** 2) for i in range(3)])
    B = Bu * (1.0 / omega)
    return B, float(omega), w


def kardir(pos: np.ndarray, B: np.ndarray) -> np.ndarray:
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    return np.stack([x * B[0, 0] + y * B[0, 1] + z * B[0, 2],
                     x * B[1, 0] + y * B[1, 1] + z * B[1, 2],
                     x * B[2, 0] + y * B[2, 1] + z * B[2, 2]], axis=1)


def dirkar(s: np.ndarray, A: np.ndarray) -> np.ndarray:
    a, b, c = s[:, 0], s[:, 1], s[:, 2]
    return np.stack([a * A[0, 0] + b * A[1, 0] + c * A[2, 0],
                     a * A[0, 1] + b * A[1, 1] + c * A[2, 1],
                     a * A[0, 2] + b * A[1, 2] + c * A[2, 2]], axis=1)


def wrap_positions(A: np.ndarray, pos: np.ndarray) -> np.ndarray:
    A = np.asarray(A, float)
    B, _, _ = lattice(A)
    s = kardir(np.asarray(pos, float), B)
    s = s - np.rint(s)
    return np.ascontiguousarray(dirkar(s, A))


def auto_es(A: np.ndarray, cutlongrange: float, epsw: float):
    """set_autoES (src/ewald.c:48-71): (alphaES, kES, cutlongrange) from the cell and epsw.

    The cutoff grows to half the smallest face distance when shorter; alpha takes the C
    integer abs() of a logarithm (truncation toward zero), so it moves in steps of
    sqrt(integer) / rc; kES = nearbyint(0.25 + |column k of A| alpha tol1 / pi).
    """
    import math

    A = np.asarray(A, float)
    _, _, w = lattice(A)
    rc = float(cutlongrange)
    half = 0.5 * float(min(w))
    if rc < half:
        rc = half
    eps = min(abs(epsw), 0.5)
    tol = math.sqrt(abs(math.log(eps * rc)))
    alpha = math.sqrt(float(abs(int(math.log(eps * rc * tol))))) / rc
    tol1 = math.sqrt(-math.log(eps * rc * (2.0 * tol * alpha) * (2.0 * tol * alpha)))
    anorm = [math.sqrt(A[0, k] * A[0, k] + A[1, k] * A[1, k] + A[2, k] * A[2, k]) for k in range(3)]
    kes = tuple(int(np.rint(0.25 + anorm[k] * alpha * tol1 / math.pi)) for k in range(3))
    return alpha, kes, rc
