"""One-turn map diagnostics from the GPU tracker.

The one-turn Jacobian M comes from central finite differences of one-turn
tracking (13 particles: the reference orbit and +-h along each coordinate),
as the reference obtains its one-turn matrix numerically around the closed
orbit (Cal_Orbit_Num, simtrack.cpp:14947, and the matrix around it).  From M
follow the uncoupled Twiss functions at the start of the line and the
symplectic defect |M^T J M - J| (J in the (x,px), (y,py), (z,pt) pairs; z =
-c dt and pt form a canonical pair with the same orientation as x, px).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .api import Table

# Finite-difference steps per coordinate: transverse 3e-7 m / rad, z 3e-5 m,
# pt 3e-7.  Smaller steps lose to rounding (the exact bend map forms
# differences of quantities near 1, so its rounding error divided by the step
# grows like 1/h), larger ones to the truncation error (h^2).  With these
# steps the defect is near 5e-7 on both the FODO and the RHIC-like ring; with
# 1e-8 steps it is near 2e-5 on the RHIC-like ring.
DEFAULT_STEPS = (3e-7, 3e-7, 3e-7, 3e-7, 3e-5, 3e-7)


def symplectic_form(dim: int = 6) -> np.ndarray:
    J = np.zeros((dim, dim))
    for k in range(0, dim, 2):
        J[k, k + 1] = 1.0
        J[k + 1, k] = -1.0
    return J


def one_turn_jacobian(table: Table, x_ref=None, steps=DEFAULT_STEPS, nturn: int = 1,
                      aperture_radius: float = 0.0) -> np.ndarray:
    """Central-difference Jacobian of the nturn-turn map around x_ref (6,)."""
    x_ref = np.zeros(6) if x_ref is None else np.asarray(x_ref, dtype=np.float64)
    pts = [x_ref.copy()]
    for k in range(6):
        for sgn in (1.0, -1.0):
            p = x_ref.copy()
            p[k] += sgn * steps[k]
            pts.append(p)
    x = np.array(pts)
    out, stable, _, _ = table.track_host(x, nturn, aperture_radius)
    if not np.all(stable == 1):
        raise RuntimeError("a finite-difference particle was lost")
    M = np.empty((6, 6))
    for k in range(6):
        M[:, k] = (out[1 + 2 * k] - out[2 + 2 * k]) / (2.0 * steps[k])
    return M


def symplectic_defect(M: np.ndarray) -> float:
    """max |M^T J M - J| over the entries."""
    J = symplectic_form(M.shape[0])
    return float(np.max(np.abs(M.T @ J @ M - J)))


@dataclass
class Twiss:
    beta_x: float
    alpha_x: float
    beta_y: float
    alpha_y: float
    tune_x: float   # fractional
    tune_y: float


def twiss_from_matrix(M: np.ndarray) -> Twiss:
    """Periodic Twiss functions from the 2x2 diagonal blocks (coupling ignored)."""
    vals = []
    for k in (0, 2):
        m = M[k:k + 2, k:k + 2]
        c = 0.5 * (m[0, 0] + m[1, 1])
        if abs(c) >= 1.0:
            raise RuntimeError("unstable one-turn motion in plane %d" % (k // 2))
        s = math.copysign(math.sqrt(1.0 - c * c), m[0, 1])
        beta = m[0, 1] / s
        alpha = (m[0, 0] - m[1, 1]) / (2.0 * s)
        mu = math.atan2(s, c) % (2.0 * math.pi)
        vals += [beta, alpha, mu / (2.0 * math.pi)]
    return Twiss(vals[0], vals[1], vals[3], vals[4], vals[2], vals[5])
