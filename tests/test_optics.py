"""One-turn Jacobian, Twiss functions and symplectic defect."""
import math

import numpy as np
import pytest

from simtrack_b200.optics import symplectic_defect, symplectic_form, twiss_from_matrix


def _twiss_matrix(beta, alpha, mu):
    g = (1 + alpha * alpha) / beta
    c, s = math.cos(mu), math.sin(mu)
    return np.array([[c + alpha * s, beta * s], [-g * s, c - alpha * s]])


def test_twiss_from_matrix_recovers_parameters():
    M = np.eye(6)
    M[0:2, 0:2] = _twiss_matrix(12.5, -1.3, 2 * math.pi * 0.31)
    M[2:4, 2:4] = _twiss_matrix(3.25, 0.4, 2 * math.pi * 0.82)
    tw = twiss_from_matrix(M)
    assert abs(tw.beta_x - 12.5) < 1e-12 and abs(tw.alpha_x + 1.3) < 1e-12
    assert abs(tw.beta_y - 3.25) < 1e-12 and abs(tw.alpha_y - 0.4) < 1e-12
    assert abs(tw.tune_x - 0.31) < 1e-12 and abs(tw.tune_y - 0.82) < 1e-12
    assert symplectic_defect(M) < 1e-14


def test_defect_detects_non_symplectic_map():
    M = np.eye(6)
    M[0, 0] = 1.001
    assert symplectic_defect(M) > 5e-4
    J = symplectic_form()
    assert np.array_equal(J.T, -J)


def _fd_jacobian_port(port, x_ref, steps):
    pts = [np.array(x_ref, dtype=float)]
    for k in range(6):
        for sgn in (1.0, -1.0):
            p = np.array(x_ref, dtype=float)
            p[k] += sgn * steps[k]
            pts.append(p)
    x = np.array(pts)
    out, st, _, _ = port.track(x, 1)
    M = np.empty((6, 6))
    for k in range(6):
        M[:, k] = (out[1 + 2 * k] - out[2 + 2 * k]) / (2 * steps[k])
    return M


@pytest.mark.gpu
@pytest.mark.parametrize("ring", ["fodo", "rhic"])
def test_gpu_jacobian_matches_oracle_and_is_symplectic(ring, port_oracle, native_lib):
    from simtrack_b200 import lattices as lt
    from simtrack_b200.api import Table
    from simtrack_b200.optics import DEFAULT_STEPS, one_turn_jacobian
    lat = lt.fodo_ring() if ring == "fodo" else lt.rhic_like_ring(seed=1)
    table = Table(lt.build_line(lat))
    M = one_turn_jacobian(table)
    port_oracle.build(lat)
    Mp = _fd_jacobian_port(port_oracle, np.zeros(6), DEFAULT_STEPS)
    # identical one-turn tracking of the same 13 particles -> identical differences
    assert np.array_equal(M, Mp)
    # finite differences of a symplectic map: defect at the level of the FD error
    assert symplectic_defect(M) < 2e-6
    tw = twiss_from_matrix(M)
    assert tw.beta_x > 0 and tw.beta_y > 0


@pytest.mark.gpu
@pytest.mark.parametrize("deltap", [0.0, 4e-4])
def test_gpu_closed_orbit_matches_reference(deltap, native_lib, ref_oracle):
    """Cal_Orbit_Num (simtrack.cpp:14947) on a ring with offset quadrupoles:
    the orbit after every element equals the reference's bit for bit."""
    from simtrack_b200 import lattices as lt
    from simtrack_b200.api import Cal_Orbit_Num
    lat = lt.rhic_like_ring(seed=2)
    rng = np.random.default_rng(4)
    for e in lat.elements:
        if e.type == "QUAD" and rng.random() < 0.1:
            e.misalign = (rng.normal(0, 1e-4), rng.normal(0, 1e-4), 0.0, 0.0, 0.0, 0.0)
    line = lt.build_line(lat)
    orbit = Cal_Orbit_Num(line, deltap)
    ref_oracle.build(lat)
    ref = ref_oracle.cal_orbit(deltap)
    assert np.max(np.abs(orbit[:, 0])) > 1e-5  # a real orbit distortion
    assert np.array_equal(orbit, ref)
