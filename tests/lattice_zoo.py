"""A short line that exercises every element type and flag the GPU path
implements (test fixture).  Strengths are physical but the line is not a
closed ring; parity tests track it for a few passes only."""
from __future__ import annotations

import math

from simtrack_b200.lattices import ElementSpec as S
from simtrack_b200.lattices import Lattice, mult_args

GAMMA_100GEV = 100000.0 / 938.27201


def zoo(bb_round: bool = True) -> Lattice:
    err = [0.0, 0.05, 1e-4, -2e-3, 5e-2, -1.0, 10.0, -300.0, 4e3, -5e4, 1e6]
    serr = [0.0, 0.0, -2e-4, 1e-3, -4e-2, 2.0, -8.0, 200.0, -3e3, 6e4, -8e5]
    els = [
        S("QUAD", "q1", (1.1, 0.12, 0.0), {"Nint": 4}, misalign=(2e-4, -1e-4, 0.0, 0.0, 0.0, 3e-3)),
        S("DRIFT", "d1", (0.7,)),
        S("SBEND", "b1", (3.0, 0.02, 0.004, -0.006)),
        S("SEXT", "s1", (0.3, 0.6, 0.05), {"Nint": 2}),
        S("OCT", "o1", (0.0, 30.0, -5.0)),
        S("OCT", "o2", (0.2, 12.0, 3.0), {"Nint": 2}),
        S("QUAD", "q2", (1.1, -0.11, 0.002), {"Nint": 4}, misalign=(0.0, 3e-4, 0.0, 0.0, 0.0, 0.0)),
        S("MULT", "m1", mult_args(1.5, [0.0] + err[1:], serr), {"Nint": 3}),
        S("MULT", "m2", mult_args(0.0, [1e-5, 0.0, 0.3, 0.0, 50.0], [0.0, 1e-3, 0.0, -20.0])),
        S("GSBEND", "gb1", (2.0, 0.015, 0.0151, 0.002, 0.003)),
        S("SBENDMULT", "sbm1", (2.5, 0.01, 0.001, 0.001, *([0.0, 0.0, 0.2, 0.0, 30.0] + [0.0] * 6),
                                *([0.0, 0.0, 0.0, 5.0] + [0.0] * 7)), {"Nint": 2}),
        S("GMULT", "gm1", (1.2, -0.008, 0.0, 0.002, *([0.0, 0.01, 0.0, 1.0] + [0.0] * 7), *([0.0] * 11))),
        S("SKEWQ", "sq1", (0.4, 0.01), {"Nint": 2}),
        S("KICKER", "k1", (0.5, 1e-5, -2e-5)),
        S("HKICKER", "hk1", (0.0, 3e-6)),
        S("VKICKER", "vk1", (0.2, -4e-6)),
        S("RFCAV", "rf1", (0.4, 3.0, 28.0e6, 0.1)),
        S("CRABRF", "cr1", (0.0, 2.0, 197.0e6, 0.0)),
        S("CCMULT", "cc1", (0.0, 1.5, 394.0e6, 0.2, 0.01, 0.02, 3.0, -2.0, 40.0, 30.0, 800.0, -500.0)),
        S("LBT", "lbt", (0.0125,)),
        S("BEAMBEAM", "bbflat", (6, 1.7e11, -1.0, 0.06, 7, 95e-6 ** 2 / 0.8, 0.8, 0.0, 8.5e-6 ** 2 / 0.072, 0.072,
                                  0.0)),
        S("ILBT", "ilbt", (0.0125,)),
        S("BEAMBEAM", "bbround", (6, 2e11, 1.0, 0.3, 5, 2.4e-8, 0.6, 0.0, 2.4e-8, 0.6, 0.0)),
        S("BEAMBEAM", "bb11", (6, 1e11, 1.0, 0.2, 11, 3e-8, 0.5, 0.1, 2e-8, 0.4, -0.05)),
        S("BEAMBEAM", "bb4", (4, 1e11, 1.0, 0.2, 1, 3e-8, 0.5, 0.0, 1e-8, 0.5, 0.0)),
        S("BEAMBEAM", "bb4r", (4, 1e11, 1.0, 0.2, 1, 3e-8, 0.5, 0.0, 3e-8, 0.5, 0.0)),
        S("MARKER", "mk", (0.0,)),
        S("QUAD", "q3", (0.0, 0.02, 0.01)),
        S("SEXT", "s0", (0.5, 0.0, 0.0)),
        S("DRIFT", "d2", (1.3,)),
    ]
    lat = Lattice("zoo", els, GAMMA_100GEV)
    lat.meta["turns"] = 3
    return lat


def zoo_particles():
    """A handful of particles across x/y/z/pt, including one that the entry
    check rejects and one launched on the axis."""
    import numpy as np
    P = [
        [1e-3, 1e-5, 5e-4, -2e-5, 0.01, 2e-4],
        [-2e-3, 0.0, 1e-3, 1e-5, -0.05, -5e-4],
        [3e-4, -3e-5, -2e-4, 0.0, 0.1, 1e-3],
        [0.0, 0.0, 0.0, 0.0, 0.0, 0.0],
        [5e-3, 2e-4, -4e-3, 1e-4, 0.2, -1e-3],
        [0.2, 0.0, 0.0, 0.0, 0.0, 0.0],
        [1e-4, 1e-6, 1e-4, 1e-6, -0.3, 3e-4],
    ]
    return np.array(P, dtype=np.float64)


def spin_zoo() -> Lattice:
    """The zoo without the element types whose spin form is not implemented
    (GSBEND, GMULT), plus thin forms that only spin tracking treats apart
    (thin sextupole, thin bend multipole, a zero-strength kicker)."""
    base = zoo()
    els = [e for e in base.elements if e.type not in ("GSBEND", "GMULT")]
    els += [
        S("SEXT", "s_thin", (0.0, 0.8, -0.2)),
        S("SBENDMULT", "sbm0", (0.0, 0.003, 0.0, 0.0, *([0.0, 0.0, 0.1, 0.0, 10.0] + [0.0] * 6),
                                 *([0.0, 0.0, 0.0, 2.0] + [0.0] * 7))),
        S("KICKER", "k0", (0.3, 0.0, 0.0)),
        S("SBEND", "b2", (2.0, -0.015, 0.0, 0.0), {"Nint": 3}),
    ]
    lat = Lattice("spin_zoo", els, GAMMA_100GEV)
    lat.meta["turns"] = 2
    return lat


def patch_solen_zoo() -> Lattice:
    """Coordinate patches and solenoids, arranged as around the detector
    solenoid of the Bmad HSR table (rotate, solenoid, translate back, rotate
    back), plus a solenoid with KS == 0, a misaligned one, a patch with both
    offsets and a rotation, and one whose rotation is below YROTAT_Pass's
    1e-9 threshold."""
    els = [
        S("QUAD", "q1", (1.0, 0.08, 0.0), {"Nint": 4}),
        S("PATCH", "pb", (0.0, 0.0, 0.0, -0.025)),
        S("SOLEN", "sol", (2.0, 0.15)),
        S("PATCH", "pe", (-0.05, 1e-4, -6.25e-4, 0.0)),
        S("PATCH", "pr", (0.0, 0.0, 0.0, 0.025)),
        S("SOLEN", "sol0", (1.5, 0.0)),
        S("SOLEN", "solm", (0.8, -0.3), misalign=(1e-4, -2e-4, 0.0, 0.0, 0.0, 2e-3)),
        S("PATCH", "pm", (2e-4, -1e-4, 3e-4, 1e-3)),
        S("PATCH", "ptiny", (0.0, 0.0, 0.0, 5e-10)),
        S("DRIFT", "d1", (0.5,)),
        S("QUAD", "q2", (1.0, -0.08, 0.0), {"Nint": 4}),
    ]
    lat = Lattice("patch_solen", els, 275000.0 / 938.27201)
    lat.meta["turns"] = 3
    return lat


def thin_fodo_ring() -> Lattice:
    """One thin-lens FODO cell with thin sextupoles as a ring (7 elements,
    tunes 0.3 / 0.3): cheap enough for the reference's own 2,048-turn
    frequency and Lyapunov maps on a CPU.  The sextupoles are strong enough
    (K2L = +/-60) that about a third of a 0-6 mm amplitude grid is lost."""
    mu = 2 * math.pi * 0.3
    k = 2 * math.sin(mu / 2) / 1.0  # 1/f for 1 m drifts
    els = [S("QUAD", "qf1", (0.0, k / 2, 0.0)), S("DRIFT", "d1", (1.0,)), S("SEXT", "sf", (0.0, 60.0, 0.0)),
           S("QUAD", "qd", (0.0, -k, 0.0)), S("DRIFT", "d2", (1.0,)), S("SEXT", "sd", (0.0, -60.0, 0.0)),
           S("QUAD", "qf2", (0.0, k / 2, 0.0))]
    return Lattice("thin_fodo", els, GAMMA_100GEV)


def spin_particles():
    """zoo_particles with a spin unit vector appended to each."""
    import numpy as np
    x = zoo_particles()
    s = np.array([[0.0, 1.0, 0.0], [0.6, 0.8, 0.0], [0.0, 0.6, 0.8], [1.0, 0.0, 0.0],
                  [0.36, 0.48, 0.8], [0.0, 1.0, 0.0], [-0.28, 0.96, 0.0]])
    return np.concatenate([x, s], axis=1)
