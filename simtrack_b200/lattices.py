"""Lattice descriptions and the synthetic rings of the benchmark workloads.

A lattice is a list of ElementSpec records: the element type and the
reference constructor arguments after the name (simtrack.h:399-1059), the
SetP calls applied after construction, and optional misalignment/aperture
fields.  The same description builds a product Line (build_line) and, in the
tests, the reference oracle's Line, so both sides see identical inputs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

from . import api

PROTON_MASS_MEV = 938.27201  # simtrack.h:38 (GP.energy0 default)


@dataclass
class ElementSpec:
    type: str
    name: str
    args: Tuple[float, ...]
    setp: Dict[str, float] = field(default_factory=dict)
    misalign: Optional[Tuple[float, float, float, float, float, float]] = None
    aperture: Optional[Tuple[float, float]] = None


@dataclass
class Lattice:
    name: str
    elements: List[ElementSpec]
    gamma: float
    E0: float = PROTON_MASS_MEV
    Q: float = 1.0
    A: float = 1.0
    quad_fringe: bool = False
    aperture_radius: float = 0.0
    meta: dict = field(default_factory=dict)

    def set_reference(self) -> None:
        api.Set_RefPartEnergy(self.gamma, self.E0, self.Q, self.A)
        api.Set_Flags(False, self.quad_fringe)

    @property
    def circumference(self) -> float:
        return sum(_length(e) for e in self.elements)


def _length(e: ElementSpec) -> float:
    if e.type in ("LBT", "ILBT", "BEAMBEAM"):
        return 0.0
    return float(e.args[0])


def make_element(e: ElementSpec) -> api.Element:
    el = api.Element(e.type, e.name, e.args)
    for k, v in e.setp.items():
        el.SetP(k, v)
    if e.misalign is not None:
        el.set_misalignment(*e.misalign)
    if e.aperture is not None:
        el.set_aperture(*e.aperture)
    return el


def build_line(lat: Lattice) -> api.Line:
    """Sets the reference particle and builds the product Line for `lat`."""
    lat.set_reference()
    line = api.Line()
    for e in lat.elements:
        line.Append(make_element(e))
    return line


def mult_args(L: float, knl: Sequence[float], knsl: Sequence[float]) -> Tuple[float, ...]:
    kn = list(knl) + [0.0] * (11 - len(knl))
    ks = list(knsl) + [0.0] * (11 - len(knsl))
    return (L, *kn, *ks)


def fodo_ring(ncell: int = 100, gamma: Optional[float] = None, nint: int = 4, k1=0.06, k2l=0.4,
              vrf_mv: float = 3.0, harmonic: int = 360, drift: float = 0.5) -> Lattice:
    """Small plain-method ring: `ncell` FODO cells with two thick sector dipoles
    (L = 2 m, angle 2*pi/(2*ncell)), QF/QD thick quadrupoles (L = 1 m,
    K1 = +/-0.06 m^-2, `nint` Yoshida slices), two thin chromatic sextupoles
    (K2L = +/-0.4 m^-2), 0.5 m drifts, and one thin RF cavity (3 MV, h = 360).
    Protons at 100 GeV total energy."""
    if gamma is None:
        gamma = 100000.0 / PROTON_MASS_MEV
    ang = 2 * math.pi / (2 * ncell)
    els: List[ElementSpec] = []
    for c in range(ncell):
        els += [
            ElementSpec("QUAD", f"qf{c}", (1.0, k1 * 1.0, 0.0), {"Nint": nint}),
            ElementSpec("DRIFT", f"d1_{c}", (drift,)),
            ElementSpec("SEXT", f"sf{c}", (0.0, k2l, 0.0)),
            ElementSpec("DRIFT", f"d2_{c}", (drift,)),
            ElementSpec("SBEND", f"b1_{c}", (2.0, ang, 0.0, 0.0)),
            ElementSpec("DRIFT", f"d3_{c}", (drift,)),
            ElementSpec("QUAD", f"qd{c}", (1.0, -k1 * 1.0, 0.0), {"Nint": nint}),
            ElementSpec("DRIFT", f"d4_{c}", (drift,)),
            ElementSpec("SEXT", f"sd{c}", (0.0, -k2l, 0.0)),
            ElementSpec("DRIFT", f"d5_{c}", (drift,)),
            ElementSpec("SBEND", f"b2_{c}", (2.0, ang, 0.0, 0.0)),
            ElementSpec("DRIFT", f"d6_{c}", (drift,)),
        ]
    lat = Lattice("fodo100", els, gamma)
    C = lat.circumference
    beta = math.sqrt(1.0 - 1.0 / gamma / gamma)
    frf = harmonic * beta * 299792458.0 / C
    els.append(ElementSpec("RFCAV", "rf", (0.0, vrf_mv, frf, 0.0)))
    lat.meta.update({"harmonic": harmonic, "frf": frf, "emit_norm": 2.5e-6})
    return lat
