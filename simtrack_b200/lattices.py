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
    radiate: bool = False  # GP.radiate
    radiation_seed: int = 1324

    def set_reference(self) -> None:
        api.Set_RefPartEnergy(self.gamma, self.E0, self.Q, self.A)
        api.Set_Flags(False, self.quad_fringe)
        api.Set_Radiation(self.radiate, self.radiation_seed)

    @property
    def circumference(self) -> float:
        return sum(_length(e) for e in self.elements)


def _length(e: ElementSpec) -> float:
    if e.type in ("LBT", "ILBT", "BEAMBEAM"):
        return 0.0
    if e.type == "PATCH":
        return float(e.args[2])  # L = DS (PATCH constructor, simtrack.cpp:12266)
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


ELECTRON_MASS_MEV = 0.51099895


def electron_ring(ncell: int = 40, energy_gev: float = 3.0, nint: int = 5, k1: float = 0.25, k2l: float = 0.3,
                  vrf_mv: float = 2.0, harmonic: int = 400, radiate: bool = True, seed: int = 1324,
                  gsbend: bool = False) -> Lattice:
    """An electron storage ring with synchrotron radiation (GP.radiate): `ncell`
    FODO cells, each with a thick sector dipole (L = 2 m, `nint` slices, each
    followed by radiation with quantum excitation) and a combined-function
    SBENDMULT (L = 1.5 m, `nint` slices with a small sextupole and skew
    quadrupole component, radiation after each slice), thick quadrupoles
    (K1 = +/-`k1` m^-2), thin sextupoles and one thin RF cavity.  Electrons
    (Q = -1) at `energy_gev` total energy; the two dipoles of a cell bend by
    2 pi / ncell together.  gsbend=True makes the sector dipoles GSBENDs whose
    field is 0.2 % above the frame's curvature (radiation by photon Monte
    Carlo, radiate2)."""
    gamma = energy_gev * 1000.0 / ELECTRON_MASS_MEV
    ang = 2 * math.pi / ncell
    a1, a2 = 0.6 * ang, 0.4 * ang
    els: List[ElementSpec] = []
    for c in range(ncell):
        knl = [0.0, 0.0, 0.02 * (1 if c % 2 == 0 else -1)] + [0.0] * 8
        knsl = [0.0, 1e-4] + [0.0] * 9
        els += [
            ElementSpec("QUAD", f"qf{c}", (0.5, k1 * 0.5, 0.0), {"Nint": 4}),
            ElementSpec("DRIFT", f"d1_{c}", (0.4,)),
            ElementSpec("SEXT", f"sf{c}", (0.0, k2l, 0.0)),
            ElementSpec("DRIFT", f"d2_{c}", (0.4,)),
            (ElementSpec("GSBEND", f"b{c}", (2.0, a1, a1 * 1.002, 0.0, 0.0), {"Nint": nint}) if gsbend else
             ElementSpec("SBEND", f"b{c}", (2.0, a1, 0.0, 0.0), {"Nint": nint})),
            ElementSpec("DRIFT", f"d3_{c}", (0.4,)),
            ElementSpec("QUAD", f"qd{c}", (0.5, -k1 * 0.5, 0.0), {"Nint": 4}),
            ElementSpec("DRIFT", f"d4_{c}", (0.4,)),
            ElementSpec("SEXT", f"sd{c}", (0.0, -k2l, 0.0)),
            ElementSpec("DRIFT", f"d5_{c}", (0.4,)),
            ElementSpec("SBENDMULT", f"bm{c}", (1.5, a2, 0.0, 0.0, *knl, *knsl), {"Nint": nint}),
            ElementSpec("DRIFT", f"d6_{c}", (0.4,)),
        ]
    lat = Lattice("electron_ring", els, gamma, E0=ELECTRON_MASS_MEV, Q=-1.0, A=1.0, radiate=radiate,
                  radiation_seed=seed)
    C = lat.circumference
    beta = math.sqrt(1.0 - 1.0 / gamma / gamma)
    frf = harmonic * beta * 299792458.0 / C
    els.append(ElementSpec("RFCAV", "rf", (0.0, vrf_mv, frf, 0.0)))
    lat.meta.update({"harmonic": harmonic, "frf": frf})
    return lat


# Strengths of the RHIC-like ring fitted by simtrack_b200.lattice_design
# (beta* = 0.6 m at both interaction points, tunes 50.31 / 48.32, linear
# chromaticity +1 / +1 from the arc sextupoles).  K1L in m^-1, K2L in m^-2.
RHIC_LIKE_STRENGTHS = dict(
    kf=0.1746771083134425, kd=-0.17162657379211274,
    q1=0.2940698212888416, q2=-0.1821646680742746, q3=-0.08577597512541496, q4=0.16666371327006477,
    ua=-0.05966870432529879, ub=0.030478182687441402,
    k2f=0.6497955572120756, k2d=-1.323393027511492,
)
RHIC_BETA_STAR = 0.6
RHIC_GAMMA = 100000.0 / PROTON_MASS_MEV  # 100 GeV protons


def triplet_errors(seed: int, nquad: int = 12, rms: float = 1e-4) -> "np.ndarray":
    """Gaussian b3..b10 / a3..a10 coefficients (units of 1e-4 at the reference
    radius are folded into `rms`) for `nquad` triplet quadrupoles: shape
    (nquad, 2, 8), [:, 0] normal, [:, 1] skew."""
    import numpy as np
    return np.random.default_rng(seed).standard_normal((nquad, 2, 8)) * rms


def rhic_like_ring(seed: Optional[int] = None, nint_arc: int = 4, nint_triplet: int = 8, bb: bool = True,
                   aperture_radius: float = 0.03, r_ref: float = 0.031) -> Lattice:
    """Synthetic RHIC-like ring, 3,834 m, ~1,800 elements.

    Six arcs of 36 FODO cells (thick sector dipoles L = 5.8 m, thick
    quadrupoles L = 1.1 m, thin chromatic sextupoles), two low-beta
    interaction regions (beta* = 0.6 m) whose thick triplet quadrupoles are
    MULT elements carrying random normal/skew errors b3..b10, a3..a10 of rms
    1e-4 relative at r_ref = 31 mm drawn from `seed` (no errors when seed is
    None), with the convention knl[n] = K1L * r_ref * 1e-4 * g * n! / r_ref^n of
    the reference's error assignment (Example2/DA_cal.cpp:284-290, Gaussian g
    instead of flat), four utility straights, RF at 28 MHz (h = 360) and
    197 MHz (h = 2520), and the weak-strong 6D beam-beam map at both IPs
    (2e11 protons, round sigma* = 0.12 mm, sigma_z = 0.3 m, 5 slices).
    Protons at 100 GeV; circular aperture of `aperture_radius`."""
    from . import lattice_design as D
    S = RHIC_LIKE_STRENGTHS
    err = triplet_errors(seed) if seed is not None else None
    a, b, c, d = D.ir_drifts()
    ua, ub, uc = D.util_drifts()
    els: List[ElementSpec] = []
    tq = [0]

    def triplet(name, L, k1l):
        knl = [0.0, k1l] + [0.0] * 9
        knsl = [0.0] * 11
        if err is not None:
            e = err[tq[0]]
            fac = 1.0
            for n in range(2, 10):
                fac *= n
                knl[n] = k1l * r_ref * 1e-4 * (e[0, n - 2] / 1e-4) * fac / r_ref ** n
                knsl[n] = k1l * r_ref * 1e-4 * (e[1, n - 2] / 1e-4) * fac / r_ref ** n
        tq[0] += 1
        return ElementSpec("MULT", name, mult_args(L, knl, knsl), {"Nint": nint_triplet})

    def half_ir(tag, reverse):
        h = [ElementSpec("DRIFT", f"dstar_{tag}", (D.L_STAR,)),
             triplet(f"q1_{tag}", D.LQ1, S["q1"]),
             ElementSpec("DRIFT", f"d12_{tag}", (d,)),
             triplet(f"q2_{tag}", D.LQ2, S["q2"]),
             ElementSpec("DRIFT", f"d23_{tag}", (c,)),
             triplet(f"q3_{tag}", D.LQ3, S["q3"]),
             ElementSpec("DRIFT", f"d34_{tag}", (b,)),
             ElementSpec("QUAD", f"q4_{tag}", (D.LQ4, S["q4"], 0.0), {"Nint": nint_arc}),
             ElementSpec("DRIFT", f"dir_{tag}", (a,))]
        return h[::-1] if reverse else h

    def half_util(tag, reverse):
        h = [ElementSpec("QUAD", f"qub_{tag}", (D.LQU, S["ub"], 0.0), {"Nint": nint_arc}),
             ElementSpec("DRIFT", f"dub_{tag}", (ub,)),
             ElementSpec("QUAD", f"qua_{tag}", (D.LQU, S["ua"], 0.0), {"Nint": nint_arc}),
             ElementSpec("DRIFT", f"dua_{tag}", (ua,))]
        return h[::-1] if reverse else h

    def bb_elem(tag):
        emit = 0.12e-3 ** 2 / RHIC_BETA_STAR
        return ElementSpec("BEAMBEAM", f"bb_{tag}", (6, 2e11, 1.0, 0.3, 5, emit, RHIC_BETA_STAR, 0.0, emit,
                                                     RHIC_BETA_STAR, 0.0))

    def arc(k):
        s = [ElementSpec("QUAD", f"qfh_{k}_0", (D.LQ / 2, S["kf"] / 2, 0.0), {"Nint": nint_arc})]
        for i in range(D.CELLS_PER_ARC):
            last = i == D.CELLS_PER_ARC - 1
            s += [ElementSpec("SEXT", f"sf_{k}_{i}", (0.0, S["k2f"], 0.0)),
                  ElementSpec("DRIFT", f"da_{k}_{i}", (D.LD,)),
                  ElementSpec("SBEND", f"ba_{k}_{i}", (D.LB, D.ANGLE, 0.0, 0.0)),
                  ElementSpec("QUAD", f"qd_{k}_{i}", (D.LQ, S["kd"], 0.0), {"Nint": nint_arc}),
                  ElementSpec("SEXT", f"sd_{k}_{i}", (0.0, S["k2d"], 0.0)),
                  ElementSpec("DRIFT", f"db_{k}_{i}", (D.LD,)),
                  ElementSpec("SBEND", f"bb_{k}_{i}", (D.LB, D.ANGLE, 0.0, 0.0)),
                  ElementSpec("QUAD", f"qf_{k}_{i}", ((D.LQ / 2, S["kf"] / 2, 0.0) if last else
                                                      (D.LQ, S["kf"], 0.0)), {"Nint": nint_arc})]
        return s

    gamma = RHIC_GAMMA
    beta = math.sqrt(1.0 - 1.0 / gamma / gamma)
    frev = beta * 299792458.0 / D.CIRC
    for k in range(D.N_ARC):
        if k == 0:
            if bb:
                els.append(bb_elem("ip1"))
            els += half_ir("ip1r", False)
        elif k == 3:
            els += half_ir("ip2l", True)
            if bb:
                els.append(bb_elem("ip2"))
            els += half_ir("ip2r", False)
        else:
            els += half_util(f"u{k}l", True)
            els.append(ElementSpec("DRIFT", f"duc_{k}", (2 * uc,)))
            if k == 1:
                els.append(ElementSpec("RFCAV", "rf28", (0.0, 0.3, 360 * frev, 0.0)))
                els.append(ElementSpec("RFCAV", "rf197", (0.0, 3.0, 2520 * frev, 0.0)))
            els += half_util(f"u{k}r", False)
        els += arc(k)
    els += half_ir("ip1l", True)
    lat = Lattice("rhic_like" + ("" if seed is None else f"_s{seed}"), els, gamma, aperture_radius=aperture_radius)
    lat.meta.update({"seed": seed, "beta_star": RHIC_BETA_STAR, "emit_norm": 2.5e-6, "frev": frev,
                     "sigma_ip": math.sqrt(2.5e-6 * RHIC_BETA_STAR / (beta * gamma))})
    return lat


def da_grid(lat: Lattice, namp: int, amax: float, nang: int, deltas: Sequence[float]) -> "np.ndarray":
    """Initial conditions of a DA scan at element 0: amplitudes 0..amax sigma
    (inclusive) x angles 90 deg*(i+1)/(nang+1) in x-y x momentum offsets (pt),
    px = py = z = 0, as Track_DA sets them (simtrack.cpp:21410-21416).
    Returned as (ndelta*nang*namp, 6), amplitude fastest."""
    import numpy as np
    sig = lat.meta["sigma_ip"]
    amps = np.linspace(0.0, amax, namp)
    out = []
    for dp in deltas:
        for i in range(nang):
            th = (90.0 / (nang + 1)) * (i + 1) * math.pi / 180
            for a in amps:
                out.append([a * math.cos(th) * sig, 0.0, a * math.sin(th) * sig, 0.0, 0.0, dp])
    return np.array(out)


def gaussian_beam(lat: Lattice, n: int, seed: int = 12345, sigma_z: float = 0.1, sigma_pt: float = 3e-4) -> "np.ndarray":
    """6D Gaussian distribution at element 0, Twiss-matched transversely
    (alpha* = 0 at the interaction point): sigma_x = sqrt(eps beta*),
    sigma_px = sqrt(eps / beta*); longitudinal sigma_z, sigma_pt as given."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sx = lat.meta["sigma_ip"]
    spx = sx / lat.meta["beta_star"]
    g = rng.standard_normal((n, 6))
    return g * np.array([sx, spx, sx, spx, sigma_z, sigma_pt])


EIC_GAMMA = 275000.0 / PROTON_MASS_MEV  # 275 GeV protons
EIC_HALF_CROSSING = 0.0125              # half of the 25 mrad full crossing angle


def eic_like_ring(seed: Optional[int] = None, nint_arc: int = 4, nint_triplet: int = 8,
                  aperture_radius: float = 0.03, crab_mv=(2.0, -0.4)) -> Lattice:
    """Synthetic EIC hadron-ring-like lattice for spin tracking, 3,834 m,
    ~2,450 elements, 275 GeV protons.

    The RHIC-like ring's optics (normalised strengths do not depend on the
    energy) with one collision point: at IP1 a Lorentz boost for the 25 mrad
    full crossing angle (LBT / ILBT, theta = 12.5 mrad) around the weak-strong
    6D beam-beam map of a flat electron bunch (1.7e11 charges of opposite sign,
    sigma_x = 95 um, sigma_y = 8.5 um, sigma_z = 7 mm, 7 slices), thin crab
    cavities at 197 and 394 MHz on either side of it (the downstream pair
    with opposite voltages), no beam-beam at IP2, a beam-position marker after
    every arc quadrupole and a zero-strength orbit corrector after the
    sextupoles of every other arc cell.  IR triplet errors as in
    rhic_like_ring."""
    base = rhic_like_ring(seed=seed, nint_arc=nint_arc, nint_triplet=nint_triplet, bb=False,
                          aperture_radius=aperture_radius)
    beta = math.sqrt(1.0 - 1.0 / EIC_GAMMA / EIC_GAMMA)
    from . import lattice_design as D
    frev = beta * 299792458.0 / D.CIRC
    bx, by = 0.8, 0.072
    bb = ElementSpec("BEAMBEAM", "bb_ip1", (6, 1.7e11, -1.0, 0.007, 7, 95e-6 ** 2 / bx, bx, 0.0, 8.5e-6 ** 2 / by,
                                            by, 0.0))
    v1, v2 = crab_mv
    up = [ElementSpec("CRABRF", "crab197_u", (0.0, v1, 197e6, 0.0)),
          ElementSpec("CRABRF", "crab394_u", (0.0, v2, 394e6, 0.0))]
    down = [ElementSpec("CRABRF", "crab394_d", (0.0, -v2, 394e6, 0.0)),
            ElementSpec("CRABRF", "crab197_d", (0.0, -v1, 197e6, 0.0))]
    ip = up + [ElementSpec("LBT", "lbt_ip1", (EIC_HALF_CROSSING,)), bb,
               ElementSpec("ILBT", "ilbt_ip1", (EIC_HALF_CROSSING,))] + down
    els: List[ElementSpec] = list(ip)
    cell = 0
    for e in base.elements:
        if e.type == "RFCAV":
            h = 360 if "28" in e.name else 2520
            e = ElementSpec("RFCAV", e.name, (e.args[0], e.args[1], h * frev, e.args[3]))
        els.append(e)
        if e.type == "QUAD" and (e.name.startswith("qd_") or e.name.startswith("qf_")):
            els.append(ElementSpec("MARKER", "bpm_" + e.name, (0.0,)))
        if e.type == "SEXT" and e.name.startswith("sd_"):
            cell += 1
            if cell % 2 == 0:
                kind = "HKICKER" if cell % 4 == 0 else "VKICKER"
                els.append(ElementSpec(kind, "cor_" + e.name, (0.0, 0.0)))
    lat = Lattice("eic_like" + ("" if seed is None else f"_s{seed}"), els, EIC_GAMMA,
                  aperture_radius=aperture_radius)
    lat.meta.update({"seed": seed, "beta_star": RHIC_BETA_STAR, "emit_norm": 2.5e-6, "frev": frev,
                     "sigma_ip": math.sqrt(2.5e-6 * RHIC_BETA_STAR / (beta * EIC_GAMMA)), "spin_g": 1.7928474})
    return lat


# ---- MAD-X TFS twiss tables (the format Read_MADX_Lattice reads) ----

_TFS_KEYWORD = {"DRIFT": "DRIFT", "SBEND": "SBEND", "QUAD": "QUADRUPOLE", "SEXT": "SEXTUPOLE", "OCT": "OCTUPOLE",
                "MULT": "MULTIPOLE", "MARKER": "MARKER", "HKICKER": "HKICKER", "VKICKER": "VKICKER",
                "KICKER": "TKICKER", "RFCAV": "RFCAVITY", "BEAMBEAM": "BEAMBEAM", "BPM": "MONITOR",
                "VBPM": "VMONITOR"}


def write_madx_tfs(lat: Lattice, path: str) -> None:
    """Writes `lat` as a MAD-X-style TFS twiss table with the columns
    Read_MADX_Lattice (simtrack.cpp:13591) reads.  Strengths are written
    with 17 significant digits (exact round trip).  What the format cannot
    carry is dropped, as reading a MAD-X table would: slice counts (the
    reader's defaults apply), corrector kicks, RF voltages and beam-beam
    parameters."""
    cols = ["NAME", "KEYWORD", "S", "L", "ANGLE", "E1", "E2", "TILT"]
    for k in range(11):
        cols += [f"K{k}L", f"K{k}SL"]
    cols += ["KS"]
    rows = []
    s = 0.0
    for e in lat.elements:
        kw = _TFS_KEYWORD.get(e.type, "INSTRUMENT")
        a = e.args
        L = 0.0 if e.type in ("LBT", "ILBT", "BEAMBEAM") else float(a[0])
        angle = e1 = e2 = 0.0
        knl = [0.0] * 11
        knsl = [0.0] * 11
        if e.type == "SBEND":
            angle, e1, e2 = a[1], a[2], a[3]
        elif e.type in ("QUAD", "SEXT", "OCT"):
            order = {"QUAD": 1, "SEXT": 2, "OCT": 3}[e.type]
            knl[order], knsl[order] = a[1], a[2]
        elif e.type == "MULT":
            knl, knsl = list(a[1:12]), list(a[12:23])
        tilt = e.misalign[5] if e.misalign is not None else 0.0
        s += L
        vals = [s, L, angle, e1, e2, tilt]
        for k in range(11):
            vals += [knl[k], knsl[k]]
        vals.append(0.0)
        rows.append(f'"{e.name.upper()}" "{kw}" ' + " ".join(repr(float(v)) for v in vals))
    with open(path, "w") as f:
        f.write('@ NAME             %05s "TWISS"\n')
        f.write(f"@ LENGTH           %le {s!r}\n")
        f.write("* " + " ".join(cols) + "\n")
        f.write("$ %s %s " + " ".join(["%le"] * (len(cols) - 2)) + "\n")
        f.write("\n".join(rows) + "\n")


def specs_from_line(line: api.Line) -> List[ElementSpec]:
    """ElementSpec list describing an existing Line (for the oracles or for
    inspection): type, name, constructor arguments, slice counts, roll."""
    out = []
    mult = tuple(f"K{k}L" for k in range(11)) + tuple(f"K{k}SL" for k in range(11))
    for i in range(line.Ncell):
        e = line.Cell(i)
        t, g = e.TYPE, e.geometry()
        P = e.GetP
        setp = {}
        if t in ("DRIFT", "MARKER", "BPM", "HBPM", "VBPM"):
            args = (g["L"],)
        elif t == "SBEND":
            args = (g["L"], P("ANGLE"), P("E1"), P("E2"))
            setp = {"Nint": P("Nint")}
        elif t == "GSBEND":
            args = (g["L"], P("ANGLE"), P("K0L"), P("E1"), P("E2"))
            setp = {"Nint": P("Nint")}
        elif t in ("QUAD", "SEXT", "OCT"):
            k = {"QUAD": "1", "SEXT": "2", "OCT": "3"}[t]
            args = (g["L"], P(f"K{k}L"), P(f"K{k}SL"))
            setp = {"Nint": P("Nint")}
        elif t == "MULT":
            args = (g["L"],) + tuple(P(n) for n in mult)
            setp = {"Nint": P("Nint"), "Norder": P("Norder")}
        elif t in ("GMULT", "SBENDMULT"):
            args = (g["L"], P("ANGLE"), P("E1"), P("E2")) + tuple(P(n) for n in mult)
            setp = {"Nint": P("Nint"), "Norder": P("Norder")}
        elif t == "HKICKER":
            args = (g["L"], P("HKICK"))
        elif t == "VKICKER":
            args = (g["L"], P("VKICK"))
        elif t == "KICKER":
            args = (g["L"], P("HKICK"), P("VKICK"))
        elif t == "RFCAV":
            args = (g["L"], P("VRF"), P("FRF"), P("PHASE0"))
        elif t == "BEAMBEAM":
            args = tuple(P(n) for n in ("TREATMENT", "NP", "BBSCALE", "SIGMAL", "NSLICE", "EMITX", "BETAX", "ALFAX",
                                        "EMITY", "BETAY", "ALFAY"))
        elif t == "SOLEN":
            args = (g["L"], P("KS"))
        elif t == "PATCH":
            args = (P("DX"), P("DY"), P("DS"), P("THETA"))
        else:
            raise ValueError(f"specs_from_line: element type {t} not handled")
        mis = (g["DX"], g["DY"], g["DS"], g["DTHETA"], g["DPHI"], g["DPSI"])
        out.append(ElementSpec(t, e.NAME, tuple(float(v) for v in args), setp,
                               misalign=mis if any(v != 0.0 for v in mis) else None,
                               aperture=(g["APx"], g["APy"]) if (g["APx"], g["APy"]) != (1.0, 1.0) else None))
    return out
