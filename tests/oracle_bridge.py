"""Test-side bridge to the CPU oracles (test infrastructure only).

* RefOracle: the unmodified SimTrack source compiled with the GSL shim into
  oracle/_ref/libsimtrack_ref.so (oracle/Makefile); Lines are built with the
  reference's own constructors and tracked by its own Track().
* PortOracle: the C restatement oracle/port/simtrack_port.c compiled into
  oracle/_build/libsimtrack_port.so.

Both consume the same simtrack_b200.lattices.Lattice description the product
is built from.
"""
from __future__ import annotations

import ctypes
import math
from ctypes import POINTER, c_char_p, c_double, c_int, c_long, c_void_p
from pathlib import Path

import numpy as np

from simtrack_b200.lattices import Lattice

ROOT = Path(__file__).resolve().parents[1]
REF_SO = ROOT / "oracle" / "_ref" / "libsimtrack_ref.so"
# the same reference objects with correctly rounded asin/sin/cos/exp/pow
REF_CR_SO = ROOT / "oracle" / "_ref" / "libsimtrack_ref_cr.so"
PORT_SO = ROOT / "oracle" / "_build" / "libsimtrack_port.so"

PORT_TYPES = ["DRIFT", "MARKER", "SBEND", "GSBEND", "QUAD", "SKEWQ", "SEXT", "OCT", "MULT", "GMULT",
              "SBENDMULT", "KICKER", "HKICKER", "VKICKER", "RFCAV", "CRABRF", "CCMULT", "LBT", "ILBT", "BEAMBEAM",
              "SOLEN", "PATCH"]


def ref_source_dir() -> Path | None:
    """The reference source tree the compiled reference was built from
    (recorded by oracle/Makefile), when it is still present."""
    f = ROOT / "oracle" / "_ref" / "ref_src.txt"
    if not f.exists():
        return None
    d = Path(f.read_text().strip())
    return d if (d / "simtrack.cpp").exists() else None


def ref_available(cr: bool = False) -> bool:
    return (REF_CR_SO if cr else REF_SO).exists()


def reference_radiation_off() -> None:
    """Turn GP.radiate off in both compiled references loaded in this process
    (their globals outlive one test; a reference line built afterwards
    without RefOracle.build would otherwise track with radiation)."""
    for cr in (False, True):
        if ref_available(cr=cr):
            L = ctypes.CDLL(str(REF_CR_SO if cr else REF_SO))
            L.ref_set_radiation.argtypes = [c_int, ctypes.c_ulonglong]
            L.ref_set_radiation(0, 1324)


def port_available() -> bool:
    return PORT_SO.exists()


class RefOracle:
    """The compiled reference.  cr=True loads the variant whose transcendentals
    are correctly rounded (oracle/crlibm_shim.cpp)."""

    def __init__(self, cr: bool = False):
        L = ctypes.CDLL(str(REF_CR_SO if cr else REF_SO))
        L.ref_line_new.restype = c_void_p
        L.ref_line_free.argtypes = [c_void_p]
        L.ref_line_ncell.restype = c_long
        L.ref_line_ncell.argtypes = [c_void_p]
        L.ref_line_append.argtypes = [c_void_p, c_char_p, c_char_p, POINTER(c_double), c_int]
        L.ref_line_setp.argtypes = [c_void_p, c_long, c_char_p, c_double]
        L.ref_line_getp.argtypes = [c_void_p, c_long, c_char_p]
        L.ref_line_getp.restype = c_double
        L.ref_line_set_misalign.argtypes = [c_void_p, c_long] + [c_double] * 6
        L.ref_line_set_aperture.argtypes = [c_void_p, c_long, c_double, c_double]
        L.ref_set_ref_energy.argtypes = [c_double] * 4
        L.ref_set_flags.argtypes = [c_int, c_int]
        L.ref_get_gp.argtypes = [POINTER(c_double)]
        L.ref_track.argtypes = [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_int), POINTER(c_int),
                                POINTER(c_int)]
        L.ref_track_circ.argtypes = [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_int),
                                     POINTER(c_int), POINTER(c_int)]
        L.ref_track_dump.argtypes = [c_void_p, POINTER(c_double), c_int, c_double, POINTER(c_double),
                                     POINTER(c_int), POINTER(c_int), POINTER(c_int)]
        L.ref_pinv.argtypes = [c_double]
        L.ref_pinv.restype = c_double
        L.ref_pass.argtypes = [c_void_p, c_long, POINTER(c_double)]
        L.ref_track_spin.argtypes = [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_int), POINTER(c_int),
                                     POINTER(c_int)]
        L.ref_line_read_madx.argtypes = [ctypes.c_char_p]
        L.ref_line_read_madx.restype = c_void_p
        L.ref_line_read_bmad.argtypes = [ctypes.c_char_p]
        L.ref_line_read_bmad.restype = c_void_p
        L.ref_track_tbt.argtypes = [c_void_p, POINTER(c_double), c_int, POINTER(c_double), POINTER(c_int),
                                    POINTER(c_int), POINTER(c_int)]
        L.ref_cal_dz0.argtypes = [c_void_p, POINTER(c_double), POINTER(c_double)]
        L.ref_track_wrt_onmom.argtypes = [c_void_p, POINTER(c_double), c_long, POINTER(c_double), c_int,
                                          POINTER(c_int), POINTER(c_int), POINTER(c_int)]
        L.ref_track_tbt_spin_bpm.argtypes = [c_void_p, POINTER(c_double), c_int, POINTER(c_double), c_int,
                                             POINTER(c_int), POINTER(c_int), POINTER(c_int)]
        L.ref_track_tbt_bpm.argtypes = [c_void_p, POINTER(c_double), c_int, POINTER(c_double), c_int, POINTER(c_int),
                                        POINTER(c_int), POINTER(c_int)]
        L.ref_track_tbt_spin.argtypes = [c_void_p, POINTER(c_double), c_int, POINTER(c_double), POINTER(c_int),
                                         POINTER(c_int), POINTER(c_int)]
        L.ref_track_tbt_fma.argtypes = [c_void_p, c_double, c_double, c_double, c_double, c_double]
        L.ref_track_tbt_lyapunov.argtypes = [c_void_p, c_double, c_double, c_double]
        L.ref_track_da_driver.argtypes = [c_void_p, c_int, c_int, c_double, c_double, c_double, ctypes.c_char_p]
        L.ref_line_elem.argtypes = [c_void_p, c_long, ctypes.c_char_p, ctypes.c_char_p, c_int, POINTER(c_double)]
        L.ref_cal_orbit.argtypes = [c_void_p, c_double, POINTER(c_double)]
        L.ref_track_da.argtypes = [c_void_p, c_int, c_double, c_double, c_double, ctypes.c_char_p]
        L.ref_track_radial.argtypes = [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_int), POINTER(c_int),
                                       POINTER(c_int)]
        L.ref_track_spin_dump.argtypes = [c_void_p, POINTER(c_double), c_int, POINTER(c_double), POINTER(c_int),
                                          POINTER(c_int), POINTER(c_int)]
        L.ref_set_spin_g.argtypes = [c_double]
        L.ref_fine_tune.argtypes = [c_int, POINTER(c_double), POINTER(c_double), c_double, c_double]
        L.ref_fine_tune.restype = c_double
        L.ref_bb4d_soft_gaussian.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                             c_double, c_double, c_double, c_double]
        L.ref_bb4d_pic.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                   c_double, c_double, c_double, c_double]
        L.ref_lumi_pic_4d.argtypes = [c_double, c_int, c_double, c_int, POINTER(c_double), POINTER(c_double), c_int,
                                      c_double]
        L.ref_lumi_pic_4d.restype = c_double
        L.ref_green_function.argtypes = [c_double, c_double, c_int, c_int, c_double, c_double, POINTER(c_double),
                                         POINTER(c_double)]
        L.ref_bb4d_pic_nonoffset.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                             c_double, c_double, c_double, c_double, c_int, c_int, c_double, c_double,
                                             POINTER(c_double), POINTER(c_double)]
        L.ref_bb6d_pic.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                   c_double, c_double, c_double, c_double, c_int, c_int]
        L.ref_lumi_pic_6d.argtypes = [c_double, c_int, c_double, c_int, c_int, c_int, POINTER(c_double),
                                      POINTER(c_double), c_double, c_double, c_double, c_double, c_int, c_double]
        L.ref_lumi_pic_6d.restype = c_double
        L.ref_bb6d_pic_nonoffset.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                             c_double, c_double, c_double, c_double, c_int, c_int, POINTER(c_double),
                                             POINTER(c_double), c_int, c_int, c_double, c_double, POINTER(c_double),
                                             POINTER(c_double)]
        L.ref_lumi_pic_6d_angle.argtypes = [c_double, c_int, c_double, c_int, c_double, c_int, c_int,
                                            POINTER(c_double), POINTER(c_double), c_double, c_double, c_double,
                                            c_double, c_int, c_double]
        L.ref_lumi_pic_6d_angle.restype = c_double
        L.ref_bb6d_pic_interpolation.argtypes = L.ref_bb6d_pic_nonoffset.argtypes
        L.ref_bb6d_soft_gaussian.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int, POINTER(c_double),
                                             c_double, c_double, c_double, c_double, c_int, c_int]
        L.ref_bb6d_soft_gaussian_zb.argtypes = [c_double, c_int, POINTER(c_double), c_double, c_int,
                                                POINTER(c_double), c_double, c_double, c_double, c_double, c_int,
                                                c_int, POINTER(c_double), POINTER(c_double)]
        L.ref_set_radiation.argtypes = [c_int, ctypes.c_ulonglong]
        L.ref_cal_srloss.argtypes = [c_void_p, c_int]
        L.ref_cal_srloss.restype = c_double
        L.ref_cal_srloss_particle.argtypes = [c_void_p, c_void_p]
        L.ref_cal_srloss_particle.restype = c_double
        L.ref_rng_id_base.argtypes = [c_long]
        L.ref_rng_stream.argtypes = [ctypes.c_ulonglong] * 3
        L.ref_rng_stream.restype = c_double
        self.L = L
        self.line = None
        self.nelem = 0

    def build(self, lat: Lattice) -> None:
        L = self.L
        L.ref_set_ref_energy(lat.gamma, lat.E0, lat.Q, lat.A)
        L.ref_set_flags(0, int(lat.quad_fringe))
        if getattr(lat, "radiate", False):
            L.ref_set_radiation(1, int(lat.radiation_seed))
        L.ref_rng_id_base(0)
        if self.line:
            L.ref_line_free(self.line)
        self.line = L.ref_line_new()
        for i, e in enumerate(lat.elements):
            args = (c_double * len(e.args))(*e.args)
            rc = L.ref_line_append(self.line, e.type.encode(), e.name.encode(), args, len(e.args))
            assert rc == 0, f"reference harness rejected {e.type}"
            for k, v in e.setp.items():
                L.ref_line_setp(self.line, i, k.encode(), float(v))
            if e.misalign is not None:
                L.ref_line_set_misalign(self.line, i, *e.misalign)
            if e.aperture is not None:
                L.ref_line_set_aperture(self.line, i, *e.aperture)
        self.nelem = int(L.ref_line_ncell(self.line))
        self.radius = lat.aperture_radius

    def gp(self):
        out = (c_double * 7)()
        self.L.ref_get_gp(out)
        return list(out)

    def track(self, x: np.ndarray, nturn: int, radius: float | None = None):
        """Returns (x_out, stable, lost_turn, lost_post); x is (n,6)."""
        radius = self.radius if radius is None else radius
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        P = lambda a, t: a.ctypes.data_as(POINTER(t))
        if radius > 0:
            self.L.ref_track_circ(self.line, P(x, c_double), n, nturn, radius, P(st, c_int), P(lt, c_int), P(lp, c_int))
        else:
            self.L.ref_track(self.line, P(x, c_double), n, nturn, P(st, c_int), P(lt, c_int), P(lp, c_int))
        return x, st, lt, lp

    def track_dump(self, x0, nturn: int, radius: float | None = None):
        radius = self.radius if radius is None else radius
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        dump = np.full((nturn, self.nelem, 6), np.nan)
        st, lt, lp = c_int(), c_int(), c_int()
        self.L.ref_track_dump(self.line, x.ctypes.data_as(POINTER(c_double)), nturn, radius,
                              dump.ctypes.data_as(POINTER(c_double)), ctypes.byref(st), ctypes.byref(lt),
                              ctypes.byref(lp))
        return x, st.value, lt.value, lp.value, dump

    def track_spin(self, x9: np.ndarray, nturn: int):
        """Track_Spin over AoS x[n, 9] (copied); returns (x, stable, lost_turn, lost_post)."""
        x = np.ascontiguousarray(x9, dtype=np.float64).copy()
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        P = POINTER
        self.L.ref_track_spin(self.line, x.ctypes.data_as(P(c_double)), n, nturn, st.ctypes.data_as(P(c_int)),
                              lt.ctypes.data_as(P(c_int)), lp.ctypes.data_as(P(c_int)))
        return x, st, lt, lp

    def read_madx(self, path: str) -> None:
        """Replaces the line by the reference's Read_MADX_Lattice of `path` (must exist)."""
        if self.line:
            self.L.ref_line_free(self.line)
        self.line = self.L.ref_line_read_madx(str(path).encode())
        self.nelem = int(self.L.ref_line_ncell(self.line))
        self.radius = 0.0

    def read_bmad(self, path: str) -> None:
        """Replaces the line by the reference's Read_BMAD_Lattice of `path`
        (must exist and hold no row with a non-numeric S column)."""
        if self.line:
            self.L.ref_line_free(self.line)
        self.line = self.L.ref_line_read_bmad(str(path).encode())
        self.nelem = int(self.L.ref_line_ncell(self.line))
        self.radius = 0.0

    def track_tbt(self, x0, nturn: int, stable: int = 1):
        """Track_tbt of one particle (Track_tbt_spin for x0 of 9): (x, stable,
        lost_turn, lost_post, x_tbt[nturn, 6 or 9]) with NaN in the turns it did
        not record."""
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        tbt = np.full((nturn, len(x)), np.nan)
        st, lt, lp = c_int(stable), c_int(0), c_int(0)
        fn = self.L.ref_track_tbt_spin if len(x) == 9 else self.L.ref_track_tbt
        fn(self.line, x.ctypes.data_as(POINTER(c_double)), nturn, tbt.ctypes.data_as(POINTER(c_double)),
           ctypes.byref(st), ctypes.byref(lt), ctypes.byref(lp))
        return x, st.value, lt.value, lp.value, tbt

    def track_tbt_bpm(self, x0, nturn: int, bpm_index: int):
        """Track_tbt with a BPM index (Track_tbt_spin for x0 of 9): (x, stable,
        lost_turn, lost_post, x_tbt[nturn, 6 or 9]), NaN where not recorded."""
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        tbt = np.full((nturn, len(x)), np.nan)
        st, lt, lp = c_int(1), c_int(0), c_int(0)
        fn = self.L.ref_track_tbt_spin_bpm if len(x) == 9 else self.L.ref_track_tbt_bpm
        fn(self.line, x.ctypes.data_as(POINTER(c_double)), nturn, tbt.ctypes.data_as(POINTER(c_double)), bpm_index,
           ctypes.byref(st), ctypes.byref(lt), ctypes.byref(lp))
        return x, st.value, lt.value, lp.value, tbt

    def element(self, i: int):
        """(TYPE, NAME, {L, S, DX, DY, DS, DTHETA, DPHI, DPSI, APx, APy}) of element i."""
        t = ctypes.create_string_buffer(256)
        nm = ctypes.create_string_buffer(256)
        g = (c_double * 10)()
        self.L.ref_line_elem(self.line, i, t, nm, 256, g)
        keys = ("L", "S", "DX", "DY", "DS", "DTHETA", "DPHI", "DPSI", "APx", "APy")
        return t.value.decode(), nm.value.decode(), {k: g[j] for j, k in enumerate(keys)}

    def getp(self, i: int, name: str) -> float:
        return self.L.ref_line_getp(self.line, i, name.encode())

    def cal_orbit(self, deltap: float) -> np.ndarray:
        out = np.empty((self.nelem, 6))
        self.L.ref_cal_orbit(self.line, deltap, out.ctypes.data_as(POINTER(c_double)))
        return out

    def track_da(self, nturn: int, deltap0: float, sigmax0: float, sigmay0: float, filename: str) -> None:
        self.L.ref_track_da(self.line, nturn, deltap0, sigmax0, sigmay0, str(filename).encode())

    def track_radial(self, x: np.ndarray, nturn: int):
        """Track_Radial over AoS x[n, 6] (copied); returns (x, stable, lost_turn, lost_post)."""
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        P = POINTER
        self.L.ref_track_radial(self.line, x.ctypes.data_as(P(c_double)), n, nturn, st.ctypes.data_as(P(c_int)),
                                lt.ctypes.data_as(P(c_int)), lp.ctypes.data_as(P(c_int)))
        return x, st, lt, lp

    def track_spin_dump(self, x0, nturn: int):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        dump = np.full((nturn, self.nelem, 9), np.nan)
        st, lt, lp = c_int(), c_int(), c_int()
        self.L.ref_track_spin_dump(self.line, x.ctypes.data_as(POINTER(c_double)), nturn,
                                   dump.ctypes.data_as(POINTER(c_double)), ctypes.byref(st), ctypes.byref(lt),
                                   ctypes.byref(lp))
        return x, st.value, lt.value, lp.value, dump

    def fine_tune(self, x, px=None, lo: float = 0.0, hi: float = 0.5) -> float:
        """FineTuneFinder (x-only, or the x/px overload when px is given)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = None if px is None else np.ascontiguousarray(px, dtype=np.float64)
        return self.L.ref_fine_tune(len(x), x.ctypes.data_as(POINTER(c_double)),
                                    None if p is None else p.ctypes.data_as(POINTER(c_double)), lo, hi)

    def pinv(self, p: float) -> float:
        return self.L.ref_pinv(p)


class PortElem(ctypes.Structure):
    _fields_ = [("type", c_int), ("nint", c_int), ("norder", c_int), ("nslice", c_int), ("treatment", c_int),
                ("pad", c_int), ("L", c_double), ("p", c_double * 16), ("knl", c_double * 11),
                ("knsl", c_double * 11), ("dx", c_double), ("dy", c_double), ("ds", c_double),
                ("dtheta", c_double), ("dphi", c_double), ("dpsi", c_double), ("apx", c_double), ("apy", c_double)]


class PortGP(ctypes.Structure):
    _fields_ = [("gamma", c_double), ("beta", c_double), ("energy", c_double), ("brho", c_double),
                ("G", c_double), ("Q", c_double), ("quad_fringe", c_int), ("pad", c_int),
                ("m0", c_double), ("q", c_double), ("p", c_double)]


def _norder(knl, knsl):
    for i in range(10):
        if knl[10 - i] != 0.0 or knsl[10 - i] != 0.0:
            return 10 - i
    return 1


class PortOracle:
    def __init__(self):
        L = ctypes.CDLL(str(PORT_SO))
        L.port_track.argtypes = [POINTER(PortElem), c_long, POINTER(PortGP), POINTER(c_double), c_long, c_int,
                                 c_double, POINTER(c_int), POINTER(c_int), POINTER(c_int)]
        L.port_track_dump.argtypes = [POINTER(PortElem), c_long, POINTER(PortGP), POINTER(c_double), c_int,
                                      c_double, POINTER(c_double), POINTER(c_int), POINTER(c_int), POINTER(c_int)]
        L.port_cerrf.argtypes = [c_double, c_double, POINTER(c_double), POINTER(c_double)]
        L.port_fine_tune.argtypes = [c_int, POINTER(c_double), POINTER(c_double), c_double, c_double]
        L.port_fine_tune.restype = c_double
        self.L = L

    def build(self, lat: Lattice) -> None:
        # Reference particle as Set_RefPartEnergy computes it (simtrack.cpp:87-108).
        gamma, E0, Q = lat.gamma, lat.E0, lat.Q
        beta = math.sqrt(1.0 - 1.0 / gamma / gamma)
        energy = gamma * E0
        brho = 3.33564095198 * beta * (energy / 1000) / int(Q)
        # m0, q, p as Set_RefPartEnergy computes them (the solenoid needs them)
        m0 = E0 * 1.0e6 * 1.6021765e-19 / 299792458. / 299792458.
        q = Q * 1.6021765e-19
        p = energy * beta * 1.0e6 * 1.6021765e-19 / 299792458.
        self.gp = PortGP(gamma, beta, energy, brho, 1.7928474, float(int(Q)), int(lat.quad_fringe), 0, m0, q, p)
        n = len(lat.elements)
        arr = (PortElem * n)()
        for i, e in enumerate(lat.elements):
            pe = arr[i]
            # monitors track as markers: a drift without misalignment (BPM::Pass 10497)
            pe.type = PORT_TYPES.index("MARKER" if e.type in ("BPM", "HBPM", "VBPM") else e.type)
            a = list(e.args)
            pe.apx, pe.apy = (1.0, 1.0) if e.aperture is None else e.aperture
            if e.misalign is not None:
                pe.dx, pe.dy, pe.ds, pe.dtheta, pe.dphi, pe.dpsi = e.misalign
            t = e.type
            if t in ("LBT", "ILBT"):
                pe.L = 0.0
                pe.p[0] = a[0]
            elif t == "BEAMBEAM":
                pe.L = 0.0
                pe.treatment = int(a[0])
                pe.nslice = int(a[4])
                vals = [a[1], a[2], a[3], a[5], a[6], a[7], a[8], a[9], a[10]]
                for k, v in enumerate(vals):
                    pe.p[k] = v
            elif t == "MULT":
                pe.L = a[0]
                for k in range(11):
                    pe.knl[k] = a[1 + k]
                    pe.knsl[k] = a[12 + k]
                pe.norder = _norder(a[1:12], a[12:23])
                pe.nint = int(a[0] / 0.05) + 1
            elif t == "PATCH":
                pe.L = a[2]  # PATCH: L = DS (simtrack.cpp:12266)
                for k, v in enumerate(a):
                    pe.p[k] = v
            elif t in ("GMULT", "SBENDMULT"):
                pe.L = a[0]
                pe.p[0], pe.p[1], pe.p[2] = a[1], a[2], a[3]
                for k in range(11):
                    pe.knl[k] = a[4 + k]
                    pe.knsl[k] = a[15 + k]
                pe.norder = _norder(a[4:15], a[15:26])
                pe.nint = int(a[0] / 0.25) + 1
            else:
                pe.L = a[0]
                for k, v in enumerate(a[1:]):
                    pe.p[k] = v
                if t in ("QUAD", "SKEWQ", "SEXT", "OCT"):
                    pe.nint = int(a[0] / 0.05) + 1
                elif t in ("SBEND", "GSBEND"):
                    pe.nint = int(a[0] / 0.25) + 1
            for k, v in e.setp.items():
                if k == "Nint":
                    pe.nint = int(v)
                elif k == "Norder":
                    pe.norder = int(v)
                else:
                    raise NotImplementedError(f"port bridge: SetP({k})")
        self.elems = arr
        self.nelem = n
        self.radius = lat.aperture_radius

    def track(self, x: np.ndarray, nturn: int, radius: float | None = None):
        radius = self.radius if radius is None else radius
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        P = lambda a, t: a.ctypes.data_as(POINTER(t))
        self.L.port_track(self.elems, self.nelem, ctypes.byref(self.gp), P(x, c_double), n, nturn, radius,
                          P(st, c_int), P(lt, c_int), P(lp, c_int))
        return x, st, lt, lp

    def track_dump(self, x0, nturn: int, radius: float | None = None):
        radius = self.radius if radius is None else radius
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        dump = np.full((nturn, self.nelem, 6), np.nan)
        st, lt, lp = c_int(), c_int(), c_int()
        self.L.port_track_dump(self.elems, self.nelem, ctypes.byref(self.gp), x.ctypes.data_as(POINTER(c_double)),
                               nturn, radius, dump.ctypes.data_as(POINTER(c_double)), ctypes.byref(st),
                               ctypes.byref(lt), ctypes.byref(lp))
        return x, st.value, lt.value, lp.value, dump

    def fine_tune(self, x, px=None, lo: float = 0.0, hi: float = 0.5) -> float:
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = None if px is None else np.ascontiguousarray(px, dtype=np.float64)
        return self.L.port_fine_tune(len(x), x.ctypes.data_as(POINTER(c_double)),
                                     None if p is None else p.ctypes.data_as(POINTER(c_double)), lo, hi)

    def cerrf(self, x: float, y: float):
        wx, wy = c_double(), c_double()
        self.L.port_cerrf(x, y, ctypes.byref(wx), ctypes.byref(wy))
        return wx.value, wy.value


def _ref_track_worker(args):
    lat, x, nturn, cr, spin, first = args
    o = RefOracle(cr=cr)
    o.build(lat)
    o.L.ref_rng_id_base(int(first))  # particle ids of the radiation deviate streams
    return o.track_spin(x, nturn) if spin else o.track(x, nturn)


def ref_track_parallel(lat: Lattice, x: np.ndarray, nturn: int, cr: bool = False, spin: bool = False,
                       procs: int = 0):
    """The compiled reference's Track() (Track_Spin for spin=True) over the
    rows of x split into contiguous ranges, one spawned process per range
    (processes, because the reference keeps the turn counter in a global).
    Returns (x_out, stable, lost_turn, lost_post) in the input order."""
    import multiprocessing as mp
    import os
    procs = procs or os.cpu_count() or 1
    procs = max(1, min(procs, len(x)))
    chunks = np.array_split(np.ascontiguousarray(x, dtype=np.float64), procs)
    firsts = np.cumsum([0] + [len(c) for c in chunks[:-1]])
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ref_track_worker, [(lat, c, nturn, cr, spin, f) for c, f in zip(chunks, firsts)])
    return tuple(np.concatenate([r[k] for r in res]) for k in range(4))
