"""Python mirror of SimTrack's construction and tracking interface.

Names, argument order and meaning follow simtrack.h: element classes are
created as ``QUAD(name, L, K1L, K1SL)``, tuned with ``SetP``, appended to a
``Line`` and tracked with ``Track``.  Everything runs through the C ABI of
the native library; tracking executes on the GPU.  Errors raise
SimTrackError instead of terminating the process (the reference prints and
calls exit(), e.g. simtrack.cpp:8653-8685).
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_long, c_void_p
from typing import Sequence

import numpy as np

from ._native import SimTrackError, check, lib

__all__ = [
    "Set_RefPartEnergy", "Set_Spin_G", "Set_Flags", "GP", "Element", "Line", "Table", "Track", "Track_Batch",
    "DRIFT", "MARKER", "SBEND", "GSBEND", "QUAD", "SKEWQ", "SEXT", "OCT", "MULT", "GMULT", "SBENDMULT",
    "KICKER", "HKICKER", "VKICKER", "RFCAV", "CRABRF", "CCMULT", "LBT", "ILBT", "BEAMBEAM",
    "Set_Radiation", "BeamBeam4D_SoftGaussian", "BeamBeam6D_SoftGaussian",
]


def Set_RefPartEnergy(gamma: float, E0: float, Q: float, A: float) -> None:
    """Set_RefPartEnergy (simtrack.cpp:87-108): reference particle gamma, rest energy [MeV], charge, nucleons."""
    check(lib().stb_set_ref_energy(gamma, E0, Q, A))


def Set_Spin_G(g: float) -> None:
    """Set_Spin_G (simtrack.cpp:110-115)."""
    check(lib().stb_set_spin_g(g))


def Set_Flags(h_expand: bool = False, quad_fringe: bool = False) -> None:
    """GP.H_expand / GP.quad_fringe (simtrack.h:62-66)."""
    check(lib().stb_set_flags(int(h_expand), int(quad_fringe)))


def Set_Radiation(radiate: bool = False, seed: int = 1324) -> None:
    """GP.radiate (simtrack.h:57) for tables created afterwards: radiation in
    the sector bends (radiate1, with quantum excitation) and GMULT/SBENDMULT
    (radiate).  `seed` keys the quantum-excitation deviates (the reference
    seeds its GSL stream with 1324, simtrack.cpp:328)."""
    check(lib().stb_set_radiation(int(radiate), int(seed)))


def _bunch(x) -> np.ndarray:
    b = np.asarray(x)
    if b.dtype != np.float64 or not b.flags.c_contiguous or b.ndim != 2 or b.shape[1] != 6:
        raise ValueError("a bunch is a C-contiguous float64 array of shape (n, 6), updated in place")
    return b


def BeamBeam4D_SoftGaussian(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, gamma1: float, gamma2: float,
                            bbscale1: float, bbscale2: float, device: int = 0) -> None:
    """BeamBeam4D_SoftGaussian (simtrack.cpp:22846-22872) on the GPU: the two
    macro-particle bunches (numpy (n, 6) float64, updated in place) kick each
    other as soft Gaussians."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    check(lib().stb_bb4d_soft_gaussian_host(Np1, len(b1), P(b1), Np2, len(b2), P(b2), gamma1, gamma2, bbscale1,
                                            bbscale2, device))


def BeamBeam4D_PIC(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, gamma1: float, gamma2: float,
                   bbscale1: float, bbscale2: float, device: int = 0) -> None:
    """BeamBeam4D_PIC (simtrack.cpp:23286-23378) on the GPU: each bunch's
    charge on a 64 x 64 grid, the potential by FFT convolution with the
    integrated Green function, the field kicking the other bunch (numpy
    (n, 6) float64, updated in place)."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    check(lib().stb_bb4d_pic_host(Np1, len(b1), P(b1), Np2, len(b2), P(b2), gamma1, gamma2, bbscale1, bbscale2,
                                  device))


def BeamBeam6D_PIC(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, gamma1: float, gamma2: float,
                   bbscale1: float, bbscale2: float, Nslice1: int, Nslice2: int, device: int = 0) -> None:
    """BeamBeam6D_PIC (simtrack.cpp:23380-23615) on the GPU: both bunches
    (numpy (n, 6) float64, updated in place and reordered by z as in the
    reference) sliced, each slice pair colliding as BeamBeam4D_PIC."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    check(lib().stb_bb6d_pic_host(Np1, len(b1), P(b1), Np2, len(b2), P(b2), gamma1, gamma2, bbscale1, bbscale2,
                                  int(Nslice1), int(Nslice2), device))


def Lumi_Cal_PIC_4D(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, Ncoll: int, freq: float,
                    device: int = 0) -> float:
    """Lumi_Cal_PIC_4D (simtrack.cpp:23617-23701) on the GPU: the two
    bunches' (numpy (n, 6) float64) charge overlap on one 64 x 64 grid,
    Ncoll collisions per turn at revolution frequency freq (cm^-2 s^-1)."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    out = c_double()
    check(lib().stb_lumi_pic_4d_host(Np1, len(b1), Np2, len(b2), P(b1), P(b2), int(Ncoll), freq, device, byref(out)))
    return out.value


def Lumi_Cal_PIC_6D(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, Nslice1: int, Nslice2: int,
                    gamma1: float, gamma2: float, bbscale1: float, bbscale2: float, Ncoll: int, freq: float,
                    device: int = 0) -> float:
    """Lumi_Cal_PIC_6D (simtrack.cpp:23703-23944) on the GPU: the sliced
    luminosity, the slice pairs colliding as soft Gaussians as they pass
    (both bunches, numpy (n, 6) float64, updated in place and reordered by z
    as in the reference)."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    out = c_double()
    check(lib().stb_lumi_pic_6d_host(Np1, len(b1), Np2, len(b2), int(Nslice1), int(Nslice2), P(b1), P(b2), gamma1,
                                     gamma2, bbscale1, bbscale2, int(Ncoll), freq, device, byref(out)))
    return out.value


def BeamBeam6D_SoftGaussian(Np1: float, x1: np.ndarray, Np2: float, x2: np.ndarray, gamma1: float, gamma2: float,
                            bbscale1: float, bbscale2: float, Nslice1: int, Nslice2: int, zb1=None, zb2=None,
                            device: int = 0) -> None:
    """BeamBeam6D_SoftGaussian on the GPU: without zb1/zb2 the sorted-slice
    form (simtrack.cpp:22874-23132; both bunches come back ordered by z,
    largest first), with them the slice-boundary form (23134-23283, zb of
    Nslice + 1 decreasing values).  Bunches: numpy (n, 6) float64, in place."""
    b1, b2 = _bunch(x1), _bunch(x2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    if zb1 is None and zb2 is None:
        check(lib().stb_bb6d_soft_gaussian_host(Np1, len(b1), P(b1), Np2, len(b2), P(b2), gamma1, gamma2, bbscale1,
                                                bbscale2, Nslice1, Nslice2, device))
        return
    z1 = np.ascontiguousarray(zb1, dtype=np.float64)
    z2 = np.ascontiguousarray(zb2, dtype=np.float64)
    if z1.shape != (Nslice1 + 1,) or z2.shape != (Nslice2 + 1,):
        raise ValueError("zb1 and zb2 need Nslice + 1 boundaries each")
    check(lib().stb_bb6d_soft_gaussian_zb_host(Np1, len(b1), P(b1), Np2, len(b2), P(b2), gamma1, gamma2, bbscale1,
                                               bbscale2, Nslice1, Nslice2, P(z1), P(z2), device))


def GP() -> dict:
    """Snapshot of the reference-particle globals."""
    out = (c_double * 8)()
    check(lib().stb_get_ref(out))
    keys = ["gamma", "beta", "energy", "brho", "Q", "energy0", "G", "p"]
    return dict(zip(keys, list(out)))


class Element:
    """An element handle.  Owned by the Python object until appended to a Line."""

    def __init__(self, type_: str, name: str, args: Sequence[float]):
        arr = (c_double * max(len(args), 1))(*[float(a) for a in args])
        h = c_void_p()
        check(lib().stb_element_new(type_.encode(), name.encode(), arr, len(args), byref(h)))
        self._h = h
        self._owned = True

    @classmethod
    def _borrow(cls, handle: c_void_p) -> "Element":
        e = cls.__new__(cls)
        e._h = handle
        e._owned = False
        return e

    @property
    def TYPE(self) -> str:
        buf = ctypes.create_string_buffer(32)
        check(lib().stb_element_type(self._h, buf, 32))
        return buf.value.decode()

    def SetP(self, name: str, value: float) -> None:
        check(lib().stb_element_setp(self._h, name.encode(), float(value)))

    def GetP(self, name: str) -> float:
        v = c_double()
        check(lib().stb_element_getp(self._h, name.encode(), byref(v)))
        return v.value

    @property
    def NAME(self) -> str:
        buf = ctypes.create_string_buffer(256)
        check(lib().stb_element_name(self._h, buf, 256))
        return buf.value.decode()

    def geometry(self) -> dict:
        """Public fields L, S, DX, DY, DS, DTHETA, DPHI, DPSI, APx, APy."""
        out = (c_double * 10)()
        check(lib().stb_element_geometry(self._h, out))
        keys = ("L", "S", "DX", "DY", "DS", "DTHETA", "DPHI", "DPSI", "APx", "APy")
        return {k: out[i] for i, k in enumerate(keys)}

    def set_misalignment(self, dx=0., dy=0., ds=0., dtheta=0., dphi=0., dpsi=0.) -> None:
        """Element::DX/DY/DS/DTHETA/DPHI/DPSI (simtrack.h:388-389)."""
        check(lib().stb_element_set_misalign(self._h, dx, dy, ds, dtheta, dphi, dpsi))

    def set_aperture(self, apx: float, apy: float) -> None:
        """Element::APx/APy (simtrack.h:394)."""
        check(lib().stb_element_set_aperture(self._h, apx, apy))

    def __del__(self):
        try:
            if getattr(self, "_owned", False) and self._h:
                lib().stb_element_free(self._h)
        except Exception:
            pass


def _mk(type_):
    def ctor(name, *args):
        return Element(type_, name, args)
    ctor.__name__ = type_
    ctor.__doc__ = f"new {type_}(name, ...) (simtrack.h element class {type_})"
    return ctor


DRIFT = _mk("DRIFT")
MARKER = _mk("MARKER")
SBEND = _mk("SBEND")
GSBEND = _mk("GSBEND")
QUAD = _mk("QUAD")
SKEWQ = _mk("SKEWQ")
SEXT = _mk("SEXT")
OCT = _mk("OCT")
KICKER = _mk("KICKER")
HKICKER = _mk("HKICKER")
VKICKER = _mk("VKICKER")
RFCAV = _mk("RFCAV")
CRABRF = _mk("CRABRF")
CCMULT = _mk("CCMULT")
LBT = _mk("LBT")
ILBT = _mk("ILBT")


def MULT(name, L, knl, knsl):
    """new MULT(name, L, KNL[11], KNSL[11]) (simtrack.h:527-538)."""
    return Element("MULT", name, [L, *_pad11(knl), *_pad11(knsl)])


def GMULT(name, L, angle, e1, e2, knl, knsl):
    return Element("GMULT", name, [L, angle, e1, e2, *_pad11(knl), *_pad11(knsl)])


def SBENDMULT(name, L, angle, e1, e2, knl, knsl):
    return Element("SBENDMULT", name, [L, angle, e1, e2, *_pad11(knl), *_pad11(knsl)])


def BEAMBEAM(name, treatment, np_, bbscale, sigmal, nslice, emitx, betax, alfax, emity, betay, alfay):
    """new BEAMBEAM(...) (simtrack.h:842-855); emittances are un-normalised rms."""
    return Element("BEAMBEAM", name, [treatment, np_, bbscale, sigmal, nslice, emitx, betax, alfax,
                                      emity, betay, alfay])


def _pad11(v):
    v = [float(a) for a in v]
    if len(v) > 11:
        raise SimTrackError(-1, "at most 11 multipole coefficients")
    return v + [0.0] * (11 - len(v))


class Line:
    """Line (simtrack.h:1067-1100).  Appended elements become owned by the line."""

    def __init__(self):
        h = c_void_p()
        check(lib().stb_line_new(byref(h)))
        self._h = h

    def Append(self, e: Element) -> None:
        check(lib().stb_line_append(self._h, e._h))
        e._owned = False

    def Insert(self, i: int, e: Element) -> None:
        check(lib().stb_line_insert(self._h, i, e._h))
        e._owned = False

    def Delete(self, i: int) -> None:
        check(lib().stb_line_delete(self._h, i))

    def Replace(self, i: int, e: Element) -> None:
        check(lib().stb_line_replace(self._h, i, e._h))
        e._owned = False

    def Rewind(self, i: int) -> None:
        check(lib().stb_line_rewind(self._h, i))

    def Invert(self) -> None:
        check(lib().stb_line_invert(self._h))

    @property
    def Ncell(self) -> int:
        return int(lib().stb_line_ncell(self._h))

    @property
    def Length(self) -> float:
        return float(lib().stb_line_length(self._h))

    def read_madx(self, path: str) -> None:
        """Read_MADX_Lattice (simtrack.cpp:13591-13791): appends the elements of a MAD-X TFS table."""
        check(lib().stb_line_read_madx(self._h, str(path).encode()))

    def read_bmad(self, path: str) -> None:
        """Read_BMAD_Lattice (simtrack.cpp:14054-14244): appends the elements of a Bmad lattice table."""
        check(lib().stb_line_read_bmad(self._h, str(path).encode()))

    def Cell(self, i: int) -> Element:
        h = c_void_p()
        check(lib().stb_line_cell(self._h, i, byref(h)))
        return Element._borrow(h)

    def __len__(self):
        return self.Ncell

    def __del__(self):
        try:
            if self._h:
                lib().stb_line_free(self._h)
        except Exception:
            pass


NUM_VARIANTS = 18
NUM_SCAN_VARIANTS = 9


def _check_device_arrays(coords, lost_turn, lost_elem, n: int, device: int, ncoord: int = 6) -> None:
    """Rejects device buffers the C entry points cannot check themselves:
    `ncoord` contiguous CUDA float64 arrays of at least n entries and two
    contiguous CUDA int32 arrays of at least n entries, all on `device`."""
    import torch
    if len(coords) != ncoord:
        raise ValueError(f"expected {ncoord} coordinate arrays, got {len(coords)}")

    def ok(t, dtype, what):
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{what} must be a torch tensor")
        if t.device.type != "cuda" or t.device.index != device:
            raise ValueError(f"{what} must be on cuda:{device}, not {t.device}")
        if t.dtype != dtype:
            raise ValueError(f"{what} must be {dtype}, not {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"{what} must be contiguous")
        if t.numel() < n:
            raise ValueError(f"{what} holds {t.numel()} entries, {n} needed")

    for k, c in enumerate(coords):
        ok(c, torch.float64, f"coordinate array {k}")
    ok(lost_turn, torch.int32, "lost_turn")
    ok(lost_elem, torch.int32, "lost_elem")


NUM_SPIN_VARIANTS = 12


def spin_variant_name(v: int) -> str:
    buf = ctypes.create_string_buffer(64)
    b, sm = c_int(), c_int()
    check(lib().stb_spin_variant_info(v, buf, 64, byref(b), byref(sm)))
    return buf.value.decode()


def variant_name(v: int) -> str:
    buf = ctypes.create_string_buffer(64)
    b, sm = c_int(), c_int()
    check(lib().stb_track_variant_info(v, buf, 64, byref(b), byref(sm)))
    return buf.value.decode()


class Table:
    """Flattened device element table of a Line (rebuild after editing the line)."""

    def __init__(self, line: Line, device: int = 0):
        h = c_void_p()
        check(lib().stb_table_create(line._h, device, byref(h)))
        self._h = h
        self.device = device

    def info(self) -> dict:
        out = (c_double * 6)()
        check(lib().stb_table_info(self._h, out))
        return {"elements": int(out[0]), "pool_doubles": int(out[1]), "flops_per_turn": out[2],
                "smem": bool(out[3]), "table_bytes": int(out[4]), "variant": int(out[5]),
                "variant_name": variant_name(int(out[5]))}

    def autotune(self, coords, nturn: int = 1, aperture_radius: float = 0.0) -> dict:
        """Times every kernel launch variant on a copy of `coords` (6 CUDA float64
        tensors, not modified) and keeps the fastest; returns {name: ms}."""
        chosen = c_int()
        t = (c_double * 32)()
        n = coords[0].numel()
        check(lib().stb_table_autotune(self._h, *[c_void_p(c.data_ptr()) for c in coords], n, nturn,
                                       aperture_radius, byref(chosen), t, 32))
        return {"chosen": variant_name(chosen.value),
                "ms": {variant_name(v): t[v] for v in range(NUM_VARIANTS)}}

    def set_variant(self, v: int) -> None:
        check(lib().stb_table_set_variant(self._h, v))

    def segments(self) -> dict:
        """Segment plan of a table too large for shared memory: {"nseg", "bytes"} (nseg 0: none)."""
        n, b = c_int(), c_int()
        check(lib().stb_table_segments(self._h, byref(n), byref(b)))
        return {"nseg": n.value, "bytes": b.value}

    def set_segment_bytes(self, nbytes: int) -> None:
        check(lib().stb_table_set_segment_bytes(self._h, int(nbytes)))

    def set_contraction(self, policy: str) -> None:
        """"strict" (default: results equal the reference's) or "fast" (the
        kernel compiled with FMA contraction)."""
        if policy not in ("strict", "fast"):
            raise ValueError("policy must be 'strict' or 'fast'")
        check(lib().stb_table_set_contraction(self._h, int(policy == "fast")))

    def track_host(self, x: np.ndarray, nturn: int, aperture_radius: float = 0.0, stable=None):
        """Track() over AoS host coordinates x[n,6] (updated in place); returns (stable, lost_turn, lost_post)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.ndim != 2 or x.shape[1] != 6:
            raise SimTrackError(-1, "x must have shape (n, 6)")
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32) if stable is None else np.ascontiguousarray(stable, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        check(lib().stb_track_host(self._h, x.ctypes.data_as(POINTER(c_double)), n, nturn, aperture_radius,
                                   st.ctypes.data_as(POINTER(c_int)), lt.ctypes.data_as(POINTER(c_int)),
                                   lp.ctypes.data_as(POINTER(c_int))))
        return x, st, lt, lp

    def track_radial_host(self, x: np.ndarray, nturn: int, aperture_radius: float = 0.0, stable=None):
        """Track_Radial (simtrack.cpp:21641-21680) over AoS host x[n, 6] (updated in place)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32) if stable is None else np.ascontiguousarray(stable, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        check(lib().stb_track_radial_host(self._h, x.ctypes.data_as(POINTER(c_double)), n, nturn, aperture_radius,
                                          st.ctypes.data_as(POINTER(c_int)), lt.ctypes.data_as(POINTER(c_int)),
                                          lp.ctypes.data_as(POINTER(c_int))))
        return x, st, lt, lp

    def track_radial_device(self, coords, lost_turn, lost_elem, turn0: int, nturn: int,
                            aperture_radius: float = 0.0, stream=None) -> None:
        n = coords[0].numel()
        _check_device_arrays(coords, lost_turn, lost_elem, n, self.device)
        s = None if stream is None else c_void_p(stream)
        check(lib().stb_track_radial_device(self._h, *[c_void_p(c.data_ptr()) for c in coords], n, turn0, nturn,
                                            aperture_radius, c_void_p(lost_turn.data_ptr()),
                                            c_void_p(lost_elem.data_ptr()), s))

    def track_probe(self, x: np.ndarray, nturn: int, aperture_radius: float = 0.0):
        """Per-element probe: returns (x, stable, lost_turn, lost_post, dump[n, nturn, ncell, 6])."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        ne = self.info()["elements"]
        dump = np.full((n, nturn, ne, 6), np.nan)
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        check(lib().stb_track_probe(self._h, x.ctypes.data_as(POINTER(c_double)), n, nturn, aperture_radius,
                                    dump.ctypes.data_as(POINTER(c_double)), st.ctypes.data_as(POINTER(c_int)),
                                    lt.ctypes.data_as(POINTER(c_int)), lp.ctypes.data_as(POINTER(c_int))))
        return x, st, lt, lp, dump

    def track_device(self, coords, lost_turn, lost_elem, turn0: int, nturn: int, aperture_radius: float = 0.0,
                     stream=None) -> None:
        """Track SoA device tensors in place (coords: 6 CUDA float64 tensors; lost_*: int32 tensors)."""
        n = coords[0].numel()
        _check_device_arrays(coords, lost_turn, lost_elem, n, self.device)
        ptrs = [c.data_ptr() for c in coords]
        s = None if stream is None else c_void_p(stream)
        check(lib().stb_track_device(self._h, *[c_void_p(p) for p in ptrs], n, turn0, nturn, aperture_radius,
                                     c_void_p(lost_turn.data_ptr()), c_void_p(lost_elem.data_ptr()), s))

    def __del__(self):
        try:
            if self._h:
                lib().stb_table_free(self._h)
        except Exception:
            pass


class SpinTable:
    """Element table flattened for spin tracking (Track_Spin, Element::sPass)."""

    def __init__(self, line: Line, device: int = 0):
        h = c_void_p()
        check(lib().stb_table_create_spin(line._h, device, byref(h)))
        self._h = h
        self.device = device

    def info(self) -> dict:
        out = (c_double * 6)()
        check(lib().stb_table_info(self._h, out))
        return {"elements": int(out[0]), "pool_doubles": int(out[1]), "flops_per_turn": out[2],
                "smem": bool(out[3]), "variant": int(out[5]), "variant_name": spin_variant_name(int(out[5]))}

    def autotune(self, coords, nturn: int = 1, aperture_radius: float = 0.0) -> dict:
        """Times every launch variant of the spin kernel on a copy of `coords`
        (9 CUDA float64 tensors, not modified) and keeps the fastest."""
        n = coords[0].numel()
        if len(coords) != 9:
            raise ValueError("a spin table is tuned on nine coordinate arrays")
        arr = (c_void_p * 9)(*[c.data_ptr() for c in coords])
        chosen = c_int()
        t = (c_double * 16)()
        check(lib().stb_table_autotune_spin(self._h, arr, n, nturn, aperture_radius, byref(chosen), t, 16))
        return {"chosen": spin_variant_name(chosen.value),
                "ms": {spin_variant_name(v): t[v] for v in range(NUM_SPIN_VARIANTS)}}

    def set_variant(self, v: int) -> None:
        check(lib().stb_table_set_variant(self._h, v))

    def track_host(self, x: np.ndarray, nturn: int, aperture_radius: float = 0.0, stable=None):
        """Track_Spin over AoS host x[n, 9] (updated in place); returns (x, stable, lost_turn, lost_post)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.ndim != 2 or x.shape[1] != 9:
            raise SimTrackError(-1, "x must have shape (n, 9)")
        n = x.shape[0]
        st = np.ones(n, dtype=np.int32) if stable is None else np.ascontiguousarray(stable, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        check(lib().stb_track_spin_host(self._h, x.ctypes.data_as(POINTER(c_double)), n, nturn, aperture_radius,
                                        st.ctypes.data_as(POINTER(c_int)), lt.ctypes.data_as(POINTER(c_int)),
                                        lp.ctypes.data_as(POINTER(c_int))))
        return x, st, lt, lp

    def track_probe(self, x: np.ndarray, nturn: int, aperture_radius: float = 0.0):
        """Per-element probe: returns (x, stable, lost_turn, lost_post, dump[n, nturn, ncell, 9])."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        ne = self.info()["elements"]
        dump = np.full((n, nturn, ne, 9), np.nan)
        st = np.ones(n, dtype=np.int32)
        lt = np.zeros(n, dtype=np.int32)
        lp = np.zeros(n, dtype=np.int32)
        check(lib().stb_track_spin_probe(self._h, x.ctypes.data_as(POINTER(c_double)), n, nturn, aperture_radius,
                                         dump.ctypes.data_as(POINTER(c_double)), st.ctypes.data_as(POINTER(c_int)),
                                         lt.ctypes.data_as(POINTER(c_int)), lp.ctypes.data_as(POINTER(c_int))))
        return x, st, lt, lp, dump

    def track_device(self, coords, lost_turn, lost_elem, turn0: int, nturn: int, aperture_radius: float = 0.0,
                     stream=None) -> None:
        """coords: 9 CUDA float64 tensors (x, px, y, py, z, pt, sx, sy, sz), updated in place."""
        n = coords[0].numel()
        _check_device_arrays(coords, lost_turn, lost_elem, n, self.device, ncoord=9)
        s = None if stream is None else c_void_p(stream)
        check(lib().stb_track_spin_device(self._h, *[c_void_p(c.data_ptr()) for c in coords], n, turn0, nturn,
                                          aperture_radius, c_void_p(lost_turn.data_ptr()),
                                          c_void_p(lost_elem.data_ptr()), s))

    def __del__(self):
        try:
            if self._h:
                lib().stb_table_free(self._h)
        except Exception:
            pass


def Cal_Orbit_Num(line: Line, deltap: float = 0.0, device: int = 0) -> np.ndarray:
    """Cal_Orbit_Num (simtrack.cpp:14947-15030): the closed orbit after every
    element, [ncell, 6] (also stored in the elements' X fields)."""
    out = np.empty((line.Ncell, 6))
    check(lib().stb_cal_orbit(line._h, deltap, out.ctypes.data_as(POINTER(c_double)), device))
    return out


def Cal_SRLoss_U0rad(line: Line, track_form: bool = False) -> float:
    """Cal_SRLoss_U0rad / Cal_SRLoss_U0rad_Track (simtrack.cpp:20691-20766):
    the reference particle's synchrotron-radiation loss per turn, MeV (0
    unless radiation is on; host computation)."""
    u = c_double()
    check(lib().stb_cal_srloss_u0rad(line._h, int(track_form), byref(u)))
    return u.value


def Cal_SRLoss_Particle(line: Line, x, device: int = 0) -> float:
    """Cal_SRLoss_Particle (simtrack.cpp:20768-20781): x (6 float64, updated
    in place) passed once through every element but the RF cavities on the
    GPU; returns (pt - pt0) * beta * energy in MeV (negative for a loss)."""
    v = np.asarray(x)
    if v.dtype != np.float64 or v.shape != (6,) or not v.flags.c_contiguous:
        raise ValueError("x is a C-contiguous float64 array of 6 coordinates, updated in place")
    loss = c_double()
    check(lib().stb_cal_srloss_particle(line._h, v.ctypes.data_as(POINTER(c_double)), byref(loss), device))
    return loss.value


DA_DRIVERS = {"Track_DA1": 1, "Track_DA2": 2, "Track_DA3": 3, "Track_DA_Radial": 4, "Track_DA_Uniform": 5,
              "Track_DA_Radial_Uniform": 6}


def Track_DA_driver(name: str, line: Line, nturn: int, deltap0: float, sigmax0: float, sigmay0: float,
                    angle: float = 0.0, filename=None, device: int = 0):
    """The reference's other DA drivers by name (Track_DA1, Track_DA2,
    Track_DA3, Track_DA_Radial: simtrack.cpp:21443-21734; Track_DA_Uniform,
    Track_DA_Radial_Uniform: 21574, 21736), writing the reference's file when
    `filename` is given.  Bisections return (angle labels [deg], sigma);
    uniform sweeps (at `angle` [rad]) return (stable flags, sigma) of the lines
    written, up to the first loss."""
    a = (c_double * 150)()
    sg = (c_double * 150)()
    n = c_long(0)
    check(lib().stb_track_da_driver(line._h, DA_DRIVERS[name], nturn, deltap0, angle, sigmax0, sigmay0,
                                    None if filename is None else str(filename).encode(), a, sg, ctypes.byref(n),
                                    device))
    return np.array(a[:n.value]), np.array(sg[:n.value])


def Cal_Tunes_Track(line: Line, x, nturn: int, tune_low: float = 0.660, tune_high: float = 0.70,
                    device: int = 0):
    """Cal_Tunes_Track (simtrack.cpp:20971-20990): (tune1, tune2) of particle
    x[6] from its turn-by-turn record, or None if it is lost; x is tracked in
    place (a float64 numpy array of 6)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    t = (c_double * 2)()
    st = c_int(0)
    check(lib().stb_cal_tunes_track(line._h, x.ctypes.data_as(POINTER(c_double)), nturn, tune_low, tune_high, t,
                                    ctypes.byref(st), device))
    return (t[0], t[1]) if st.value else None


def Cal_Tunes_Track_orbit(line: Line, deltap0: float, tune_low: float = 0.660, tune_high: float = 0.70,
                          device: int = 0):
    """Cal_Tunes_Track(line, deltap0) (simtrack.cpp:20992-21025): tunes of the
    closed orbit at deltap0 over 1,024 turns (0, 0 if it is lost)."""
    t = (c_double * 2)()
    check(lib().stb_cal_tunes_track_orbit(line._h, deltap0, tune_low, tune_high, t, device))
    return t[0], t[1]


def Cal_dz0_OnMomentumPart(line: Line, x0, device: int = 0):
    """Cal_dz0_OnMomentumPart (simtrack.cpp:20929-20940): returns (x0 after
    the pass, dz0[ncell]); z and pt are reset before every element."""
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    dz0 = np.empty(line.Ncell)
    check(lib().stb_cal_dz0(line._h, x.ctypes.data_as(POINTER(c_double)), dz0.ctypes.data_as(POINTER(c_double)),
                            device))
    return x, dz0


def Track_wrt_OnMomentumPart(line: Line, x, dz0, nturn: int, device: int = 0):
    """Track_wrt_OnMomentumPart (simtrack.cpp:20942-20967) for x[n, 6]
    (copied): returns (x, stable, lost_turn, lost_post)."""
    x = np.ascontiguousarray(np.atleast_2d(np.asarray(x, dtype=np.float64))).copy()
    d = np.ascontiguousarray(dz0, dtype=np.float64)
    n = x.shape[0]
    st = np.ones(n, dtype=np.int32)
    lt = np.zeros(n, dtype=np.int32)
    lp = np.zeros(n, dtype=np.int32)
    P = lambda a, t: a.ctypes.data_as(POINTER(t))
    check(lib().stb_track_wrt_onmom(line._h, P(x, c_double), n, P(d, c_double), nturn, P(st, c_int), P(lt, c_int),
                                    P(lp, c_int), device))
    return x, st, lt, lp


def Cal_Chrom_Track(line: Line, tune_low: float = 0.660, tune_high: float = 0.70, device: int = 0):
    """Cal_Chrom_Track (simtrack.cpp:21027-21051): (Chromx1, Chromy1, Chromx2,
    Chromy2) from the tracked tunes at deltap = +3e-4, -3e-4 and 0."""
    c = (c_double * 4)()
    check(lib().stb_cal_chrom_track(line._h, tune_low, tune_high, c, device))
    return tuple(c[:])


def Track_tbt(line: Line, x, nturn: int, stable=None, device: int = 0, spin: bool = False, bpm_index=None):
    """Track_tbt (simtrack.cpp:20841-20860; with spin=True Track_tbt_spin,
    20863-20882, x[n, 9]) for particles x[n, 6] (copied): returns (x, stable,
    lost_turn, lost_post, x_tbt[n, nturn, 6 or 9]); x_tbt holds the
    coordinates at the start of each turn up to the turn of the loss and NaN
    after it.  With bpm_index (20884-20905) the record is taken after that
    element, in the turns that reach it."""
    x = np.ascontiguousarray(np.atleast_2d(np.asarray(x, dtype=np.float64))).copy()
    n, nc = x.shape
    if nc != (9 if spin else 6):
        raise ValueError("x must have 9 columns with spin, 6 without")
    st = np.ones(n, dtype=np.int32) if stable is None else np.ascontiguousarray(stable, dtype=np.int32).copy()
    lt = np.zeros(n, dtype=np.int32)
    lp = np.zeros(n, dtype=np.int32)
    tbt = np.full((n, nturn, nc), np.nan)
    P = lambda a, t: a.ctypes.data_as(POINTER(t))
    if bpm_index is not None:
        fn = lib().stb_track_tbt_spin_bpm if spin else lib().stb_track_tbt_bpm
        check(fn(line._h, P(x, c_double), n, nturn, P(tbt, c_double), int(bpm_index), P(st, c_int), P(lt, c_int),
                 P(lp, c_int), device))
        return x, st, lt, lp, tbt
    fn = lib().stb_track_tbt_spin if spin else lib().stb_track_tbt
    check(fn(line._h, P(x, c_double), n, nturn, P(tbt, c_double), P(st, c_int), P(lt, c_int), P(lp, c_int), device))
    return x, st, lt, lp, tbt


def Track_tbt_FMA(line: Line, deltap0: float, sigmax0: float, sigmay0: float, filename="./FMA-output.dat",
                  tune_low: float = 0.660, tune_high: float = 0.70, device: int = 0) -> int:
    """Track_tbt_FMA (simtrack.cpp:21179-21241): writes the frequency map to
    `filename` in the reference's format; returns the number of rows."""
    rows = c_long(0)
    check(lib().stb_track_tbt_fma(line._h, deltap0, sigmax0, sigmay0, tune_low, tune_high, str(filename).encode(),
                                  ctypes.byref(rows), device))
    return rows.value


def Track_tbt_Lyapunov(line: Line, deltap0: float, sigmax0: float, sigmay0: float, filename="./Lmap-output.dat",
                       device: int = 0) -> int:
    """Track_tbt_Lyapunov (simtrack.cpp:21243-21306): writes the Lyapunov map
    to `filename` in the reference's format; returns the number of rows."""
    rows = c_long(0)
    check(lib().stb_track_tbt_lyapunov(line._h, deltap0, sigmax0, sigmay0, str(filename).encode(),
                                       ctypes.byref(rows), device))
    return rows.value


def Track_DA(line: Line, nturn: int, deltap0: float, sigmax0: float, sigmay0: float, filename=None,
             device: int = 0):
    """Track_DA (simtrack.cpp:21389-21441): returns (angles_deg[10], sigma[10]);
    writes the reference's output file when `filename` is given."""
    ang = (c_double * 10)()
    sig = (c_double * 10)()
    check(lib().stb_track_da(line._h, nturn, deltap0, sigmax0, sigmay0,
                             None if filename is None else str(filename).encode(), ang, sig, device))
    return np.array(ang[:]), np.array(sig[:])


def Track_Radial(line: Line, x, nturn: int, stable: int = 1):
    """Track_Radial (simtrack.cpp:21641-21680) for one particle x[6] (updated in place).

    Returns (stable, lost_turn, lost_post)."""
    arr = np.asarray(x, dtype=np.float64).reshape(1, 6).copy()
    _, st, lt, lp = Table(line).track_radial_host(arr, nturn, 0.0, np.array([stable], dtype=np.int32))
    x[:] = arr[0]
    return int(st[0]), int(lt[0]), int(lp[0])


def Track_Spin(line: Line, x, nturn: int, stable: int = 1):
    """Track_Spin (simtrack.cpp:21766-21789) for one particle x[9] (updated in place).

    Returns (stable, lost_turn, lost_post)."""
    arr = np.asarray(x, dtype=np.float64).reshape(1, 9).copy()
    _, st, lt, lp = SpinTable(line).track_host(arr, nturn, 0.0, np.array([stable], dtype=np.int32))
    x[:] = arr[0]
    return int(st[0]), int(lt[0]), int(lp[0])


def Track_Batch(line: Line, x: np.ndarray, nturn: int, aperture_radius: float = 0.0, stable=None, device: int = 0):
    """Track() for many particles at once: x[n,6] AoS, updated in place."""
    return Table(line, device).track_host(x, nturn, aperture_radius, stable)[1:]


def Track(line: Line, x, nturn: int, stable: int = 1):
    """Track (simtrack.cpp:20791-20814) for one particle x[6] (list or array, updated in place).

    Returns (stable, lost_turn, lost_post)."""
    arr = np.asarray(x, dtype=np.float64).reshape(1, 6).copy()
    _, st, lt, lp = Table(line).track_host(arr, nturn, 0.0, np.array([stable], dtype=np.int32))
    for k in range(6):
        x[k] = arr[0, k]
    return int(st[0]), int(lt[0]), int(lp[0])


class Scan:
    """Batched dynamic-aperture scan over several seed tables (stb_scan_*)."""

    def __init__(self, tables, x0_per_seed, aperture_radius: float = 0.0, device: int = 0):
        self._tables = list(tables)  # keep the tables alive for the scan's lifetime
        xs = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 6) for x in x0_per_seed]
        if len(xs) != len(self._tables):
            raise SimTrackError(-1, "one particle array per table")
        self.n_per_seed = np.array([len(x) for x in xs], dtype=np.int64)
        x0 = np.ascontiguousarray(np.concatenate(xs, axis=0))
        arr = (c_void_p * len(self._tables))(*[t._h for t in self._tables])
        nps = (ctypes.c_long * len(xs))(*[int(v) for v in self.n_per_seed])
        h = c_void_p()
        check(lib().stb_scan_create(arr, len(xs), x0.ctypes.data_as(POINTER(c_double)), nps, aperture_radius,
                                    device, byref(h)))
        self._h = h
        self.n = int(self.n_per_seed.sum())

    def configure(self, variant: int = -1, chunk: int = 0) -> None:
        check(lib().stb_scan_configure(self._h, variant, chunk))

    def autotune(self, nturn: int = 16) -> dict:
        """Picks the fastest tracking-kernel variant on a snapshot of the current state."""
        ch = c_int()
        t = (c_double * 16)()
        check(lib().stb_scan_autotune(self._h, nturn, byref(ch), t, 16))
        return {"chosen": ch.value, "packed": self.packing(), "ms": [t[i] for i in range(NUM_SCAN_VARIANTS)]}

    def run(self, nturn: int, turns_per_block: int = 256, use_graph: bool = True) -> None:
        check(lib().stb_scan_run(self._h, nturn, turns_per_block, int(use_graph)))

    def results(self):
        """(lost_turn[n] (-1 alive), lost_elem[n], x[n, 6]) in input order."""
        lt = np.empty(self.n, dtype=np.int32)
        le = np.empty(self.n, dtype=np.int32)
        x = np.empty((self.n, 6))
        check(lib().stb_scan_results(self._h, c_void_p(lt.ctypes.data), c_void_p(le.ctypes.data),
                                     c_void_p(x.ctypes.data)))
        return lt, le, x

    def set_tbt(self, tbt, nturns: int) -> None:
        """Records x, px, y, py of every particle after each of the first nturns
        turns into the CUDA float64 tensor tbt[nturns, 4, n] (None: stop)."""
        if tbt is None or nturns == 0:
            check(lib().stb_scan_set_tbt(self._h, None, 0))
            self._tbt = None
            return
        if tuple(tbt.shape) != (nturns, 4, self.n) or not tbt.is_contiguous():
            raise SimTrackError(-1, "tbt must be a contiguous [nturns, 4, n] tensor")
        self._tbt = tbt  # keep the buffer alive while the scan writes it
        check(lib().stb_scan_set_tbt(self._h, c_void_p(tbt.data_ptr()), nturns))

    def retire(self, mask) -> None:
        """Stops tracking the live particles with mask[i] true (x0 order)."""
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1))
        if m.size != self.n:
            raise SimTrackError(-1, "mask must have one entry per particle")
        check(lib().stb_scan_retire(self._h, c_void_p(m.ctypes.data)))

    def set_packing(self, pack: bool) -> None:
        check(lib().stb_scan_set_packing(self._h, int(bool(pack))))

    def packing(self) -> bool:
        v = c_int()
        check(lib().stb_scan_packing(self._h, byref(v)))
        return bool(v.value)

    def set_abort(self, value: bool = True) -> None:
        """Asks a run in progress (in another thread) to stop at the next turn
        block (run raises SimTrackError with STB_EABORTED); False re-arms."""
        check(lib().stb_scan_set_abort(self._h, int(bool(value))))

    def set_budget(self, seconds: float) -> None:
        """Wall-clock budget of each run call (0: none); a spent budget raises
        SimTrackError with STB_ETIMEOUT at a turn-block boundary."""
        check(lib().stb_scan_set_budget(self._h, float(seconds)))

    def checkpoint(self, path) -> None:
        check(lib().stb_scan_checkpoint(self._h, str(path).encode()))

    def restore(self, path) -> None:
        check(lib().stb_scan_restore(self._h, str(path).encode()))

    def stats(self) -> dict:
        st = (c_double * 6)()
        check(lib().stb_scan_stats(self._h, st))
        return {"turns": int(st[0]), "device_ms": st[1], "blocks": int(st[2]), "variant": int(st[3]),
                "chunk": int(st[4]), "particles": int(st[5])}

    def __del__(self):
        try:
            if self._h:
                lib().stb_scan_free(self._h)
        except Exception:
            pass


RETIRED = 0x40000000  # lost_turn of particles removed by Scan.retire


def track_seeds_static(tables, n_per_seed, coords, lost_turn, lost_elem, turn0: int, nturn: int,
                       aperture_radius: float = 0.0, stream=None) -> None:
    """stb_track_seeds_static: tracks several seed tables' particles in one
    work-list launch without allocating device memory.  coords: CUDA float64
    tensor [6, n] (x, px, y, py, z, pt rows; seed 0's particles first);
    lost_turn, lost_elem: CUDA int32 tensors [n]."""
    if len(tables) != len(n_per_seed) or not tables:
        raise ValueError("one particle count per table")
    ntot = int(sum(int(v) for v in n_per_seed))
    if coords.dim() != 2 or coords.shape[0] != 6 or coords.shape[1] < ntot:
        raise ValueError(f"coords must have shape [6, >= {ntot}], not {tuple(coords.shape)}")
    _check_device_arrays([coords[k] for k in range(6)], lost_turn, lost_elem, ntot, tables[0].device)
    arr = (c_void_p * len(tables))(*[t._h for t in tables])
    nps = (ctypes.c_long * len(tables))(*[int(v) for v in n_per_seed])
    ptrs = [c_void_p(coords[k].data_ptr()) for k in range(6)]
    st = None if stream is None else c_void_p(stream)
    check(lib().stb_track_seeds_static(arr, len(tables), nps, *ptrs, c_void_p(lost_turn.data_ptr()),
                                       c_void_p(lost_elem.data_ptr()), turn0, nturn, aperture_radius, st))


def fine_tune(x, n: int, nsig: int, stride: int, tune_lower: float, tune_upper: float, out, px=None,
              offset: int = 0, device: int = 0, stream=None) -> None:
    """FineTuneFinder (simtrack.cpp:2288 / 2321) for nsig signals at once on
    the GPU: sample i of signal j is x.flat[offset + i * stride + j] (CUDA
    float64 tensors; px optional, same layout); out: CUDA float64 [nsig]."""
    esz = 8
    xp = c_void_p(x.data_ptr() + offset * esz)
    pp = None if px is None else c_void_p(px.data_ptr() + offset * esz)
    check(lib().stb_fine_tune(xp, pp, n, nsig, stride, tune_lower, tune_upper, c_void_p(out.data_ptr()), device,
                              None if stream is None else c_void_p(stream)))


NUM_FEATURES = 12
FEATURE_NAMES = ["amp_x", "amp_y", "delta_1e3", "angle", "qx_w1", "qy_w1", "qx_w2", "qy_w2",
                 "log10_dqx", "log10_dqy", "log10_action_spread", "max_amp"]


def tbt_features(tbt, x0, tunes, twiss6, out, device: int = 0, stream=None) -> None:
    """Surrogate features from a turn-by-turn record tbt[nturn, 4, n], initial
    coordinates x0[6, n] and window tunes[4, n] (all CUDA float64) into
    out[n, 12] (CUDA float32).  twiss6 = (beta_x, alpha_x, beta_y, alpha_y,
    emit_x, emit_y) at the record point."""
    nturn, _, n = tbt.shape
    tw = (c_double * 6)(*[float(v) for v in twiss6])
    check(lib().stb_tbt_features(c_void_p(tbt.data_ptr()), n, nturn, c_void_p(x0.data_ptr()),
                                 c_void_p(tunes.data_ptr()), tw, c_void_p(out.data_ptr()), device,
                                 None if stream is None else c_void_p(stream)))


class MLP:
    """The loss-prediction surrogate network on the tensor cores (stb_mlp_*)."""

    def __init__(self, nin: int = 12, hidden: int = 256, nout: int = 2, max_batch: int = 4096, seed: int = 0,
                 device: int = 0):
        h = c_void_p()
        check(lib().stb_mlp_create(nin, hidden, nout, max_batch, seed, device, byref(h)))
        self._h = h
        self.nin, self.hidden, self.nout, self.max_batch = nin, hidden, nout, max_batch

    @property
    def nparams(self) -> int:
        return int(lib().stb_mlp_param_count(self._h))

    def get_params(self, which: int = 0) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        check(lib().stb_mlp_get_params(self._h, out.ctypes.data_as(POINTER(ctypes.c_float)), which))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().stb_mlp_set_params(self._h, p.ctypes.data_as(POINTER(ctypes.c_float))))

    def set_adamw(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=1e-2) -> None:
        check(lib().stb_mlp_set_adamw(self._h, lr, beta1, beta2, eps, weight_decay))

    def forward(self, x, probs) -> None:
        """x: CUDA float32 tensor [B, nin]; probs: CUDA float32 tensor [B, nout] (written)."""
        check(lib().stb_mlp_forward(self._h, c_void_p(x.data_ptr()), x.shape[0], c_void_p(probs.data_ptr())))

    def gradients(self, x, labels, weights=None) -> float:
        loss = ctypes.c_float()
        check(lib().stb_mlp_gradients(self._h, c_void_p(x.data_ptr()), c_void_p(labels.data_ptr()),
                                      None if weights is None else c_void_p(weights.data_ptr()), x.shape[0],
                                      byref(loss)))
        return loss.value

    def train_step(self, x, labels, weights=None) -> float:
        loss = ctypes.c_float()
        check(lib().stb_mlp_train_step(self._h, c_void_p(x.data_ptr()), c_void_p(labels.data_ptr()),
                                       None if weights is None else c_void_p(weights.data_ptr()), x.shape[0],
                                       byref(loss)))
        return loss.value

    def __del__(self):
        try:
            if self._h:
                lib().stb_mlp_free(self._h)
        except Exception:
            pass
