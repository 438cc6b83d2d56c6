"""C ABI and host-side construction logic (CPU only: no kernel is launched)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(stb_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(native_lib):
    syms = declared_symbols()
    assert len(syms) > 20
    missing = [s for s in syms if not hasattr(native_lib, s)]
    assert not missing, missing


def test_python_signatures_cover_header(native_lib):
    from simtrack_b200._native import SIGNATURES
    bound = {s[0] for s in SIGNATURES}
    assert set(declared_symbols()) <= bound | set()


def test_element_defaults_and_setp(native_lib):
    import simtrack_b200 as st
    st.Set_RefPartEnergy(100000.0 / 938.27201, 938.27201, 1, 1)
    q = st.QUAD("qf", 1.0, 0.06, 0.0)
    assert q.TYPE == "QUAD"
    assert q.GetP("Nint") == int(1.0 / 0.05) + 1  # QUAD ctor, simtrack.cpp:8635
    q.SetP("Nint", 4.7)
    assert q.GetP("Nint") == 4  # int(value), simtrack.cpp:8657
    b = st.SBEND("b", 2.0, 0.0314, 0.0, 0.0)
    assert b.GetP("Nint") == int(2.0 / 0.25) + 1
    m = st.MULT("m", 1.0, [0, 0.1, 0, 0.3], [0, 0, 0, 0, 0, 2.0])
    assert m.GetP("Norder") == 5  # highest non-zero order, simtrack.cpp:8943-8950
    m.SetP("K7L", 1.0)
    assert m.GetP("Norder") == 5  # SetP does not recompute Norder
    with pytest.raises(st.SimTrackError) as ei:
        q.SetP("K2L", 1.0)
    assert "does not have a parameter" in str(ei.value)
    with pytest.raises(st.SimTrackError):
        st.SBEND("bad", -1.0, 0.1, 0, 0)  # SBEND length must be positive
    with pytest.raises(st.SimTrackError):
        st.BEAMBEAM("bb", 5, 1e11, 1, 0.1, 3, 1e-8, 1, 0, 1e-8, 1, 0)
    bb = st.BEAMBEAM("bb", 6, 1e11, 1, 0.1, 3, 1e-8, 1, 0, 1e-8, 1, 0)
    with pytest.raises(st.SimTrackError):
        bb.SetP("TREATMENT", 5)
    assert bb.GetP("TREATMENT") == 6


def test_line_editing(native_lib):
    import simtrack_b200 as st
    st.Set_RefPartEnergy(100000.0 / 938.27201, 938.27201, 1, 1)
    line = st.Line()
    for i in range(4):
        line.Append(st.DRIFT(f"d{i}", 1.0 + i))
    assert line.Ncell == 4 and line.Length == pytest.approx(10.0)
    line.Insert(1, st.QUAD("q", 0.5, 0.1, 0.0))
    assert line.Ncell == 5 and line.Cell(1).TYPE == "QUAD"
    line.Replace(1, st.SEXT("s", 0.0, 1.0, 0.0))
    assert line.Cell(1).TYPE == "SEXT" and line.Length == pytest.approx(10.0)
    line.Delete(0)
    assert line.Ncell == 4 and line.Cell(0).TYPE == "SEXT"
    line.Rewind(1)
    assert line.Cell(3).TYPE == "SEXT"
    line.Invert()
    assert line.Cell(0).TYPE == "SEXT"
    line.Delete(99)  # out of range: ignored, as in the reference (simtrack.cpp:12381)
    assert line.Ncell == 4


def test_last_error_and_status_codes(native_lib):
    from simtrack_b200 import _native
    L = native_lib
    h = ctypes.c_void_p()
    rc = L.stb_element_new(b"NOPE", b"x", None, 0, ctypes.byref(h))
    assert rc == _native.STB_EUNSUPPORTED
    assert b"NOPE" in L.stb_last_error()
    rc = L.stb_element_new(b"QUAD", b"x", (ctypes.c_double * 1)(1.0), 1, ctypes.byref(h))
    assert rc == _native.STB_EINVAL
    assert L.stb_track_host(None, None, 0, 0, 0.0, None, None, None) == _native.STB_EINVAL


def test_flatten_rejects_unsupported_settings(native_lib):
    import simtrack_b200 as st
    st.Set_RefPartEnergy(100000.0 / 938.27201, 938.27201, 1, 1)
    line = st.Line()
    q = st.QUAD("q", 1.0, 0.1, 0.0)
    q.set_misalignment(0, 0, 0, 1e-3, 0, 0)  # pitch: GtoL2 is not implemented
    line.Append(q)
    with pytest.raises(st.SimTrackError) as ei:
        st.Table(line)
    assert ei.value.code in (-6, -3)


def test_soft_gaussian_collision_rejects_empty_beams(native_lib):
    """BeamBeam4D_SoftGaussian's entry points check their beams before any
    device work (an empty beam has no moments)."""
    from ctypes import POINTER, c_double
    from simtrack_b200 import _native
    b = (c_double * 6)()
    L = native_lib
    assert L.stb_bb4d_soft_gaussian_host(1e11, 0, b, 1e11, 1, b, 100.0, 100.0, 1.0, 1.0, 0) == _native.STB_EINVAL
    assert L.stb_bb4d_soft_gaussian_host(1e11, 1, None, 1e11, 1, b, 100.0, 100.0, 1.0, 1.0, 0) == _native.STB_EINVAL
    assert L.stb_bb4d_soft_gaussian_device(1e11, 1, None, 1e11, 1, None, 100.0, 100.0, 1.0, 1.0, 0, None) \
        == _native.STB_EINVAL


def test_pic_and_luminosity_entry_points_check_arguments_first(native_lib):
    """The particle-in-cell and luminosity entry points reject bad beams,
    grids and slice counts before any device work (no GPU needed)."""
    from ctypes import byref, c_double
    from simtrack_b200 import _native
    L, E = native_lib, _native.STB_EINVAL
    b = (c_double * 60)()
    g = (c_double * (4 * 48 * 48))()
    out = c_double()
    # BeamBeam4D_PIC: at least two macro-particles per beam, positive gamma
    assert L.stb_bb4d_pic_host(1e11, 1, b, 1e11, 10, b, 100.0, 100.0, 1.0, 1.0, 0) == E
    assert L.stb_bb4d_pic_host(1e11, 10, b, 1e11, 10, b, -1.0, 100.0, 1.0, 1.0, 0) == E
    assert L.stb_bb4d_pic_device(1e11, 10, None, 1e11, 10, None, 100.0, 100.0, 1.0, 1.0, 0, None) == E
    # grids: square, a power of two from 8 to 512
    for nx, ny in ((48, 48), (32, 64), (4, 4), (1024, 1024)):
        assert L.stb_pic_green_function(0.0, 0.0, nx, ny, 1e-5, 1e-5, g, g, 0) == E
        assert L.stb_bb4d_pic_nonoffset_host(1e11, 10, b, 1e11, 10, b, 100.0, 100.0, 1.0, 1.0, nx, ny, 1e-5, 1e-5, g,
                                             g, 0) == E
    # luminosities: non-empty beams; sliced forms: slice counts and populations
    assert L.stb_lumi_pic_4d_host(1e11, 0, 1e11, 10, b, b, 1, 1e4, 0, byref(out)) == E
    assert L.stb_lumi_pic_6d_host(1e11, 10, 1e11, 10, 0, 1, b, b, 100.0, 100.0, 1.0, 1.0, 1, 1e4, 0, byref(out)) == E
    assert L.stb_lumi_pic_6d_angle_host(1e11, 10, 1e11, 10, 2.0, 1, 1, b, b, 100.0, 100.0, 1.0, 1.0, 1, 1e4, 0,
                                        byref(out)) == E
    assert L.stb_bb6d_pic_host(1e11, 10, b, 1e11, 10, b, 100.0, 100.0, 1.0, 1.0, 6, 1, 0) == E  # slices of 1
    zb = (c_double * 3)(1.0, 0.0, -1.0)
    assert L.stb_bb6d_pic_interpolation_host(1e11, 10, b, 1e11, 10, b, 100.0, 100.0, 1.0, 1.0, 2, 1, zb, zb, 64, 64,
                                             1e-5, 1e-5, g, g, 0) == E  # unequal slice counts
    # Cal_SRLoss_Particle: NULL arguments
    assert L.stb_cal_srloss_particle(None, None, None, 0) == E
