"""Read_MADX_Lattice (simtrack.cpp:13591-13791): the reader against the
reference's own reader, on the RHIC lattice shipped with the reference
(Example1/parameters_input, 6,858 elements; read in place, CPU only) and on
tables written by lattices.write_madx_tfs, and tracking through what was read.

Read_BMAD_Lattice (simtrack.cpp:14054-14244): the reader against the
reference's own reader on the HSR table of the reference's Example2
(tests/golden/hsr_bmad.tab.xz, 2,836 elements with patches and solenoids),
and against the element names and S positions of the orbit the reference
printed for it (tests/golden/hsr_orbit0.dat.xz)."""
import lzma
from pathlib import Path

import numpy as np
import pytest

import oracle_bridge
from simtrack_b200 import api
from simtrack_b200 import lattices as lt

_REF = oracle_bridge.ref_source_dir()
RHIC_TFS = _REF / "Example1" / "parameters_input" if _REF else Path("/nonexistent")

PARAMS = {
    "SBEND": ("ANGLE", "E1", "E2", "Nint"),
    "GSBEND": ("ANGLE", "K0L", "E1", "E2", "Nint"),
    "QUAD": ("K1L", "K1SL", "Nint"),
    "SEXT": ("K2L", "K2SL", "Nint"),
    "OCT": ("K3L", "K3SL", "Nint"),
    "MULT": tuple(f"K{k}L" for k in range(11)) + tuple(f"K{k}SL" for k in range(11)) + ("Norder", "Nint"),
    "HKICKER": ("HKICK",),
    "VKICKER": ("VKICK",),
    "KICKER": ("HKICK", "VKICK"),
    "RFCAV": ("VRF", "FRF", "PHASE0"),
    "SOLEN": ("KS",),
    "PATCH": ("DX", "DY", "DS", "THETA"),
    "SBENDMULT": ("ANGLE", "E1", "E2", "Norder", "Nint") + tuple(f"K{k}L" for k in range(11)) +
                 tuple(f"K{k}SL" for k in range(11)),
    "BEAMBEAM": ("TREATMENT", "NP", "BBSCALE", "SIGMAL", "NSLICE", "EMITX", "EMITY", "BETAX", "ALFAX", "BETAY",
                 "ALFAY"),
}

GOLDEN = Path(__file__).resolve().parent / "golden"
HSR_ENERGY = (275000. / 938.27201, 938.27201, 1.0, 1.0)  # Example2/DA_cal.cpp:613


def hsr_table(tmp_path, numeric_only=False) -> Path:
    """The Example2 Bmad table written to tmp_path (optionally without the
    column-name and unit rows, which the reference's reader cannot take)."""
    from golden.make_golden import numeric_rows
    text = lzma.decompress((GOLDEN / "hsr_bmad.tab.xz").read_bytes()).decode()
    path = tmp_path / ("hsr_numeric.tab" if numeric_only else "hsr.tab")
    path.write_text(numeric_rows(text) if numeric_only else text)
    return path


def hsr_orbit0():
    """(names, types, S, orbit[n, 6]) printed by the reference (6 digits)."""
    rows = lzma.decompress((GOLDEN / "hsr_orbit0.dat.xz").read_bytes()).decode().splitlines()[1:]
    t = [r.split() for r in rows]
    return ([r[0] for r in t], [r[1] for r in t], np.array([float(r[2]) for r in t]),
            np.array([[float(v) for v in r[3:9]] for r in t]))


def compare_lines(line, ref):
    assert line.Ncell == ref.nelem
    for i in range(line.Ncell):
        e = line.Cell(i)
        rt, rn, rg = ref.element(i)
        assert (e.TYPE, e.NAME) == (rt, rn), i
        g = e.geometry()
        for k in ("L", "S", "DX", "DY", "DPSI", "APx", "APy"):
            assert g[k] == rg[k], (i, k, g[k], rg[k])
        for p in PARAMS.get(rt, ()):
            assert e.GetP(p) == ref.getp(i, p), (i, rt, p)


@pytest.mark.skipif(not RHIC_TFS.exists(), reason="reference example lattice not present")
def test_reader_matches_reference_on_rhic_lattice(ref_oracle, port_oracle):
    api.Set_RefPartEnergy(100.0, 938.27201, 1, 1)
    ref_oracle.L.ref_set_ref_energy(100.0, 938.27201, 1.0, 1.0)
    line = api.Line()
    line.read_madx(str(RHIC_TFS))
    ref_oracle.read_madx(str(RHIC_TFS))
    compare_lines(line, ref_oracle)
    # tracking through what was read: the C restatement on our reader's line
    # equals the reference's Track() on the reference reader's line
    lat = lt.Lattice("rhic_tfs", lt.specs_from_line(line), 100.0)
    port_oracle.build(lat)
    X = np.array([[1e-3, 0, 5e-4, 0, 0, 0], [-2e-3, 1e-5, 1e-3, 0, 0.01, 3e-4]])
    xp, sp, lp_, pp = port_oracle.track(X.copy(), 3)
    xr = X.copy()
    st = np.ones(2, dtype=np.int32)
    lt_ = np.zeros(2, dtype=np.int32)
    lp = np.zeros(2, dtype=np.int32)
    from ctypes import POINTER, c_double, c_int
    ref_oracle.L.ref_track(ref_oracle.line, xr.ctypes.data_as(POINTER(c_double)), 2, 3,
                           st.ctypes.data_as(POINTER(c_int)), lt_.ctypes.data_as(POINTER(c_int)),
                           lp.ctypes.data_as(POINTER(c_int)))
    assert np.array_equal(sp, st) and np.array_equal(lp_, lt_)
    assert np.array_equal(xp, xr)


def test_written_table_reads_back(tmp_path, ref_oracle):
    lat = lt.rhic_like_ring(seed=4)
    # give a few elements a roll so that TILT is exercised
    for e in lat.elements[10:400:37]:
        if e.type in ("QUAD", "SEXT", "MULT", "SBEND"):
            e.misalign = (0.0, 0.0, 0.0, 0.0, 0.0, 2e-3)
    path = tmp_path / "ring.tfs"
    lt.write_madx_tfs(lat, str(path))
    lat.set_reference()
    ref_oracle.L.ref_set_ref_energy(lat.gamma, lat.E0, lat.Q, lat.A)
    line = api.Line()
    line.read_madx(str(path))
    ref_oracle.read_madx(str(path))
    compare_lines(line, ref_oracle)
    assert abs(line.Length - lat.circumference) < 1e-6


@pytest.mark.gpu
def test_gpu_tracking_through_read_table(tmp_path, native_lib, ref_oracle):
    lat = lt.rhic_like_ring(seed=5)
    for e in lat.elements[5:900:41]:
        if e.type in ("QUAD", "SEXT", "MULT", "SBEND"):
            e.misalign = (0.0, 0.0, 0.0, 0.0, 0.0, -1.5e-3)
    path = tmp_path / "ring.tfs"
    lt.write_madx_tfs(lat, str(path))
    lat.set_reference()
    ref_oracle.L.ref_set_ref_energy(lat.gamma, lat.E0, lat.Q, lat.A)
    line = api.Line()
    line.read_madx(str(path))
    ref_oracle.read_madx(str(path))
    tab = api.Table(line)
    sig = lat.meta["sigma_ip"]
    X = np.array([[a * sig, 0, 0.5 * a * sig, 0, 0.02, 2e-4] for a in (0.5, 2.0, 5.0, 9.0)])
    nt = 20
    xg, sg, lg, pg = tab.track_host(X.copy(), nt)
    xr = X.copy()
    st = np.ones(4, dtype=np.int32)
    lt_ = np.zeros(4, dtype=np.int32)
    lp = np.zeros(4, dtype=np.int32)
    from ctypes import POINTER, c_double, c_int
    ref_oracle.L.ref_track(ref_oracle.line, xr.ctypes.data_as(POINTER(c_double)), 4, nt,
                           st.ctypes.data_as(POINTER(c_int)), lt_.ctypes.data_as(POINTER(c_int)),
                           lp.ctypes.data_as(POINTER(c_int)))
    assert np.array_equal(sg, st) and np.array_equal(lg, lt_) and np.array_equal(pg, lp)
    ok = sg == 1
    floor = np.maximum(np.sqrt(np.mean(xr[ok] ** 2, axis=0)), 1e-300)
    assert np.all(np.abs(xg[ok] - xr[ok]) <= 1e-12 * np.maximum(np.abs(xr[ok]), floor))


def test_bmad_reader_matches_reference(tmp_path, ref_oracle):
    api.Set_RefPartEnergy(*HSR_ENERGY)
    ref_oracle.L.ref_set_ref_energy(*HSR_ENERGY)
    line = api.Line()
    line.read_bmad(str(hsr_table(tmp_path)))
    ref_oracle.read_bmad(str(hsr_table(tmp_path, numeric_only=True)))
    compare_lines(line, ref_oracle)
    types = [line.Cell(i).TYPE for i in range(line.Ncell)]
    assert types.count("PATCH") == 34 and types.count("SOLEN") == 2


def test_bmad_reader_against_printed_orbit_table(tmp_path):
    """Names, count and S positions of the elements equal the reference's
    printed table (6 significant digits).  That table came from an older
    reader: monitors and solenoids (KS = 0, a drift either way) print as
    DRIFT there."""
    api.Set_RefPartEnergy(*HSR_ENERGY)
    line = api.Line()
    line.read_bmad(str(hsr_table(tmp_path)))
    names, types, S, _ = hsr_orbit0()
    assert line.Ncell == len(names) == 2836
    assert [line.Cell(i).NAME for i in range(line.Ncell)] == names
    ours = [line.Cell(i).TYPE for i in range(line.Ncell)]
    for a, b in zip(ours, types):
        assert a == b or (a in ("BPM", "SOLEN") and b == "DRIFT"), (a, b)
    s = np.array([line.Cell(i).geometry()["S"] for i in range(line.Ncell)])
    assert np.all(np.abs(s - S) <= 5e-6 * np.abs(S) + 1e-9)


def test_bmad_read_line_tracks_like_reference(tmp_path, ref_oracle, port_oracle):
    """The C restatement on the line our reader built equals the reference's
    Track() on the line the reference's reader built, through every element
    of the HSR table (patches and solenoids included), bit for bit."""
    api.Set_RefPartEnergy(*HSR_ENERGY)
    line = api.Line()
    line.read_bmad(str(hsr_table(tmp_path)))
    lat = lt.Lattice("hsr", lt.specs_from_line(line), HSR_ENERGY[0])
    port_oracle.build(lat)
    ref_oracle.L.ref_set_ref_energy(*HSR_ENERGY)
    ref_oracle.L.ref_set_flags(0, 0)
    ref_oracle.read_bmad(str(hsr_table(tmp_path, numeric_only=True)))
    x0 = np.load(GOLDEN / "hsr_orbit_ref.npz")["orbit"][-1]
    for d in ([0, 0, 0, 0, 0, 0], [-3e-4, 1e-6, 2e-4, -1e-6, 0.01, 2e-4]):
        a = ref_oracle.track_dump(x0 + np.array(d), 2)
        b = port_oracle.track_dump(x0 + np.array(d), 2)
        assert a[1:4] == b[1:4]
        assert np.array_equal(a[4], b[4])


def _bmad_row(name, key, s=0.0, l=0.0, angle=0.0, e1=0.0, e2=0.0, xoff=0.0, zoff=0.0, xpitch=0.0, knl=None,
              knsl=None, ks=0.0, hkick=0.0, vkick=0.0, ncol=None):
    knl = list(knl or []) + [0.0] * (11 - len(knl or []))
    knsl = list(knsl or []) + [0.0] * (11 - len(knsl or []))
    vals = [s, l, angle, angle, e1, e2, 0.0, xoff, zoff, xpitch]
    for a, b in zip(knl, knsl):
        vals += [a, b]
    vals += [ks, hkick, vkick]
    if ncol is not None:
        vals = vals[:ncol]
    return f"{name} {key} " + " ".join(repr(float(v)) for v in vals) + "\n"


def test_bmad_reader_every_key_matches_reference(tmp_path, ref_oracle):
    """Every key Read_BMAD_Lattice maps (simtrack.cpp:14100-14230), the bend
    variants it chooses between, and a short row (missing fields keep the
    previous row's values, the first missing one reads as 0), read by both
    readers and compared element by element."""
    rows = ["# header line\n",
            _bmad_row("B0", "Beginning_Ele"),
            _bmad_row("D1", "Drift", l=1.5),
            _bmad_row("SB_MULT", "Sbend", l=2.0, angle=0.0, knl=[1e-3, 0.02, 0.3]),
            _bmad_row("SB_G", "Sbend", l=2.0, angle=0.01, knl=[0.0102], e1=0.001, e2=0.002),
            _bmad_row("SB_S", "Sbend", l=2.0, angle=0.01, knl=[0.01], e1=0.003),
            _bmad_row("SB_M", "Sbend", l=2.0, angle=0.01, knl=[0.01, 0.02, 0.5], knsl=[0.0, 0.0, 0.1]),
            _bmad_row("RB_S", "RBEND", l=1.0, angle=0.02),
            _bmad_row("RB_M", "RBEND", l=1.0, angle=0.02, knl=[0.0, 0.05]),
            _bmad_row("Q1", "Quadrupole", l=1.1, knl=[0.0, 0.12], knsl=[0.0, 0.001]),
            _bmad_row("S1", "Sextupole", l=0.3, knl=[0.0, 0.0, 0.7], knsl=[0.0, 0.0, 0.02]),
            _bmad_row("O1", "OCTUPOLE", l=0.2, knl=[0.0, 0.0, 0.0, 9.0]),
            _bmad_row("HK", "HKICKER", l=0.1, hkick=1e-5),
            _bmad_row("VK", "VKICKER", l=0.1, vkick=-2e-5),
            _bmad_row("K1", "Kicker", l=0.2, hkick=3e-6, vkick=4e-6),
            _bmad_row("HK_MIXED", "Hkicker", l=0.1, hkick=1e-5),
            _bmad_row("M0", "Multipole", knl=[0.0, 0.01, 0.2, 3.0], knsl=[0.0, 0.0, 0.1]),
            _bmad_row("MK", "Multipole", knl=[2e-4, 0.01]),
            _bmad_row("HM", "HMONITOR", l=0.1),
            _bmad_row("VM", "VMONITOR", l=0.1),
            _bmad_row("BPM1", "Monitor", l=0.2),
            _bmad_row("MK1", "MARKER"),
            _bmad_row("SOL0", "Solenoid", l=0.0, ks=0.1),
            _bmad_row("SOL1", "Solenoid", l=2.0, ks=0.1),
            _bmad_row("RF1", "RFcavity", l=0.5),
            _bmad_row("BB", "BEAMBEAM"),
            _bmad_row("P1", "Patch", xoff=0.01, zoff=-0.002, xpitch=0.02),
            _bmad_row("PIPE", "Pipe", l=0.7),
            _bmad_row("Q2", "Quadrupole", l=1.0, knl=[0.0, -0.1]),
            # short row: S, L, ANGLE given, ANGLE1 missing (reads 0), the rest as in Q2
            _bmad_row("Q3", "Quadrupole", s=1.0, l=0.9, angle=0.0, ncol=3),
            _bmad_row("END", "Marker")]
    path = tmp_path / "every_key.tab"
    path.write_text("".join(rows))
    api.Set_RefPartEnergy(100.0, 938.27201, 1, 1)
    ref_oracle.L.ref_set_ref_energy(100.0, 938.27201, 1.0, 1.0)
    line = api.Line()
    line.read_bmad(str(path))
    ref_oracle.read_bmad(str(path))
    compare_lines(line, ref_oracle)
    types = [line.Cell(i).TYPE for i in range(line.Ncell)]
    for t in ("MULT", "GSBEND", "SBEND", "SBENDMULT", "QUAD", "SEXT", "OCT", "HKICKER", "VKICKER", "KICKER", "HBPM",
              "VBPM", "BPM", "MARKER", "SOLEN", "RFCAV", "BEAMBEAM", "PATCH", "DRIFT"):
        assert t in types, t
    names = [line.Cell(i).NAME for i in range(line.Ncell)]
    assert "MK_tb" in names  # a multipole with K0L becomes a short bend
    q3 = line.Cell(names.index("Q3"))
    assert q3.GetP("K1L") == -0.1  # carried over from the previous row
