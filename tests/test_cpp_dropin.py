"""A C++ driver written like the reference's Example1/DA_cal.cpp (9-62)
against include/simtrack_b200.hpp: it sets the reference particle, builds the
RHIC-like ring element by element with `new QUAD(...)`, `SetP("Nint", ...)`
and `Line::Append`, and calls Track_DA (simtrack.cpp:21389-21441) for 64
turns.  The only lines that differ from a driver of the reference are the
include, `using namespace stb;` and the link line.

CPU: the generated driver compiles and links against the library.
GPU: its DA-output file equals, byte for byte, the file the reference's own
Track_DA writes for the same ring.
"""
import math
import shutil
import subprocess
from pathlib import Path

import pytest

from simtrack_b200 import lattices as lt

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "simtrack_b200" / "_lib"
NTURN = 64
DELTAP = 5e-4


def _lit(v: float) -> str:
    return repr(float(v))  # shortest round-trip form; the C++ parser restores the same double


def _ctor(e) -> str:
    n = f'"{e.name}"'
    a = [_lit(v) for v in e.args]
    if e.type in ("DRIFT", "MARKER"):
        return f"new {e.type}({n}, {a[0]})"
    if e.type == "SBEND":
        return f"new SBEND({n}, {a[0]}, {a[1]}, {a[2]}, {a[3]})"
    if e.type in ("QUAD", "SEXT"):
        return f"new {e.type}({n}, {a[0]}, {a[1]}, {a[2]})"
    if e.type == "RFCAV":
        return f"new RFCAV({n}, {a[0]}, {a[1]}, {a[2]}, {a[3]})"
    if e.type == "BEAMBEAM":
        return (f"new BEAMBEAM({n}, {int(e.args[0])}, {a[1]}, {a[2]}, {a[3]}, {int(e.args[4])}, "
                f"{', '.join(a[5:11])})")
    raise ValueError(f"no constructor mapping for {e.type}")


def driver_source(lat) -> str:
    s = lat.meta["sigma_ip"]
    body = []
    for e in lat.elements:
        if e.type == "MULT":
            body.append("  {\n"
                        f"    const double knl[11] = {{{', '.join(_lit(v) for v in e.args[1:12])}}};\n"
                        f"    const double knsl[11] = {{{', '.join(_lit(v) for v in e.args[12:23])}}};\n"
                        f'    temp_element = new MULT("{e.name}", {_lit(e.args[0])}, knl, knsl);\n'
                        "  }")
        else:
            body.append(f"  temp_element = {_ctor(e)};")
        for k, v in e.setp.items():
            body.append(f'  temp_element->SetP("{k}", {_lit(v)});')
        body.append("  ring.Append(temp_element);")
    lines = "\n".join(body)
    return f"""#include <cmath>
#include <iostream>
#include "simtrack_b200.hpp"

using namespace std;
using namespace stb;

int main(int argc, char **argv)
{{
  Line ring;
  Element *temp_element;

  //----set global parameters for protons
  Set_RefPartEnergy({_lit(lat.gamma)}, {_lit(lat.E0)}, {_lit(lat.Q)}, {_lit(lat.A)});

  //---build the lattice
{lines}

  //---DA tracking
  int nturn = {NTURN};
  double deltap = {_lit(DELTAP)};
  double sigmax0 = {_lit(s)};
  double sigmay0 = {_lit(s)};
  Track_DA(ring, nturn, deltap, sigmax0, sigmay0, argc > 1 ? argv[1] : "DA-output.dat");
  return 0;
}}
"""


def build_driver(tmp_path: Path, lat) -> Path:
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    from simtrack_b200 import _native
    if not _native.LIB_PATH.exists():
        from simtrack_b200 import build
        build.build()
    src = tmp_path / "DA_cal.cpp"
    src.write_text(driver_source(lat))
    exe = tmp_path / "DA_cal"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(src), "-o", str(exe),
                    f"-L{LIBDIR}", "-l:libsimtrack_b200.so", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


@pytest.fixture(scope="module")
def ring():
    return lt.rhic_like_ring(seed=1)


def test_driver_compiles_and_links(tmp_path, ring):
    exe = build_driver(tmp_path, ring)
    assert exe.exists()
    src = (tmp_path / "DA_cal.cpp").read_text()
    assert src.count("ring.Append(") == len(ring.elements)


@pytest.mark.gpu
def test_driver_da_file_equals_reference(tmp_path, ring, ref_oracle):
    exe = build_driver(tmp_path, ring)
    ours = tmp_path / "DA-output.dat"
    subprocess.run([str(exe), str(ours)], check=True, cwd=tmp_path, timeout=600)
    ref_oracle.build(ring)
    theirs = tmp_path / "DA-ref.dat"
    s = ring.meta["sigma_ip"]
    ref_oracle.track_da(NTURN, DELTAP, s, s, str(theirs))
    assert ours.read_text() == theirs.read_text()
    assert len(ours.read_text().splitlines()) == 10
    assert math.isfinite(float(ours.read_text().split()[1]))
