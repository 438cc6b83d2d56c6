"""Generates the golden fixtures in this directory from the SimTrack
reference itself (test infrastructure).

Needs the compiled reference oracle (make -C oracle ref, which reads the
reference source in place).  For each fixture lattice it records, per
particle, Track()'s loss outputs and the six coordinates after every element
for a few sampled turns, as produced by the reference's own element Pass
functions.  The fixtures let the C restatement be pinned on machines where
the reference cannot be built.  It also copies the reference's Example1 RHIC lattice and its Example2 HSR
lattice table and its printed closed orbit (compressed) and records the
reference's closed orbit for that table.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))

import oracle_bridge  # noqa: E402
from lattice_zoo import spin_particles, spin_zoo, zoo, zoo_particles  # noqa: E402
from simtrack_b200.lattices import fodo_ring  # noqa: E402


def lattice_for(name: str):
    if name == "zoo":
        return zoo()
    if name == "fodo100":
        return fodo_ring()
    raise KeyError(name)


CASES = {
    "zoo": dict(x0=zoo_particles(), nturn=3, sample_turns=[0, 1, 2]),
    "fodo100": dict(x0=np.array([[1e-3, 0, 5e-4, 0, 0, 0], [4e-3, 1e-5, -3e-3, 0, 0.01, 5e-4]]), nturn=40,
                    sample_turns=[0, 39]),
}


def tune_signals(n: int = 512, count: int = 12, seed: int = 7):
    """Turn-by-turn-like test signals: a betatron line with random tune,
    phase and amplitude, a weaker second line, slow amplitude modulation and
    noise; px is the matching conjugate signal."""
    rng = np.random.default_rng(seed)
    i = np.arange(n)
    xs, pxs = [], []
    for k in range(count):
        q1 = rng.uniform(0.21, 0.44)
        q2 = rng.uniform(0.05, 0.48)
        a1 = rng.uniform(1e-4, 1e-2)
        ph = rng.uniform(0, 2 * np.pi)
        mod = 1.0 + 0.05 * np.sin(2 * np.pi * i * rng.uniform(0.001, 0.01))
        x = a1 * mod * np.cos(2 * np.pi * q1 * i + ph) + 0.1 * a1 * np.cos(2 * np.pi * q2 * i)
        px = -a1 * mod * np.sin(2 * np.pi * q1 * i + ph)
        x = x + rng.normal(0, 1e-3 * a1, n)
        xs.append(x)
        pxs.append(px)
    return np.array(xs), np.array(pxs)


# tune windows of the fixture: (lower, upper, with px)
TUNE_WINDOWS = [(0.2, 0.45, False), (0.0, 0.5, False), (0.0, 1.0, True)]


# The reference's Example2 inputs: the HSR lattice as a Bmad table and the
# closed orbit the reference printed for it (Print_Orbit after Cal_Optics).
_REF = oracle_bridge.ref_source_dir()
EXAMPLE2 = _REF / "Example2" if _REF else Path("/nonexistent")
# The reference's Example1 RHIC lattice (MAD-X TFS, 6,858 elements), the
# table too large for one shared-memory copy that the segmented-staging tests
# track on the GPU.
EXAMPLE1 = _REF / "Example1" if _REF else Path("/nonexistent")
HSR_ENERGY = (275000. / 938.27201, 938.27201, 1.0, 1.0)  # Set_RefPartEnergy, Example2/DA_cal.cpp:613


def numeric_rows(text: str) -> str:
    """The table without rows whose S column is not a number (its
    column-name and unit lines), which the reference's reader would turn
    into drifts of an undefined length."""
    rows = text.splitlines(True)
    keep = [rows[0]]
    for r in rows[1:]:
        t = r.split()
        try:
            float(t[2])
        except (IndexError, ValueError):
            continue
        keep.append(r)
    return "".join(keep)


def hsr_fixtures(ref) -> None:
    """Compressed copies of Example2's Bmad table and orbit0.dat, and the
    reference's own Read_BMAD_Lattice + Cal_Orbit_Num(0) on that table."""
    import lzma
    import tempfile
    tab = (EXAMPLE2 / "SimTrack_hsr_base_forIRerr.tab").read_text()
    (HERE / "hsr_bmad.tab.xz").write_bytes(lzma.compress(tab.encode(), preset=9))
    (HERE / "hsr_orbit0.dat.xz").write_bytes(lzma.compress((EXAMPLE2 / "orbit0.dat").read_bytes(), preset=9))
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "hsr.tab"
        path.write_text(numeric_rows(tab))
        ref.L.ref_set_ref_energy(*HSR_ENERGY)
        ref.L.ref_set_flags(0, 0)
        ref.read_bmad(str(path))
        orbit = ref.cal_orbit(0.0)
    np.savez_compressed(HERE / "hsr_orbit_ref.npz", orbit=orbit, energy=np.array(HSR_ENERGY))
    print("wrote hsr fixtures")


def rhic_example1_fixture() -> None:
    import lzma
    (HERE / "rhic_example1.tfs.xz").write_bytes(lzma.compress((EXAMPLE1 / "parameters_input").read_bytes(), preset=9))
    print("wrote rhic_example1.tfs.xz")


def main():
    from oracle_bridge import RefOracle
    if len(sys.argv) > 1 and sys.argv[1] == "rhic_example1":
        rhic_example1_fixture()
        return
    ref = RefOracle()
    rhic_example1_fixture()
    hsr_fixtures(ref)
    xs, pxs = tune_signals()
    tunes = np.array([[ref.fine_tune(x, px if w else None, lo, hi) for lo, hi, w in TUNE_WINDOWS]
                      for x, px in zip(xs, pxs)])
    np.savez_compressed(HERE / "fine_tune.npz", x=xs, px=pxs, windows=np.array(TUNE_WINDOWS, dtype=np.float64),
                        tunes=tunes)
    print("wrote fine_tune")
    # spin tracking: Track_Spin's per-element x[9] on the spin zoo
    lat = spin_zoo()
    ref.build(lat)
    x9 = spin_particles()
    nturn = lat.meta["turns"]
    dumps, loss = [], []
    for x0 in x9:
        _, st, lt, lp, d = ref.track_spin_dump(x0, nturn)
        dumps.append(d)
        loss.append((st, lt, lp))
    np.savez_compressed(HERE / "spin_zoo.npz", x0=x9, nturn=nturn, dump=np.array(dumps),
                        loss=np.array(loss, dtype=np.int64))
    print("wrote spin_zoo")
    for name, c in CASES.items():
        ref.build(lattice_for(name))
        dumps, loss = [], []
        for x0 in c["x0"]:
            _, st, lt, lp, d = ref.track_dump(x0, c["nturn"])
            dumps.append(d[c["sample_turns"]])
            loss.append((st, lt, lp))
        np.savez_compressed(HERE / f"{name}.npz", lattice=name, nturn=c["nturn"], x0=c["x0"],
                            sample_turns=np.array(c["sample_turns"]), dump=np.array(dumps),
                            loss=np.array(loss, dtype=np.int64))
        print("wrote", name)


if __name__ == "__main__":
    main()
