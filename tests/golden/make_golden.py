"""Generates the golden fixtures in this directory from the SimTrack
reference itself (test infrastructure).

Needs the compiled reference oracle (make -C oracle ref, which reads the
reference source in place).  For each fixture lattice it records, per
particle, Track()'s loss outputs and the six coordinates after every element
for a few sampled turns, as produced by the reference's own element Pass
functions.  The fixtures let the C restatement be pinned on machines where
the reference cannot be built.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))

from lattice_zoo import zoo, zoo_particles  # noqa: E402
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


def main():
    from oracle_bridge import RefOracle
    ref = RefOracle()
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
