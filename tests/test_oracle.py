"""The oracle is pinned before it is trusted (CPU only).

* The GSL shim's inverse normal CDF reproduces the N=11 strong-bunch slice
  table that BB6D hard-codes (simtrack.cpp:6593-6604) through the general
  centroid formula (6612-6619), and N=5 / N=7 centroids computed
  independently with Python's AS241 inverse normal CDF.
* The C restatement (oracle/port) is bit-identical to the compiled reference
  at every element: live when oracle/_ref is built, and against the golden
  fixtures in tests/golden/ (generated from the reference by
  tests/golden/make_golden.py) everywhere.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from lattice_zoo import patch_solen_zoo, zoo, zoo_particles
from simtrack_b200.lattices import fodo_ring

GOLDEN = Path(__file__).resolve().parent / "golden"

N11 = [1.7996765362153655, 1.1049618149811977, 0.75072324235797372, 0.47407703558819131, 0.23041113693387344, 0.,
       -0.23041113693387344, -0.47407703558819131, -0.75072324235797372, -1.1049618149811977, -1.7996765362153655]


def centroids(N, pinv):
    y = [pinv((i + 1) * 1.0 / N) for i in range(N - 1)]
    z = [0.0] * N
    c = math.sqrt(2.0 * 3.14159265)
    z[0] = N * (math.exp(-y[0] * y[0] / 2)) / c
    z[N - 1] = N * (0 - math.exp(-y[0] * y[0] / 2)) / c
    for i in range(1, N - 1):
        z[i] = N * (math.exp(-y[i] * y[i] / 2) - math.exp(-y[i - 1] * y[i - 1] / 2)) / c
    return z


def test_shim_pinv_reproduces_bb6d_table(ref_oracle):
    z = centroids(11, ref_oracle.pinv)
    assert max(abs(a - b) for a, b in zip(z, N11)) <= 1e-15


def test_shim_pinv_n5_n7(ref_oracle):
    from statistics import NormalDist
    inv = NormalDist().inv_cdf
    for n in (5, 7):
        z, zp = centroids(n, ref_oracle.pinv), centroids(n, inv)
        assert max(abs(a - b) for a, b in zip(z, zp)) <= 2e-15
    assert abs(centroids(5, ref_oracle.pinv)[0] - 1.3998096028387994) <= 2e-15


def test_shim_pinv_against_python_as241(ref_oracle):
    from statistics import NormalDist
    nd = NormalDist()
    rng = np.random.default_rng(7)
    for p in list(rng.random(2000)) + [1e-300, 1e-20, 0.02425, 0.5, 0.97575, 1 - 1e-12]:
        a, b = ref_oracle.pinv(float(p)), nd.inv_cdf(float(p))
        assert abs(a - b) <= 4e-16 * max(1.0, abs(b))


def _same(a, b):
    return np.array_equal(np.nan_to_num(a, nan=7.0), np.nan_to_num(b, nan=7.0))


@pytest.mark.parametrize("which", ["zoo", "fodo", "patch_solen"])
def test_port_matches_reference_every_element(which, ref_oracle, port_oracle):
    if which == "zoo":
        lat, X, nturn = zoo(), zoo_particles(), 3
    elif which == "patch_solen":
        lat, X, nturn = patch_solen_zoo(), zoo_particles(), 3
    else:
        lat = fodo_ring()
        X = np.array([[1e-3, 0, 5e-4, 0, 0, 0], [4e-3, 1e-5, -3e-3, 0, 0.01, 5e-4]])
        nturn = 40
    ref_oracle.build(lat)
    port_oracle.build(lat)
    for x0 in X:
        a = ref_oracle.track_dump(x0, nturn)
        b = port_oracle.track_dump(x0, nturn)
        assert a[1:4] == b[1:4]
        assert _same(a[4], b[4])


def test_port_matches_golden(port_oracle):
    """Bit-level agreement with outputs of the reference itself, run here."""
    from golden.make_golden import CASES, lattice_for
    files = [GOLDEN / f"{name}.npz" for name in CASES]
    assert all(f.exists() for f in files), "golden fixtures missing"
    for f in files:
        g = np.load(f)
        lat = lattice_for(str(g["lattice"]))
        port_oracle.build(lat)
        nturn = int(g["nturn"])
        for i, x0 in enumerate(g["x0"]):
            a = port_oracle.track_dump(x0, nturn)
            assert (a[1], a[2], a[3]) == tuple(int(v) for v in g["loss"][i]), f.name
            assert _same(a[4][g["sample_turns"]], g["dump"][i]), f"{f.name} particle {i}"
