"""pytest configuration: the `gpu` marker and shared oracle fixtures.

Tests marked gpu need a CUDA device; everything else runs on the CPU.  The
oracles are test infrastructure: the C restatement is (re)built from
oracle/port when its library is missing; the compiled reference
(oracle/_ref) is used when present and its tests are skipped otherwise.
"""
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

import oracle_bridge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def port_oracle():
    if not oracle_bridge.port_available():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "port"], check=True)
    return oracle_bridge.PortOracle()


@pytest.fixture(scope="session")
def ref_oracle():
    if not oracle_bridge.ref_available():
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")
    return oracle_bridge.RefOracle()


@pytest.fixture(scope="session")
def ref_cr_oracle():
    if not oracle_bridge.ref_available(cr=True):
        pytest.skip("compiled reference oracle with correctly rounded libm (oracle/_ref) not built here")
    return oracle_bridge.RefOracle(cr=True)


@pytest.fixture(scope="session")
def native_lib():
    from simtrack_b200 import _native
    if not _native.LIB_PATH.exists():
        from simtrack_b200 import build
        build.build()
    return _native.lib()
