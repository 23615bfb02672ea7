import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the oracle (CPU) if missing; the solver library must be prebuilt."""
    oracle_so = os.path.join(ROOT, "oracle", "libmcg_oracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "libmcg_oracle.so"], check=True)
    yield


@pytest.fixture(scope="session")
def has_gpu():
    from multicomponent_color_gradient_b200 import device_count

    return device_count() > 0


def ref_binary(case: str):
    """Path of the reference's own CUDA build for a case, or None if not built."""
    p = os.path.join(ROOT, "oracle", "_ref", "ref_" + case)
    return p if os.path.exists(p) else None


def reference_dir():
    """The reference checkout: MCG_REFERENCE_DIR, else the directory
    oracle/build_ref.sh compiled the reference from (recorded in
    oracle/_ref/REFERENCE_DIR), when it exists on this machine; else None."""
    d = os.environ.get("MCG_REFERENCE_DIR")
    rec = os.path.join(ROOT, "oracle", "_ref", "REFERENCE_DIR")
    if not d and os.path.exists(rec):
        d = open(rec).read().strip()
    return d if d and os.path.isdir(d) else None
