import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ck-bc_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200)")


def _ensure_built():
    if not os.path.exists(os.path.join(PKG, "libbcg.so")) or not os.path.exists(os.path.join(PKG, "bc2d")):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    for lib in ("liboracle.so", "libtrees_ref.so"):
        if not os.path.exists(os.path.join(ORACLE, lib)):
            subprocess.run(["make", "-s", "-C", ORACLE, lib], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "nx_golden.json")) as f:
        return json.load(f)
