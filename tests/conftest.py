import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


def params_from_json(s):
    from finess_b200._abi import FinParams
    d = json.loads(str(s))
    p = FinParams()
    for k, v in d.items():
        setattr(p, k, v)
    return p


def golden_cases(prefix):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz"))):
        out.append(pytest.param(f, id=os.path.basename(f)[:-4]))
    return out


def load_golden(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["p"] = params_from_json(d.pop("params"))
    return d


def interior(p, a):
    mb = p.mbc
    return a[mb:mb + p.mx, mb:mb + p.my]


def rel_linf(a, b):
    """max|a-b| / max|b| (relative L-infinity)."""
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle import RefLib
    if not RefLib.available():
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    return RefLib()
