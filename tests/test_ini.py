"""parameters.ini reader of the C library (keys, defaults and checks of the
reference's python/finess/params specs).  Runs on CPU."""
import os

import pytest

from conftest import ROOT
from finess_b200._abi import FIN_BC_TRANSMISSIVE, FIN_PREC_FP64, FIN_TS_RK, FIN_WENO_Z
from finess_b200.solver import FinError, params_from_ini

INI = os.path.join(ROOT, "tests", "data", "riemann4q.ini")


@pytest.fixture(scope="module", autouse=True)
def built():
    from finess_b200.build import build
    build()


def test_reads_application_ini():
    p = params_from_ini(INI)
    assert (p.mx, p.my, p.mbc, p.meqn, p.nout) == (64, 64, 3, 5, 4)
    assert p.tfinal == 0.8 and p.initial_dt == 1e-4 and p.desired_cfl == 0.4 and p.max_cfl == 0.45
    assert p.time_stepping_method == FIN_TS_RK and p.time_order == 3 and p.space_order == 5
    assert p.weno_version == FIN_WENO_Z and p.epsilon == 1e-6 and p.alpha_scaling == 1.1
    assert p.global_alpha == 1 and p.source_term == 0 and p.gamma == 1.4
    assert p.bc_xlow == FIN_BC_TRANSMISSIVE and p.precision == FIN_PREC_FP64


def _variant(tmp_path, old, new):
    s = open(INI).read()
    assert old in s
    f = tmp_path / "p.ini"
    f.write_text(s.replace(old, new))
    return str(f)


@pytest.mark.parametrize("old,new,msg", [
    ("max_cfl     = 0.45", "max_cfl     = 0.3", "max_cfl should >= finess.desired_cfl"),
    ("initial_dt  = 1.0e-4", "initial_dt  = 0", "initial_dt should > 0"),
    ("alpha_scaling = 1.1", "alpha_scaling = 0.9", "alpha_scaling should >= 1"),
    ("xhigh =  1.0e0", "xhigh = -1.0", "xhigh should > grid.xlow"),
    ("weno_version = Z", "weno_version = Q", "unknown weno_version"),
    ("mx    = 64", "mx    = sixty", "not an integer"),
    ("source_term = false", "source_term = maybe", "not a bool"),
    ("nv          = 500000", "", "missing parameter finess.nv"),
])
def test_checks_fail_like_the_reference(tmp_path, old, new, msg):
    with pytest.raises(FinError) as e:
        params_from_ini(_variant(tmp_path, old, new))
    assert msg in str(e.value)


def test_defaults_when_optional_keys_absent(tmp_path):
    f = _variant(tmp_path, "global_alpha = true", "")
    p = params_from_ini(f)
    assert p.global_alpha == 0      # finess.py:13-17 default False
