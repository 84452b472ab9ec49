"""Initial data sampled on the device (fin_set_state_qinit: SampleFunction,
lib/2d/SampleFunction.cpp:62-125, with a QinitFunc functor) against

* the reference's own SampleFunction with its applications' own QinitFunc
  (apps/2d/euler/riemann_test and test_exact2, oracle/_ref), on ragged grids;
* the benchmark problems' host restatements (finess_b200/problems.py) at
  their full sizes.

Interior cells are compared (the device state has no ghost frame; the
reference's sampled ghosts are overwritten by SetBndValues before any stage).
Bars: bit-exact where the data are piecewise constant; 2e-15 relative
L-infinity where exp, pow or sin enter (CUDA's functions are within a couple
of ulps of the host's)."""
import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import (FIN_QINIT_RIEMANN4, FIN_QINIT_SHOCK_ENTROPY, FIN_QINIT_SHOCK_TUBE, FIN_QINIT_VORTEX,
                              FIN_QINIT_VORTEX_EXACT2)

pytestmark = pytest.mark.gpu
TOL_TRANSCENDENTAL = 2e-15


def _device(p, problem, prm=()):
    from finess_b200.solver import Solver
    with Solver(p) as s:
        s.set_state_qinit(problem, prm, 0.0)
        q, t = s.get_state()
    assert t == 0.0
    return q


def _ref(app):
    from oracle import RefQinit
    if not RefQinit.available(app):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    return RefQinit(app)


@pytest.mark.parametrize("opt", [1, 2])
def test_reference_shock_tube_app(opt):
    ref = _ref("riemann_test")
    p = P.riemann_params(n=37)
    p.my = 50
    qd = _device(p, FIN_QINIT_SHOCK_TUBE, [opt])
    qr = ref.sample(p, opt)
    assert np.array_equal(interior(p, qd), interior(p, qr))


def test_reference_vortex_app():
    ref = _ref("test_exact2")
    p = P.vortex_params(n=45)
    p.my = 38
    p.xlow, p.xhigh, p.ylow, p.yhigh = -5.0, 5.0, -5.0, 5.0
    qd = _device(p, FIN_QINIT_VORTEX_EXACT2)
    qr = ref.sample(p)
    assert rel_linf(interior(p, qd), interior(p, qr)) <= TOL_TRANSCENDENTAL


def test_benchmark_riemann4096_bit_exact():
    p = P.riemann_params(n=4096)
    qd = _device(p, FIN_QINIT_RIEMANN4)
    assert np.array_equal(interior(p, qd), interior(p, P.riemann_init(p)))


def test_riemann4_custom_states():
    rng = np.random.default_rng(4)
    p = P.riemann_params(n=33)
    p.my = 21
    xc, yc = 0.37, 0.61
    st = {k: (rng.uniform(0.1, 2), rng.uniform(-1.5, 1.5), rng.uniform(-1.5, 1.5), rng.uniform(0.02, 2))
          for k in ("ur", "ul", "ll", "lr")}
    prm = [xc, yc] + [v for k in ("ur", "ul", "ll", "lr") for v in st[k]]
    qd = _device(p, FIN_QINIT_RIEMANN4, prm)
    assert np.array_equal(interior(p, qd), interior(p, P.riemann_init(p, xc, yc, st)))


def test_benchmark_vortex200():
    p = P.vortex_params(n=200)
    qd = _device(p, FIN_QINIT_VORTEX)
    assert rel_linf(interior(p, qd), interior(p, P.vortex_exact(p))) <= TOL_TRANSCENDENTAL


def test_benchmark_shock_entropy8192x1024():
    p = P.shock_entropy_params(nx=8192, ny=1024)
    qd = _device(p, FIN_QINIT_SHOCK_ENTROPY)
    assert rel_linf(interior(p, qd), interior(p, P.shock_entropy_init(p))) <= TOL_TRANSCENDENTAL


def test_unknown_problem_and_bad_parameters_are_refused():
    from finess_b200.solver import FinError, Solver
    p = P.riemann_params(n=16)
    with Solver(p) as s:
        for problem, prm in ((99, ()), (FIN_QINIT_RIEMANN4, [0.5]), (FIN_QINIT_SHOCK_TUBE, ())):
            with pytest.raises(FinError):
                s.set_state_qinit(problem, prm)
