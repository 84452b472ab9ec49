"""Frame files, conservation.dat and restart from device state against the
reference's own output routines (lib/2d/Output.cpp, ConSoln.cpp, compiled
into oracle/_ref/libfinref_io.so): the frame files byte for byte, the
conservation totals to the reference's summation error, the restart bit for
bit."""
import os

import numpy as np
import pytest

from conftest import interior
from finess_b200 import problems as P
from finess_b200._abi import FIN_WENO_Z

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ioref():
    from oracle import IoRefLib
    if not IoRefLib.available():
        pytest.skip("oracle/_ref/libfinref_io.so not built (needs the reference checkout)")
    return IoRefLib()


def _state(n=37, my=50, seed=4, maux=0):
    p = P.riemann_params(n=n, weno=FIN_WENO_Z)
    p.my = my
    p.maux = maux
    p.nout = 7
    q = P.random_riemann_state(p, np.random.default_rng(seed))
    # values that exercise the conversion: signed zero, subnormal, tiny and
    # three-digit exponents, in the momentum components
    mb = p.mbc
    q[mb, mb, 1] = -0.0
    q[mb + 1, mb, 2] = 5e-324
    q[mb + 2, mb + 3, 3] = -1.25e-300
    q[mb + 3, mb + 1, 3] = 7.5e-101
    q[mb + 4, mb + 2, 1] = 123456.78901234567
    return p, q


def _read_values(path, ncomp, mx, my):
    with open(path) as f:
        t = float(f.readline())
        v = np.array([float(x) for x in f.read().split()])
    return t, v.reshape(ncomp, my, mx).transpose(2, 1, 0)


@pytest.mark.parametrize("maux", [0, 1])
def test_frame_files_match_reference(tmp_path, ioref, maux):
    from finess_b200.solver import Solver
    p, q = _state(maux=maux)
    t = 0.123456789012345678
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    with Solver(p) as s:
        s.set_state(q, t)
        s.output_frame(3, str(ours))
        s.output_wait()
    ioref.output(p, str(ref), q, t, 3)
    for name in ("q0003.dat", "a0003.dat"):
        a = (ours / name).read_bytes()
        b = (ref / name).read_bytes()
        assert a == b, name
    assert len((ours / "q0003.dat").read_bytes()) == 25 * (1 + 5 * p.mx * p.my)


def test_conservation_file_matches_reference(tmp_path, ioref):
    """A line at t = 0 and one per accepted step; t printed identically, the
    totals within the reference's own summation error."""
    from finess_b200.solver import Solver
    p = P.riemann_params(n=40, weno=FIN_WENO_Z)
    p.my = 33
    q0 = P.random_riemann_state(p, np.random.default_rng(9))
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    from finess_b200.batch import first_dt
    dtv = np.array([0.0, first_dt(p, q0), p.max_dt])
    dxdy = (p.xhigh - p.xlow) / p.mx * (p.yhigh - p.ylow) / p.my
    abs_sums = []
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        s.set_conservation_file(str(ours))
        s.write_conservation()
        q, t = s.get_state()
        ioref.consoln(p, str(ref), q, t)
        abs_sums.append(np.abs(dxdy * interior(p, q)).sum(axis=(0, 1)))
        for _ in range(6):
            dtv, n = s.advance(1.0, dtv, 1)
            assert n == 1
            q, t = s.get_state()
            ioref.consoln(p, str(ref), q, t)
            abs_sums.append(np.abs(dxdy * interior(p, q)).sum(axis=(0, 1)))
        s.set_conservation_file(None)
    a = (ours / "conservation.dat").read_text().splitlines()
    b = (ref / "conservation.dat").read_text().splitlines()
    assert len(a) == len(b) == 7
    n = p.mx * p.my
    for la, lb, sabs in zip(a, b, abs_sums):
        fa, fb = la.split(), lb.split()
        assert fa[0] == fb[0]                      # t
        va, vb = np.array(fa[1:], float), np.array(fb[1:], float)
        # the reference's in-order sum is within n eps sum|x| of the exact
        # one, the compensated sum within 2 eps |total|; both printed to 17 digits
        bound = (n + 4) * 1.12e-16 * sabs + 1e-16 * np.abs(vb)
        assert np.all(np.abs(va - vb) <= bound), (la, lb)
        assert len(la) == len(lb)


def test_restart_round_trip(tmp_path, ioref):
    """A frame written by this library or by the reference reads back as the
    same state, bit for bit, with its time."""
    from finess_b200.solver import Solver
    p, q = _state()
    t = 0.0625
    ioref.output(p, str(tmp_path), q, t, 1)
    with Solver(p) as s:
        s.set_state(q, t)
        s.output_frame(2, str(tmp_path))
        s.output_wait()
    for name in ("q0001.dat", "q0002.dat"):
        with Solver(p) as s:
            s.read_frame(str(tmp_path / name))
            q2, t2 = s.get_state()
        assert t2 == t
        assert np.array_equal(interior(p, q2), interior(p, q)), name


def test_output_is_asynchronous_and_leaves_the_run_unchanged(tmp_path):
    """The frame holds the state at the call even though the solver steps on
    while it is written, and the run matches one without output."""
    from finess_b200.batch import first_dt
    from finess_b200.solver import Solver
    p = P.riemann_params(n=64, weno=FIN_WENO_Z)
    q0 = P.random_riemann_state(p, np.random.default_rng(2))
    dt0 = first_dt(p, q0)
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        s.advance(1.0, np.array([0.0, dt0, p.max_dt]), 2)
        qa, ta = s.get_state()
        s.output_frame(5, str(tmp_path))
        s.advance(1.0, np.array([0.0, dt0, p.max_dt]), 3)
        s.output_wait()
        qb, _ = s.get_state()
    tf, vf = _read_values(str(tmp_path / "q0005.dat"), 5, p.mx, p.my)
    assert tf == ta
    assert np.array_equal(vf, interior(p, qa))
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        s.advance(1.0, np.array([0.0, dt0, p.max_dt]), 2)
        s.advance(1.0, np.array([0.0, dt0, p.max_dt]), 3)
        qc, _ = s.get_state()
    assert np.array_equal(interior(p, qb), interior(p, qc))


def test_bad_output_directory_reports_an_error(tmp_path):
    from finess_b200.solver import FinError, Solver
    p, q = _state()
    with Solver(p) as s:
        s.set_state(q, 0.0)
        s.output_frame(0, str(tmp_path / "missing" / "dir"))
        with pytest.raises(FinError):
            s.output_wait()
        with pytest.raises(FinError):
            s.read_frame(str(tmp_path / "nothing.dat"))
