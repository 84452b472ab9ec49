"""qhelp.dat (needs no device) against the reference's own WriteQhelp
(lib/2d/WriteQhelp.cpp, compiled into oracle/_ref/libfinref_io.so), byte for
byte."""
import pytest

from finess_b200 import problems as P


@pytest.fixture(scope="module")
def ioref():
    from oracle import IoRefLib
    if not IoRefLib.available():
        pytest.skip("oracle/_ref/libfinref_io.so not built (needs the reference checkout)")
    return IoRefLib()


@pytest.mark.parametrize("case", ["riemann", "shock_entropy", "wide"])
def test_qhelp_matches_reference(tmp_path, ioref, case):
    from finess_b200.solver import write_qhelp
    if case == "riemann":
        p = P.riemann_params(n=4096)
    elif case == "shock_entropy":
        p = P.shock_entropy_params()
    else:
        p = P.riemann_params(n=12)
        p.xlow, p.xhigh, p.ylow, p.yhigh = -123456.789, 9.87654321e-5, -1e-300, 2.5e17
        p.maux, p.nout = 3, 123456789
    p.nout = p.nout or 10
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    write_qhelp(p, str(ours))
    ioref.qhelp(p, str(ref))
    assert (ours / "qhelp.dat").read_bytes() == (ref / "qhelp.dat").read_bytes()
