"""The generic-physics restatement (oracle/generic_oracle.py), the checker of
the device callback surface, pinned on the CPU: with the reference's own
Euler callbacks restated in their formula order it reproduces the
reference's golden ConstructL fixtures (L, smax and the global wave speeds)."""
import numpy as np
import pytest

from conftest import golden_cases, interior, load_golden, rel_linf


@pytest.mark.parametrize("path", golden_cases("constructl_"))
def test_generic_restatement_reproduces_reference_construct_l(path):
    import generic_oracle as G
    g = load_golden(path)
    p = g["p"]
    ph = G.EulerCallbacks(p.gamma)
    L, smax = G.construct_l(ph, p, g["q"])
    # the same formulas in the same order: equal but for numpy's pow
    assert rel_linf(interior(p, L), interior(p, g["L"])) <= 1e-14
    assert np.array_equal(smax, g["smax"])
    if p.global_alpha:
        assert G.global_wave_spd(ph, p, g["q"]) == tuple(g["alpha"])


def test_constant_state_has_zero_rhs():
    import generic_oracle as G
    from finess_b200 import problems as P
    p = P.vortex_params(n=12)
    p.meqn = 3
    q = np.zeros((p.mx + 2 * p.mbc, p.my + 2 * p.mbc, 3))
    q[..., 0], q[..., 1], q[..., 2] = 2.0, 0.3, -0.7
    L, smax = G.construct_l(G.AdvAcousticsCallbacks(4.0, 1.5, 0.4, -0.25), p, q)
    assert np.max(np.abs(L)) < 1e-14
    assert np.all(smax[p.mbc:p.mbc + p.mx, p.mbc:p.mbc + p.my, 0] > 0)
