"""The batched solver against separate single-problem runs: per problem the
batch runs the same stage arithmetic and step control, so it must take the
same number of steps and agree with the separate run to rounding (the plain
FP64 form's 1e-12 bar; FP32 to FP32 rounding)."""
import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_PREC_FP32, FIN_PREC_FP64, FIN_WENO_Z

pytestmark = pytest.mark.gpu


def _problems(precision):
    rng = np.random.default_rng(3)
    params, states = [], []
    for n in (20, 33, 48, 17, 40):
        p = P.riemann_params(n=n, weno=FIN_WENO_Z)
        p.precision = precision
        params.append(p)
        states.append(P.random_riemann_state(p, rng))
    p = P.riemann_params(n=30, weno=FIN_WENO_Z)
    p.my = 25
    p.precision = precision
    params.append(p)
    states.append(P.random_riemann_state(p, rng))
    p = P.vortex_params(n=36, weno=FIN_WENO_Z)   # periodic, on another domain
    p.precision = precision
    params.append(p)
    states.append(P.vortex_exact(p))
    return params, states


@pytest.mark.parametrize("precision", [FIN_PREC_FP64, FIN_PREC_FP32])
def test_batch_equals_separate_runs(oracle, precision):
    from finess_b200.batch import Batch, first_dt
    from finess_b200.solver import Solver
    params, states = _problems(precision)
    states = [oracle.set_bnd(p, q) for p, q in zip(params, states)]
    tend = 0.05
    dts = np.array([first_dt(p, q) for p, q in zip(params, states)])
    with Batch(params) as b:
        for k, q in enumerate(states):
            b.set_state(k, q)
        dt_out, steps = b.solve(tend, dts)
        got = [b.get_state(k) for k in range(len(params))]
        st = b.stats()
    assert st["replays"] >= steps.max()
    for k, (p, q) in enumerate(zip(params, states)):
        with Solver(p) as s:
            s.set_state(q)
            dtv, n = s.FinSolveRK(tend, np.array([0.0, dts[k], p.max_dt]))
            qs, ts = s.get_state()
        qb, tb = got[k]
        tol = 1e-12 if precision == FIN_PREC_FP64 else 1e-5
        assert steps[k] == n, (k, steps[k], n)
        assert abs(dt_out[k] - dtv[1]) <= tol * dtv[1], (k, dt_out[k], dtv[1])
        assert abs(tb - ts) <= 1e-14 * max(1.0, abs(ts))
        assert rel_linf(interior(p, qb), interior(p, qs)) <= tol, k


@pytest.mark.parametrize("judge_every,judge_tol,every", [(4, 1e-3, 2), (3, 0.0, 1)])
def test_batch_hybrid_equals_separate_runs(oracle, judge_every, judge_tol, every):
    """The hybrid form batched: per problem the same indicator period, judge
    steps and reverts (judge_tol 0 reverts every judged step, so the plain
    attempts that follow and the buffer swap run too) as a separate hybrid
    run, the same steps, and the state to FP32 rounding."""
    from finess_b200.batch import Batch, first_dt, load_indicator
    from finess_b200.solver import Solver
    from finess_b200._abi import FIN_PREC_HYBRID
    ind = load_indicator()
    params, states = _problems(FIN_PREC_HYBRID)
    states = [oracle.set_bnd(p, q) for p, q in zip(params, states)]
    tend = 0.05
    dts = np.array([first_dt(p, q) for p, q in zip(params, states)])
    with Batch(params) as b:
        b.set_indicator(ind[0], ind[1], judge_every, judge_tol, every)
        for k, q in enumerate(states):
            b.set_state(k, q)
        dt_out, steps = b.solve(tend, dts)
        got = [b.get_state(k) for k in range(len(params))]
        hst = b.hybrid_stats()
    judges = reverts = 0
    for k, (p, q) in enumerate(zip(params, states)):
        with Solver(p) as s:
            s.set_indicator(ind[0], ind[1], judge_every, judge_tol, every)
            s.set_state(q)
            dtv, n = s.FinSolveRK(tend, np.array([0.0, dts[k], p.max_dt]))
            qs, ts = s.get_state()
            st = s.hybrid_stats()
        judges += st["judges"]
        reverts += st["reverts"]
        qb, tb = got[k]
        assert steps[k] == n, (k, steps[k], n)
        assert abs(dt_out[k] - dtv[1]) <= 1e-5 * dtv[1], (k, dt_out[k], dtv[1])
        assert abs(tb - ts) <= 1e-14 * max(1.0, abs(ts))
        assert rel_linf(interior(p, qb), interior(p, qs)) <= 1e-5, k
    assert hst["judges"] == judges and hst["reverts"] == reverts
    assert judges > 0
    if judge_tol == 0.0:
        assert reverts > 0
    assert 0 < hst["troubled_faces"] < hst["faces"]


def test_batch_rejects_mixed_forms():
    from finess_b200.batch import Batch
    from finess_b200.solver import FinError
    a = P.riemann_params(n=16)
    b = P.riemann_params(n=16)
    b.precision = FIN_PREC_FP32
    with pytest.raises(FinError):
        Batch([a, b])


def test_sweep_split_across_ranks_equals_one_batch():
    """The sweep split for two GPUs (finess_b200/sweep_ranks.py): each share
    run as its own batch, as each rank would on its own GPU (the ranks share
    nothing, so running the shares one after the other on one GPU is the same
    computation), gives every problem's single-batch result and steps."""
    from finess_b200._abi import FIN_PREC_FP64
    from finess_b200.sweep_ranks import batch_solve, partition, problem_sizes
    seed, n, nmin, nmax, tend = 5, 9, 24, 72, 0.05
    sizes = problem_sizes(n, seed, nmin, nmax)
    solve = batch_solve(seed, FIN_PREC_FP64, tend, nmin, nmax)
    _, steps_all, states_all = solve(list(range(n)), keep_states=True)
    parts, _ = partition([float(N) ** 3 for N in sizes], 2)
    assert all(parts)
    for part in parts:
        _, steps, states = solve(part, keep_states=True)
        for k, st, q in zip(part, steps, states):
            assert st == steps_all[k]
            assert np.max(np.abs(q - states_all[k])) <= 1e-12 * np.max(np.abs(states_all[k]))
