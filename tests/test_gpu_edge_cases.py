"""Edge cases against the oracle, bit for bit (friction off): a completely dry
domain, the smallest mesh (two triangles, all walls), an inflow string with zero
discharge, and a batch of very uneven members."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _pair(sc, steps, oracle_mod):
    sc.problem.cd[:] = 0.0
    o = oracle_mod.Oracle(sc.problem, sc.options)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, sc.options, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        so, sg = o.step(steps), g.step(steps)
        a, b = o.state(), g.state()
        for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), k
        assert so["iter"] == sg["iter"]
        return b, sg


def test_all_dry_domain(storm_lib, oracle_mod):
    sc = scenarios.dambreak(n_target=4000, seed=4)
    sc.h0[:] = 0.0
    b, sg = _pair(sc, 20, oracle_mod)
    assert not b["h"].any() and not b["u"].any()
    assert sg["tmass"] == 0.0


def _square4():
    """The smallest mesh the reference accepts (read_data stops below 4 triangles):
    a unit square split into four triangles around its centre, all walls."""
    x = np.array([0.0, 1.0, 1.0, 0.0, 0.5])
    y = np.array([0.0, 0.0, 1.0, 1.0, 0.5])
    tri = np.array([[1, 2, 5], [2, 3, 5], [3, 4, 5], [4, 1, 5]], dtype=np.int32)
    zb = np.array([0.0, 0.01, 0.02, 0.005, 0.0])
    return abi.ProblemHolder(x, y, tri, zb, np.zeros(4))


def test_smallest_mesh(storm_lib, oracle_mod):
    opts = abi.default_options(steady=0, dt_op=1, cfl=0.5, rkorder=3)
    sc = scenarios.Scenario("four", _square4(), np.array([0.5, 0.3, 0.2, 0.4]), np.zeros(4), np.zeros(4), opts, {})
    b, sg = _pair(sc, 25, oracle_mod)
    assert np.isfinite(b["h"]).all() and sg["device_status"] == 0


def test_zero_inflow(storm_lib, oracle_mod):
    sc = scenarios.channel(nx=30, ny=6, q=0.0)
    _pair(sc, 30, oracle_mod)


def test_uneven_batch(storm_lib, oracle_mod):
    big = scenarios.meander(n_target=20000, seed=7)
    scs = [big, scenarios.Scenario("tiny", _square4(), np.array([0.2, 0.1, 0.3, 0.2]), np.zeros(4), np.zeros(4),
                                   big.options, {})]
    big.problem.cd[:] = 0.0
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, big.options, keep=pms)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    b.step(15)
    for i, sc in enumerate(scs):
        o = oracle_mod.Oracle(sc.problem, big.options)
        o.set_state(sc.h0, sc.u0, sc.v0)
        o.step(15)
        a, g = o.state(), b.scenario_state(i)
        for k in ("h", "u", "v"):
            assert np.array_equal(_bits(a[k]), _bits(g[k])), (i, k)
