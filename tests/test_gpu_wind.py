"""Wind forcing (windforcing.f90, added to phi at solverFVT.f90:218-224) on the GPU
against the oracle: bit for bit in FP64 (friction off, so no pow() enters)."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _windy(sc, at_vertices, seed=11):
    sc.problem.cd[:] = 0.0
    return scenarios.with_wind(sc, scenarios.wind_fields(sc.problem, at_vertices, seed))


@pytest.mark.parametrize("kind", ["channel_cells", "meander_vertices"])
def test_wind_bitwise(storm_lib, oracle_mod, kind):
    if kind == "channel_cells":
        sc = _windy(scenarios.channel(nx=40, ny=8), at_vertices=False)
    else:
        sc = _windy(scenarios.meander(n_target=9000, seed=2), at_vertices=True)
    o = oracle_mod.Oracle(sc.problem, sc.options)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, sc.options, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        so = o.step(40)
        sg = g.step(40)
        a, b = o.state(), g.state()
        for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), k
        assert so["iter"] == sg["iter"]


def test_wind_changes_the_solution(storm_lib):
    sc = scenarios.channel(nx=40, ny=8)
    sc.problem.cd[:] = 0.0
    calm = fvt.build_mesh(sc.problem)
    windy = fvt.build_mesh(_windy(scenarios.channel(nx=40, ny=8), at_vertices=False).problem)
    res = []
    for pm in (calm, windy):
        with fvt.Solver(pm, sc.options, keep=pm) as g:
            g.set_state(sc.h0, sc.u0, sc.v0)
            g.step(20)
            res.append(g.state()["u"])
    assert not np.array_equal(res[0], res[1])


def test_wind_batch_member_equals_alone(storm_lib, oracle_mod):
    """A batch mixing a windy member with calm ones: every member as it runs alone."""
    scs = scenarios.batch_channels(3, 600, 1500, seed=21, opt_limiter=0)
    for sc in scs:
        sc.problem.cd[:] = 0.0
    scs[1] = _windy(scs[1], at_vertices=True)
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, scs[0].options, keep=pms)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    b.step(30)
    for i, sc in enumerate(scs):
        o = oracle_mod.Oracle(sc.problem, scs[0].options)
        o.set_state(sc.h0, sc.u0, sc.v0)
        o.step(30)
        a, g = o.state(), b.scenario_state(i)
        for k in ("h", "u", "v"):
            assert np.array_equal(_bits(a[k]), _bits(g[k])), (i, k)
