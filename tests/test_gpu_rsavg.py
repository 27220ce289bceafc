"""Residual smoothing (activateRSAVG, solverFVT.f90:238-256) on the GPU, colour order,
against the oracle's colour-order restatement: bit for bit (friction off)."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _opts(sc, **kw):
    o = abi.Options.from_buffer_copy(sc.options)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


@pytest.mark.parametrize("kind", ["channel", "meander"])
def test_rsavg_colour_order_bitwise(storm_lib, oracle_mod, kind):
    sc = scenarios.channel(nx=40, ny=8) if kind == "channel" else scenarios.meander(n_target=9000, seed=2)
    sc.problem.cd[:] = 0.0
    opt = _opts(sc, rsavg_passes=3, rsavg_order=1, rsavg_eps=0.6)
    o = oracle_mod.Oracle(sc.problem, opt)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, opt, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        so = o.step(30)
        sg = g.step(30)
        a, b = o.state(), g.state()
        for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), k
        assert so["iter"] == sg["iter"]
        assert abs(so["rmax"] - sg["rmax"]) <= 1e-11 * max(abs(so["rmax"]), 1e-300)


def test_rsavg_batch_members_equal_alone(storm_lib, oracle_mod):
    scs = scenarios.batch_channels(3, 600, 1500, seed=12, opt_limiter=0)
    opt = _opts(scs[0], rsavg_passes=2, rsavg_order=1, rsavg_eps=0.5)
    for sc in scs:
        sc.problem.cd[:] = 0.0
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, opt, keep=pms)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    b.step(40)
    for i, sc in enumerate(scs):
        o = oracle_mod.Oracle(sc.problem, opt)
        o.set_state(sc.h0, sc.u0, sc.v0)
        o.step(40)
        a, g = o.state(), b.scenario_state(i)
        for k in ("h", "u", "v"):
            assert np.array_equal(_bits(a[k]), _bits(g[k])), (i, k)


def test_rsavg_index_order_is_oracle_only(storm_lib):
    sc = scenarios.channel(nx=10, ny=4)
    pm = fvt.build_mesh(sc.problem)
    with pytest.raises(fvt.StormError) as e:
        fvt.Solver(pm, _opts(sc, rsavg_passes=2, rsavg_order=0, rsavg_eps=0.5), keep=pm)
    assert e.value.code == abi.STORM_ERR_UNSUPPORTED
