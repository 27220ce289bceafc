"""The output step (storm_fvt_output_vertices: to_vertices, ctr2vtx of cd,
error_est(2)) against the oracle's restatement: the same bits for the vertex depth,
velocity and roughness, the error estimate, and for the solution afterwards (the
output step zeroes u,v of wet cells with a dry vertex, which changes the following
iterations exactly as in the reference).  Friction off, so every operation is
bitwise (see test_gpu_parity)."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _pair(sc, oracle_mod):
    sc.problem.cd[:] = 0.0
    o = oracle_mod.Oracle(sc.problem, sc.options)
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    ob = abi.OutputBoundaryHolder(sc.problem, pm.numpy())
    for s in (o, g):
        s.set_state(sc.h0, sc.u0, sc.v0)
    return o, g, ob


def _run(sc, oracle_mod, schedule):
    """schedule: list of (steps, in_loop) -- step, then output."""
    o, g, ob = _pair(sc, oracle_mod)
    for steps, in_loop in schedule:
        o.step(steps)
        g.step(steps)
        a = o.output_vertices(ob, in_loop)
        b = g.output_vertices(ob, in_loop)
        for k in ("hvtx", "uvtx", "vvtx", "cdvtx", "e_est"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), (k, np.abs(a[k] - b[k]).max())
    o.step(7)
    g.step(7)
    a, b = o.state(), g.state()
    for k in ("h", "u", "v", "rku", "rkv"):
        assert np.array_equal(_bits(a[k]), _bits(b[k])), k
    return a


@pytest.mark.parametrize("btype", [0, 1])
def test_channel_output_bitwise(storm_lib, oracle_mod, btype):
    sc = scenarios.channel(nx=40, ny=8, btype=btype)
    _run(sc, oracle_mod, [(15, True), (9, True), (4, False)])


def test_meander_wetdry_output_changes_the_run_like_the_reference(storm_lib, oracle_mod):
    sc = scenarios.meander(n_target=9000, seed=1)
    a = _run(sc, oracle_mod, [(12, True), (12, True)])
    # the output step did zero some partially wet cells: a run without it differs
    o2 = oracle_mod.Oracle(sc.problem, sc.options)
    o2.set_state(sc.h0, sc.u0, sc.v0)
    o2.step(31)
    assert not np.array_equal(_bits(o2.state()["u"]), _bits(a["u"]))


def test_time_series_and_mixed_boundaries_output(storm_lib, oracle_mod):
    base = scenarios.channel(nx=50, ny=6)
    p = base.problem
    inflow = [dict(p.inflow_spec[0], series=(np.array([0.0, 0.5, 2.0]), np.array([2.0, 6.0, 4.0])))]
    outflow = [dict(p.outflow_spec[0], series=(np.array([0.0, 1.0]), np.array([1.0, 1.1])))]
    prob = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, np.zeros_like(p.cd), inflow=inflow, outflow=outflow)
    opts = abi.default_options(steady=0, dt_op=1, cfl=0.5, rkorder=2)
    sc = scenarios.Scenario("ts", prob, base.h0, base.u0, base.v0, opts, {})
    _run(sc, oracle_mod, [(20, True), (20, False), (10, True)])
    base = scenarios.channel(nx=60, ny=12)
    p = base.problem
    out_nodes = np.array(p.outflow_spec[0]["nodes"])
    inflow = [{"type": 4, "nodes": p.inflow_spec[0]["nodes"], "value": 1.15}]
    outflow = [{"type": 2, "nodes": out_nodes[:7], "value": 0.0}, {"type": 0, "nodes": out_nodes[6:], "value": 0.0}]
    prob = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, np.zeros_like(p.cd), inflow=inflow, outflow=outflow)
    opts = abi.default_options(steady=0, dt_op=1, cfl=0.5, rkorder=3, btype=1)
    sc = scenarios.Scenario("mixed", prob, base.h0, base.u0, base.v0, opts, {})
    _run(sc, oracle_mod, [(25, True), (10, True)])


def test_output_argument_checks(storm_lib):
    sc = scenarios.channel(nx=10, ny=4, rkorder=1)
    pm = fvt.build_mesh(sc.problem)
    ob = abi.OutputBoundaryHolder(sc.problem, pm.numpy())
    with fvt.Solver(pm, sc.options, keep=pm) as g:
        g.set_state(sc.h0, sc.u0, sc.v0)
        g.step(2)
        with pytest.raises(fvt.StormError) as e:
            g.output_vertices(ob)
        assert e.value.code == abi.STORM_ERR_UNSUPPORTED
