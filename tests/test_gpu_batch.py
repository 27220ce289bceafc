"""Batched scenarios (storm_fvt_create_batch) against one oracle run per scenario.

Every scenario of a batch must evolve exactly as it does alone: same bits for h, u,
v and the RK levels (friction off, see test_gpu_parity), its own dt, clocks and stop
iteration, whatever the other scenarios do."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _run_batch(scs, steps, oracle_mod, options):
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, options, keep=pms)
    assert b.n == len(scs)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    b.step(steps)
    outs = []
    for i, sc in enumerate(scs):
        o = oracle_mod.Oracle(sc.problem, options)
        o.set_state(sc.h0, sc.u0, sc.v0)
        so = o.step(steps)
        outs.append((o, so, b.scenario_state(i), b.scenario_stats(i)))
    return b, outs


def test_batch_unsteady_meanders_bitwise(storm_lib, oracle_mod):
    scs = [scenarios.meander(n_target=n, seed=s) for n, s in ((9000, 1), (15000, 2), (5000, 3))]
    for sc in scs:
        sc.problem.cd[:] = 0.0
    b, outs = _run_batch(scs, 25, oracle_mod, scs[0].options)
    for o, so, sg, stg in outs:
        a = o.state()
        for k in ("h", "u", "v", "rku", "rkv", "hvtx"):
            assert np.array_equal(_bits(a[k]), _bits(sg[k])), k
        assert stg["iter"] == so["iter"]
        assert stg["stime"] == pytest.approx(so["stime"], rel=1e-12)  # each its own dt
        assert stg["tmass"] == pytest.approx(so["tmass"], rel=1e-11)
    assert len({round(x[3]["stime"], 12) for x in outs}) == len(outs)


def test_batch_steady_stops_per_scenario(storm_lib, oracle_mod):
    """Scenarios converge at different iterations; each stops where its oracle does
    and the others keep going."""
    scs = [scenarios.channel(nx=30, ny=4, length=15.0, width=2.0, q=q, seed=s, rstop=3e-4, stop_cr=1)
           for q, s in ((0.5, 1), (1.0, 2), (2.0, 3))]
    for sc in scs:
        sc.problem.cd[:] = 0.0
    b, outs = _run_batch(scs, 4000, oracle_mod, scs[0].options)
    iters = []
    for o, so, sg, stg in outs:
        assert so["converged"] and stg["converged"]
        assert stg["iter"] == so["iter"]
        a = o.state()
        for k in ("h", "u", "v"):
            assert np.array_equal(_bits(a[k]), _bits(sg[k])), k
        iters.append(stg["iter"])
    assert len(set(iters)) > 1


def test_batch_rejects_single_scenario_calls(storm_lib):
    scs = [scenarios.channel(nx=10, ny=4, seed=s) for s in (1, 2)]
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, scs[0].options, keep=pms)
    z = np.zeros(b.T)
    with pytest.raises(fvt.StormError) as e:
        b.set_state(z, z, z)  # the whole-handle call is for single-scenario handles
    assert e.value.code == abi.STORM_ERR_ARG


def test_autotune_keeps_state_and_results(storm_lib, oracle_mod):
    """The autotuner restores the state it timed from, and other block shapes give the
    same bits (every per-cell result is independent of the launch shape)."""
    sc = scenarios.meander(n_target=12000, seed=13)
    sc.problem.cd[:] = 0.0
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    g.step(5)
    before = g.state()
    chosen = g.autotune(iters=2)
    after = g.state()
    for k in ("h", "u", "v", "rku", "rkv"):
        assert np.array_equal(_bits(before[k]), _bits(after[k])), k
    assert set(chosen) == {"node", "grad", "eflux", "flux"}
    g.step(20)
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    o.step(25)
    a, b = o.state(), g.state()
    for k in ("h", "u", "v", "rku", "rkv"):
        assert np.array_equal(_bits(a[k]), _bits(b[k])), k
