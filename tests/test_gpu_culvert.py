"""Culverts (cvdisch.f90 discharges entered in phi(:,1) at solverFVT.f90:227-233) on
the GPU against the oracle: bit for bit in FP64."""
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


@pytest.mark.parametrize("flux", [abi.FLUX_HLL, abi.FLUX_ROE])
def test_culvert_channel_bitwise(storm_lib, oracle_mod, flux):
    """Embankment with two culverts, dry embankment cells, friction off (no pow())."""
    sc = scenarios.culvert_channel()
    sc.problem.cd[:] = 0.0
    opt = _opts(sc, flux=flux)
    o = oracle_mod.Oracle(sc.problem, opt)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, opt, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        for _ in range(3):
            so = o.step(40)
            sg = g.step(40)
            a, b = o.state(), g.state()
            for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
                assert np.array_equal(_bits(a[k]), _bits(b[k])), k
            assert so["iter"] == sg["iter"]


def test_culvert_with_friction_close(storm_lib, oracle_mod):
    """With Manning friction (pow() on both sides) the states agree to round-off."""
    sc = scenarios.culvert_channel()
    o = oracle_mod.Oracle(sc.problem, sc.options)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, sc.options, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        o.step(100)
        g.step(100)
        a, b = o.state(), g.state()
        assert np.max(np.abs(a["h"] - b["h"])) < 1e-10


def test_culvert_batch_member_equals_alone(storm_lib, oracle_mod):
    """A batch of a plain channel, the culvert channel and another plain channel."""
    scs = scenarios.batch_channels(2, 600, 1500, seed=31, opt_limiter=0)
    cv = scenarios.culvert_channel(nx=40, ny=6, opt_limiter=0)
    scs.insert(1, cv)
    for sc in scs:
        sc.problem.cd[:] = 0.0
    opt = scs[0].options
    pms = [fvt.build_mesh(sc.problem) for sc in scs]
    b = fvt.BatchSolver(pms, opt, keep=pms)
    for i, sc in enumerate(scs):
        b.set_scenario_state(i, sc.h0, sc.u0, sc.v0)
    b.step(30)
    for i, sc in enumerate(scs):
        o = oracle_mod.Oracle(sc.problem, opt)
        o.set_state(sc.h0, sc.u0, sc.v0)
        o.step(30)
        a, g = o.state(), b.scenario_state(i)
        for k in ("h", "u", "v"):
            assert np.array_equal(_bits(a[k]), _bits(g[k])), (i, k)


def test_culvert_mixed_precision_close(storm_lib):
    """The mixed path (FP32 gradients and fluxes, FP64 state) with culverts stays
    within 1 cm of FP64 over 200 iterations, and the water volume in the channel
    (open at both ends, so set by the boundary fluxes) within 1e-4 of FP64's."""
    sc = scenarios.culvert_channel()
    pm = fvt.build_mesh(sc.problem)
    out = []
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        with fvt.Solver(pm, _opts(sc, precision=prec), keep=pm) as g:
            g.set_state(sc.h0, sc.u0, sc.v0)
            st = g.step(200)
            out.append((g.state()["h"], st))
    (h64, s64), (hmx, smx) = out
    assert np.all(np.isfinite(hmx))
    assert np.max(np.abs(h64 - hmx)) < 0.01
    assert smx["tmass"] == pytest.approx(s64["tmass"], rel=1e-4)


def test_culvert_wind_and_smoothing_together_bitwise(storm_lib, oracle_mod):
    """All three extra source paths at once (culverts, wind, residual smoothing in
    colour order) against the oracle, bit for bit."""
    sc = scenarios.culvert_channel()
    sc.problem.cd[:] = 0.0
    sc = scenarios.with_wind(sc, scenarios.wind_fields(sc.problem, at_vertices=False, seed=5))
    opt = _opts(sc, rsavg_passes=2, rsavg_order=1, rsavg_eps=0.5)
    o = oracle_mod.Oracle(sc.problem, opt)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, opt, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        o.step(40)
        g.step(40)
        a, b = o.state(), g.state()
        for k in ("h", "u", "v", "rkh", "rku", "rkv"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), k
