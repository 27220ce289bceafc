"""CUDA FVT step vs the CPU FP64 oracle, through the C-ABI.

Bit-exact cases set the roughness to zero: the only operation whose CUDA result may
differ from the host libm in the last bit is pow() in the Manning friction factor
(fric_terms_impl.f90:36), and with cd = 0 its value drops out (g*0*0/h**(1/3) = 0).
Every other kernel evaluates the reference's expressions in the reference's order
(no FMA contraction, same per-cell summation order), so h, u, v, the RK levels and
the vertex depths must agree to the last bit.  With friction the tolerance is
relative 1e-10 on h and 1e-8 (of the velocity scale) on u, v after the stated steps.
"""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu

REL_H = 1e-10  # tolerance with Manning friction (pow of the host libm vs CUDA)
REL_UV = 1e-8


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def run_pair(sc, steps, oracle_mod, *, mesh_from="product", chunks=1):
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    if mesh_from == "product":
        pm = fvt.build_mesh(sc.problem)
        g = fvt.Solver(pm, sc.options, keep=pm)
    else:
        g = fvt.Solver(o.mesh(), sc.options, keep=o)
    g.set_state(sc.h0, sc.u0, sc.v0)
    assert np.array_equal(g.drycell(), o.drycell()), "first-step dry flags differ"
    per = max(1, steps // chunks)
    so = sg = None
    done = 0
    while done < steps:
        n = min(per, steps - done)
        so = o.step(n)
        sg = g.step(n)
        done += n
    return o, g, so, sg


def assert_bitwise(o, g):
    a, b = o.state(), g.state()
    for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
        ok = np.array_equal(_bits(a[k]), _bits(b[k]))
        if not ok:
            d = np.abs(a[k] - b[k])
            i = int(np.argmax(d))
            raise AssertionError(f"{k}: {np.count_nonzero(_bits(a[k]) != _bits(b[k]))} entries differ, "
                                 f"max |diff| {d[i]:.3e} at {i} (oracle {a[k][i]!r}, gpu {b[k][i]!r})")


def assert_close(o, g, rel_h=REL_H, rel_uv=REL_UV):
    a, b = o.state(), g.state()
    hs = max(1.0, float(np.abs(a["h"]).max()))
    us = max(1.0, float(np.abs(a["u"]).max()), float(np.abs(a["v"]).max()))
    assert np.abs(a["h"] - b["h"]).max() <= rel_h * hs
    assert np.abs(a["u"] - b["u"]).max() <= rel_uv * us
    assert np.abs(a["v"] - b["v"]).max() <= rel_uv * us


def assert_stats_close(so, sg, rel=1e-11):
    assert so["iter"] == sg["iter"]
    for k in ("tmass", "ttime", "stime"):
        assert sg[k] == pytest.approx(so[k], rel=rel, abs=1e-300), k
    for k in ("rmax", "rms_dh"):
        assert sg[k] == pytest.approx(so[k], rel=1e-9, abs=1e-14), k
    np.testing.assert_allclose(sg["cqin3"], so["cqin3"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(sg["cqout3"], so["cqout3"], rtol=1e-9, atol=1e-12)


def _no_friction(sc):
    sc.problem.cd[:] = 0.0
    return sc


# --------------------------------------------------------------------------- #
def test_first_step_dry_flags_bitexact(storm_lib, oracle_mod):
    sc = scenarios.meander(n_target=20000, seed=11)
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    dg, do = g.drycell(), o.drycell()
    assert do.sum() > 0.2 * len(do)  # a wet/dry case
    assert np.array_equal(dg, do)


@pytest.mark.parametrize("flux", [abi.FLUX_HLL, abi.FLUX_ROE, abi.FLUX_RUSANOV])
def test_channel_bitwise(flux, storm_lib, oracle_mod):
    sc = _no_friction(scenarios.channel(flux=flux))
    o, g, so, sg = run_pair(sc, 60, oracle_mod, chunks=3)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_channel_manning_close(storm_lib, oracle_mod):
    sc = scenarios.channel()
    o, g, so, sg = run_pair(sc, 200, oracle_mod, chunks=4)
    assert_close(o, g)
    assert_stats_close(so, sg, rel=1e-10)


@pytest.mark.parametrize("variant", [
    dict(rkorder=1), dict(rkorder=2), dict(opt_limiter=0), dict(opt_limiter=1), dict(btype=1),
    dict(stop_cr=0), dict(vclip=1, vceiling=0.5), dict(hvalve=0), dict(h_wet=0.003),
    dict(opt_friction=2),
])
def test_channel_option_matrix_bitwise(variant, storm_lib, oracle_mod):
    sc = scenarios.channel(nx=60, ny=8, **variant)
    if variant.get("opt_friction") == 2:
        sc.problem.cd[:] = 0.002  # drag coefficient: no pow() involved
    else:
        _no_friction(sc)
    o, g, so, sg = run_pair(sc, 40, oracle_mod, chunks=2)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_meander_wetdry_bitwise(storm_lib, oracle_mod):
    sc = _no_friction(scenarios.meander(n_target=20000, seed=5))
    o, g, so, sg = run_pair(sc, 40, oracle_mod, chunks=2)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_meander_wetdry_manning_close(storm_lib, oracle_mod):
    sc = scenarios.meander(n_target=20000, seed=5)
    o, g, so, sg = run_pair(sc, 40, oracle_mod)
    assert_close(o, g, rel_h=1e-9, rel_uv=1e-7)


def test_dambreak_rusanov_bitwise(storm_lib, oracle_mod):
    sc = _no_friction(scenarios.dambreak(n_target=20000, seed=4))
    o, g, so, sg = run_pair(sc, 40, oracle_mod, chunks=2)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_oracle_prepared_mesh_is_accepted(storm_lib, oracle_mod):
    """The Fortran-layout arrays exported by the oracle drive the same result."""
    sc = _no_friction(scenarios.channel(nx=50, ny=6))
    o, g, so, sg = run_pair(sc, 30, oracle_mod, mesh_from="oracle")
    assert_bitwise(o, g)


def test_gpu_runs_are_deterministic(storm_lib):
    sc = scenarios.meander(n_target=20000, seed=3)
    outs = []
    for _ in range(2):
        pm = fvt.build_mesh(sc.problem)
        g = fvt.Solver(pm, sc.options, keep=pm)
        g.set_state(sc.h0, sc.u0, sc.v0)
        st = g.step(25)
        outs.append((g.state(), st))
    for k in ("h", "u", "v", "rku", "rkv", "hvtx"):
        assert np.array_equal(_bits(outs[0][0][k]), _bits(outs[1][0][k])), k
    assert outs[0][1] == outs[1][1]


def test_steady_stop_matches_oracle(storm_lib, oracle_mod):
    """Steady run to a loose threshold: both stop at the same iteration."""
    sc = _no_friction(scenarios.channel(nx=40, ny=4, rstop=2e-4, stop_cr=1))
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    so = o.step(3000)
    sg = g.step(3000)
    assert so["converged"] and sg["converged"]
    assert so["iter"] == sg["iter"]
    assert_bitwise(o, g)


def test_time_series_boundaries(storm_lib, oracle_mod):
    """Unsteady run with piecewise-linear inflow and stage series (get_time_bcs)."""
    base = scenarios.channel(nx=50, ny=6)
    p = base.problem
    inflow = [dict(p.inflow_spec[0], series=(np.array([0.0, 0.5, 2.0]), np.array([2.0, 6.0, 4.0])))]
    outflow = [dict(p.outflow_spec[0], series=(np.array([0.0, 1.0]), np.array([1.0, 1.1])))]
    prob = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, np.zeros_like(p.cd), inflow=inflow, outflow=outflow)
    opts = abi.default_options(steady=0, dt_op=1, cfl=0.5, rkorder=2)
    sc = scenarios.Scenario("ts", prob, base.h0, base.u0, base.v0, opts, {})
    o, g, so, sg = run_pair(sc, 60, oracle_mod, chunks=3)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_mixed_boundary_types(storm_lib, oracle_mod):
    """Stage inflow (vtype 4), critical (htype 2) and free (htype 0) outflows."""
    base = scenarios.channel(nx=60, ny=12)
    p = base.problem
    ny = 12
    out_nodes = np.array(p.outflow_spec[0]["nodes"])
    inflow = [{"type": 4, "nodes": p.inflow_spec[0]["nodes"], "value": 1.15}]
    outflow = [{"type": 2, "nodes": out_nodes[: ny // 2 + 1], "value": 0.0},
               {"type": 0, "nodes": out_nodes[ny // 2:], "value": 0.0}]
    prob = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, np.zeros_like(p.cd), inflow=inflow, outflow=outflow)
    opts = abi.default_options(steady=0, dt_op=1, cfl=0.5, rkorder=3)
    sc = scenarios.Scenario("mixed", prob, base.h0, base.u0, base.v0, opts, {})
    o, g, so, sg = run_pair(sc, 50, oracle_mod, chunks=2)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_given_lsq_coefficients_are_read_when_not_derivable(storm_lib, oracle_mod):
    """A caller's lsq_a that is not the sum lsq_setup forms (here one ulp above it in
    every cell, as another compiler's rounding might leave it) is read, not formed
    again: the GPU follows the oracle, which reads the same perturbed array."""
    sc = _no_friction(scenarios.meander(n_target=20000, seed=5))
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    m = o.mesh()
    T = m.n_elems
    a = np.ctypeslib.as_array(m.lsq_a, shape=(T,))
    a[:] = np.nextafter(a, np.inf)  # writes through to the oracle's own array
    g = fvt.Solver(o.mesh(), sc.options, keep=o)
    g.set_state(sc.h0, sc.u0, sc.v0)
    so, sg = o.step(20), g.step(20)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)
