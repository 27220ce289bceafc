"""Sub-options of the FVT step against the FP64 oracle, through the C-ABI.

* Friction options of fric_terms_impl.f90:37-70: Chezy (opt 1) has no pow() or
  log() and must match bit for bit; Colebrook (opt 3: log and **1.11) and Strickler
  (opt 4: two pow()) use CUDA's log/pow, whose last bit may differ from the host
  libm, so they are compared at the stated relative tolerances.
* The wet-only inflow (vtype 5, inflowQbyH.f90:221-402) on a channel whose inflow
  section is partly dry: bit for bit.
* Manning friction (opt 0, the configs' own law) on the wet/dry meander over 1,000
  iterations, at a stated tolerance.
"""
import os

import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

from test_gpu_parity import assert_bitwise, assert_close, assert_stats_close, run_pair

pytestmark = pytest.mark.gpu

# pow()/log() of CUDA vs the host libm differ at most in the last bit per call; over
# the stated iterations the relative difference of the state stays below these
REL_H_POW = 1e-10
REL_UV_POW = 1e-8


def _friction_channel(opt, cd):
    sc = scenarios.channel(nx=60, ny=8, opt_friction=opt)
    sc.problem.cd[:] = cd
    return sc


def test_friction_chezy_bitwise(storm_lib, oracle_mod):
    sc = _friction_channel(1, 45.0)  # Chezy C = 45 m^0.5/s: rough = g/C^2, no pow
    o, g, so, sg = run_pair(sc, 60, oracle_mod, chunks=2)
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


@pytest.mark.parametrize("opt,cd", [(3, 0.05), (4, 0.04)])
def test_friction_colebrook_strickler_close(opt, cd, storm_lib, oracle_mod):
    sc = _friction_channel(opt, cd)  # roughness height / grain size in metres
    o, g, so, sg = run_pair(sc, 150, oracle_mod, chunks=3)
    assert_close(o, g, rel_h=REL_H_POW, rel_uv=REL_UV_POW)
    assert_stats_close(so, sg, rel=1e-10)
    # the friction actually acts: the state differs from the frictionless run
    sc0 = _friction_channel(opt, cd)
    sc0.problem.cd[:] = 0.0 if opt != 3 else 1e-9
    o0, g0, _, _ = run_pair(sc0, 150, oracle_mod, chunks=1)
    assert np.abs(g0.state()["u"] - g.state()["u"]).max() > 1e-6


def _partly_dry_inflow(vtype):
    """Channel with a 1.5 m bank over the upper half of the first 10 m: the inflow
    section is half dry at the start (still water 1 m above the outlet bed)."""
    base = scenarios.channel(nx=60, ny=10)
    p = base.problem
    zb = p.zb.copy()
    bank = (p.x < 10.0) & (p.y > 5.0)
    zb[bank] += 1.5
    spec = dict(p.inflow_spec[0])
    spec["type"] = vtype
    spec["value"] = 4.0
    prob = abi.ProblemHolder(p.x, p.y, p.tri, zb, np.zeros(p.n_elems), zb_at_vertices=True, cd_at_vertices=False,
                             inflow=[spec], outflow=p.outflow_spec)
    tri = p.tri.reshape(-1, 3) - 1
    zc = zb[tri].mean(axis=1)
    wse = 0.001 * (100.0 - p.x[tri].mean(axis=1)) + 1.0
    h0 = np.maximum(wse - zc, 0.0)
    h0[h0 < 1e-3] = 0.0
    opts = abi.default_options(rkorder=3, opt_limiter=2, flux=abi.FLUX_HLL, cfl=0.9, steady=1, stop_cr=1,
                               rstop=1e-12, btype=0, hvalve=1, h_dry=1e-3, h_wet=1e-3, opt_friction=0)
    return scenarios.Scenario(f"inflow-vtype{vtype}", prob, h0, np.zeros_like(h0), np.zeros_like(h0), opts, {})


@pytest.mark.parametrize("vtype", [5, 1])
def test_inflow_wet_only_bitwise(vtype, storm_lib, oracle_mod):
    sc = _partly_dry_inflow(vtype)
    o, g, so, sg = run_pair(sc, 80, oracle_mod, chunks=2)
    assert o.drycell().sum() > 0  # some cells are still dry at the end
    assert_bitwise(o, g)
    assert_stats_close(so, sg)


def test_inflow_vtype5_differs_from_vtype1(storm_lib, oracle_mod):
    """vtype 5 leaves dry inflow edges out of the fixed point, so it is a different
    boundary from vtype 1 on this channel (the test above is not vacuous)."""
    s5, s1 = _partly_dry_inflow(5), _partly_dry_inflow(1)
    o5 = oracle_mod.Oracle(s5.problem, s5.options)
    o5.set_state(s5.h0, s5.u0, s5.v0)
    o1 = oracle_mod.Oracle(s1.problem, s1.options)
    o1.set_state(s1.h0, s1.u0, s1.v0)
    o5.step(20)
    o1.step(20)
    assert np.abs(o5.state()["h"] - o1.state()["h"]).max() > 0.0


def test_meander_manning_1000_iterations(storm_lib, oracle_mod):
    """Manning friction on the 20k-cell wet/dry meander: 1,000 iterations of the
    transient run (dt from the CFL reduction), oracle on all host threads.
    Tolerance: depth 1e-8 m relative to the largest depth, velocity 1e-6 of the
    largest speed (pow's last bit, amplified by the wet/dry fronts over 1,000
    iterations), mass to 1e-10."""
    sc = scenarios.meander(n_target=20000, seed=5)
    o = oracle_mod.Oracle(sc.problem, sc.options, threads=len(os.sched_getaffinity(0)))
    o.set_state(sc.h0, sc.u0, sc.v0)
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    so = sg = None
    for _ in range(4):
        so = o.step(250)
        sg = g.step(250)
    assert so["iter"] == sg["iter"] == 1000
    assert_close(o, g, rel_h=1e-8, rel_uv=1e-6)
    assert sg["tmass"] == pytest.approx(so["tmass"], rel=1e-10)
