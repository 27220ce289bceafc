"""FP32/FP64 mixed-precision path (StormFvtOptions.precision = STORM_PREC_MIXED)
against the FP64 oracle.

On the mixed path the gradient, limiter, flux and bed-slope arithmetic runs in FP32
while the state, the eta - zb face reconstruction (h + FP32 correction in FP64), the
vertex depths, friction, the RK accumulation and the mass reduction stay in FP64.
Each test states its error against the FP64 oracle: depth error in metres, momentum
error relative to the momentum scale, and the relative total-mass difference.
"""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _pair(sc, oracle_mod):
    o = oracle_mod.Oracle(sc.problem, sc.options)
    o.set_state(sc.h0, sc.u0, sc.v0)
    opts = abi.Options.from_buffer_copy(sc.options)
    opts.precision = abi.PREC_MIXED
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, opts, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    return o, g


def errors(o, g):
    a, b = o.state(), g.state()
    hu_a, hv_a = a["h"] * a["u"], a["h"] * a["v"]
    hu_b, hv_b = b["h"] * b["u"], b["h"] * b["v"]
    qs = max(float(np.abs(hu_a).max()), float(np.abs(hv_a).max()), 1e-12)
    return {
        "depth_max_m": float(np.abs(a["h"] - b["h"]).max()),
        "depth_rms_m": float(np.sqrt(np.mean((a["h"] - b["h"]) ** 2))),
        "momentum_max_rel": float(max(np.abs(hu_a - hu_b).max(), np.abs(hv_a - hv_b).max()) / qs),
    }


def test_mixed_meander_error(storm_lib, oracle_mod):
    sc = scenarios.meander(n_target=20000, seed=5)
    o, g = _pair(sc, oracle_mod)
    so, sg = o.step(40), g.step(40)
    e = errors(o, g)
    e["mass_rel"] = abs(sg["tmass"] - so["tmass"]) / so["tmass"]
    assert e["depth_max_m"] < 1e-3, e
    assert e["momentum_max_rel"] < 1e-2, e
    assert e["mass_rel"] < 1e-6, e
    assert not np.array_equal(o.state()["h"], g.state()["h"])  # it is a different arithmetic


def test_mixed_dambreak_per_step(storm_lib, oracle_mod):
    """The wet/dry stress case (Rusanov, dry bed with mounds) compared every step for
    depth, momentum and total mass."""
    sc = scenarios.dambreak(n_target=20000, seed=4)
    o, g = _pair(sc, oracle_mod)
    worst = {"depth_max_m": 0.0, "momentum_max_rel": 0.0, "mass_rel": 0.0}
    for _ in range(30):
        so, sg = o.step(1), g.step(1)
        e = errors(o, g)
        e["mass_rel"] = abs(sg["tmass"] - so["tmass"]) / so["tmass"]
        for k in worst:
            worst[k] = max(worst[k], e[k])
    assert worst["depth_max_m"] < 1e-2, worst
    assert worst["mass_rel"] < 1e-9, worst


def test_mixed_steady_depth_within_1cm(storm_lib, oracle_mod):
    """mixed-precision steady state within 1 cm of the FP64 one."""
    sc = scenarios.channel(nx=40, ny=4, length=20.0, width=2.0, q=1.0, rstop=1e-5, stop_cr=1)
    o, g = _pair(sc, oracle_mod)
    so = o.step(20000)
    sg = g.step(20000)
    assert so["converged"] and sg["converged"]
    e = errors(o, g)
    assert e["depth_max_m"] < 0.01, e
