"""Parity and invariants at the benchmark configurations' full sizes: the 2M-cell
transient meander and the 1M-cell dam break, bit for bit against the oracle over a
few iterations (friction off, see test_gpu_parity), and mass conservation of the
closed dam-break basin over many iterations."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


@pytest.fixture(scope="module")
def meander_2m():
    sc = scenarios.meander(n_target=2_000_000)
    sc.problem.cd[:] = 0.0
    return sc


@pytest.fixture(scope="module")
def dambreak_1m():
    return scenarios.dambreak(n_target=1_000_000)


def _bitwise(sc, steps, oracle_mod):
    import os
    o = oracle_mod.Oracle(sc.problem, sc.options, threads=os.cpu_count() or 1)
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, sc.options, keep=pm) as g:
        for s in (o, g):
            s.set_state(sc.h0, sc.u0, sc.v0)
        so, sg = o.step(steps), g.step(steps)
        a, b = o.state(), g.state()
        for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
            assert np.array_equal(_bits(a[k]), _bits(b[k])), k
        assert so["iter"] == sg["iter"] == steps
        assert abs(so["tmass"] - sg["tmass"]) <= 1e-12 * so["tmass"]


def test_meander_2m_bitwise(storm_lib, oracle_mod, meander_2m):
    _bitwise(meander_2m, 4, oracle_mod)


def test_dambreak_1m_bitwise(storm_lib, oracle_mod, dambreak_1m):
    sc = dambreak_1m
    cd = sc.problem.cd.copy()
    sc.problem.cd[:] = 0.0
    try:
        _bitwise(sc, 6, oracle_mod)
    finally:
        sc.problem.cd[:] = cd


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_dambreak_1m_mass_conserved(storm_lib, dambreak_1m, precision):
    """All walls: the water volume changes only by rounding (and by the h >= 0 clip,
    which the dry bed of this case keeps small)."""
    sc = dambreak_1m
    o = abi.Options.from_buffer_copy(sc.options)
    o.precision = precision
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, o, keep=pm) as g:
        g.set_state(sc.h0, sc.u0, sc.v0)
        m0 = g.step(1)["tmass"]
        st = g.step(300)
        assert st["device_status"] == 0
        assert abs(st["tmass"] - m0) <= 1e-9 * m0, (st["tmass"], m0)
