"""The fused stage kernel (k_tile) against the phase kernels (k_grad, k_eflux,
k_flux, the default path), through the C-ABI.  Both paths run the same device
functions for the gradient, edge-flux and update arithmetic.  In FP64 (compiled
without FMA contraction) every state array, RK level, vertex depth and iteration
statistic must agree to the last bit, with and without open boundaries, for single
meshes and batches; the oracle comparisons of test_gpu_parity.py run on the phase
kernels (the default), so the fused path equals the oracle through them.  The
mixed-precision kernels are compiled with FMA contraction, which the compiler
decides per inlined context, so there the two paths are held to the mixed path's
own accuracy: each is compared with an FP64 run, and they may differ from each
other by no more than twice the larger of those errors."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _assert_mixed_pair(a, b, f, what):
    """a, b: the two mixed-precision states; f: the FP64 state of the same run."""
    for k in ("h", "u", "v", "hvtx"):
        scale = max(float(np.abs(f[k]).max()), 1e-12)
        err = max(float(np.abs(a[k] - f[k]).max()), float(np.abs(b[k] - f[k]).max()))
        diff = float(np.abs(a[k] - b[k]).max())
        assert diff <= 2.0 * err + 1e-12 * scale, (what, k, diff, err)
        assert err <= 0.05 * scale, (what, k, err, scale)  # the mixed path itself is sane


def _run(pm, opts, sc, path, steps):
    g = fvt.Solver(pm, opts, keep=pm)
    g.set_stage_path(path)
    assert g.stage_path() == path
    g.set_state(sc.h0, sc.u0, sc.v0)
    st = None
    for n in (steps // 2, steps - steps // 2):
        st = g.step(n)
    out = g.state(), st
    g.close()
    return out


@pytest.mark.parametrize("name,make,steps", [
    ("channel-hll", lambda: scenarios.channel(flux=abi.FLUX_HLL), 60),
    ("channel-roe-btype1", lambda: scenarios.channel(nx=60, ny=8, btype=1), 40),
    ("channel-lim0-rk2", lambda: scenarios.channel(nx=60, ny=8, opt_limiter=0, rkorder=2), 40),
    ("meander", lambda: scenarios.meander(n_target=40_000, seed=5), 40),
    ("dambreak", lambda: scenarios.dambreak(n_target=30_000, seed=4), 40),
])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
@pytest.mark.parametrize("fused", [fvt.STAGE_FUSED, fvt.STAGE_FUSED_NODE_KERNEL])
def test_fused_equals_phases(name, make, steps, precision, fused, storm_lib):
    sc = make()
    sc.options.precision = precision
    pm = fvt.build_mesh(sc.problem)
    (a, sa) = _run(pm, sc.options, sc, fused, steps)
    (b, sb) = _run(pm, sc.options, sc, fvt.STAGE_PHASES, steps)
    if precision == abi.PREC_MIXED:
        sc.options.precision = abi.PREC_FP64
        (f, sf) = _run(pm, sc.options, sc, fvt.STAGE_PHASES, steps)
        _assert_mixed_pair(a, b, f, name)
        assert sa["iter"] == sb["iter"]
        assert sa["tmass"] == pytest.approx(sb["tmass"], rel=1e-6)
        return
    for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"):
        if not np.array_equal(_bits(a[k]), _bits(b[k])):
            d = np.abs(a[k] - b[k])
            raise AssertionError(f"{name} {k}: {np.count_nonzero(_bits(a[k]) != _bits(b[k]))} differ, max {d.max():.3e}")
    assert sa == sb


def test_fused_batch_equals_phases(storm_lib):
    scs = scenarios.batch_channels(6, 1500, 5000, seed=9, opt_limiter=0, precision=abi.PREC_MIXED)
    pms = [fvt.build_mesh(s.problem) for s in scs]
    outs = []
    f64 = abi.Options.from_buffer_copy(scs[0].options)
    f64.precision = abi.PREC_FP64
    for path, opts in ((fvt.STAGE_FUSED, scs[0].options), (fvt.STAGE_PHASES, scs[0].options),
                       (fvt.STAGE_PHASES, f64)):
        b = fvt.BatchSolver(pms, opts, keep=pms)
        b.set_stage_path(path)
        assert b.stage_path() == path
        for i, s in enumerate(scs):
            b.set_scenario_state(i, s.h0, s.u0, s.v0)
        b.step(300)
        outs.append([(b.scenario_state(i), b.scenario_stats(i)) for i in range(len(scs))])
        b.close()
    for i, ((a, sa), (c, sc_), (f, _)) in enumerate(zip(*outs)):
        _assert_mixed_pair(a, c, f, f"scenario {i}")
        assert sa["iter"] == sc_["iter"], i


def test_fused_not_used_for_culverts_or_smoothing(storm_lib):
    sc = scenarios.channel(nx=40, ny=6)
    sc.options.rsavg_passes = 2
    sc.options.rsavg_eps = 0.5
    sc.options.rsavg_order = 1
    pm = fvt.build_mesh(sc.problem)
    g = fvt.Solver(pm, sc.options, keep=pm)
    assert g.stage_path() == fvt.STAGE_PHASES  # the default
    g.set_stage_path(fvt.STAGE_FUSED)
    assert g.stage_path() == fvt.STAGE_PHASES  # not applicable with residual smoothing
    g.close()


def test_autotune_keeps_state_and_picks_a_path(storm_lib):
    """storm_fvt_autotune times the stage paths and the block sizes from the same
    state and restores it: the run afterwards is bitwise the untuned run."""
    sc = scenarios.meander(n_target=30_000, seed=5)
    pm = fvt.build_mesh(sc.problem)
    outs = []
    for tune in (False, True):
        g = fvt.Solver(pm, sc.options, keep=pm)
        g.set_state(sc.h0, sc.u0, sc.v0)
        if tune:
            g.autotune(iters=2)
            assert g.stage_path() in (fvt.STAGE_PHASES, fvt.STAGE_FUSED, fvt.STAGE_FUSED_NODE_KERNEL)
        g.step(20)
        outs.append(g.state())
        g.close()
    for k in ("h", "u", "v", "hvtx"):
        assert np.array_equal(_bits(outs[0][k]), _bits(outs[1][k])), k
