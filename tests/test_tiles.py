"""The fused stage kernel's tile plan, built and checked on the host (no GPU): every
local index of every tile maps back to the cell or edge the layout names, each
interior edge belongs to exactly one tile's range, and the per-tile sizes stay within
what one CTA's shared memory holds."""
import pytest

from storm_b200 import abi, fvt, scenarios


@pytest.mark.parametrize("make", [
    lambda: scenarios.channel(),
    lambda: scenarios.channel(nx=7, ny=3),
    lambda: scenarios.meander(n_target=60_000, seed=2),
    lambda: scenarios.dambreak(n_target=30_000, seed=3),
])
@pytest.mark.parametrize("tc", [64, 256, 512])
def test_tile_plan_checks(make, tc, storm_lib):
    sc = make()
    pm = fvt.build_mesh(sc.problem)
    st = fvt.tile_check([pm], tile_cells=tc)
    assert st["check"] == 0, st
    slots = -(-sc.n_elems // 256) * 256  # cell slots are padded to the reduction block
    assert st["tiles"] == -(-slots // tc)
    assert st["ng_max"] <= st["ns_max"] < 65535 and st["ne_max"] < 65535


def test_tile_plan_of_a_batch(storm_lib):
    scs = scenarios.batch_channels(5, 1500, 6000, seed=9, opt_limiter=0, precision=abi.PREC_MIXED)
    pms = [fvt.build_mesh(s.problem) for s in scs]
    st = fvt.tile_check(pms, tile_cells=256)
    assert st["check"] == 0, st
    # H1 and H2 are a ring of the tile: a fraction of the owned cells
    T = sum(s.n_elems for s in scs)
    assert st["h1_cells"] < 0.5 * T and st["h2_cells"] < 0.6 * T
