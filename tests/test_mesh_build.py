"""Host-side builder of the prepared mesh vs the oracle's restatement, bit for bit,
and the C-ABI surface of libstorm_fvt.so (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


def assert_mesh_equal(mo, mp):
    assert set(mo) == set(mp)
    for k in mo:
        a, b = mo[k], mp[k]
        if isinstance(a, np.ndarray):
            assert a.shape == b.shape, k
            assert np.array_equal(_bits(a), _bits(b)), f"{k} differs"
        else:
            assert a == b, (k, a, b)


CASES = {
    "channel": lambda: scenarios.channel(),
    "meander": lambda: scenarios.meander(n_target=12000, seed=7),
    "dambreak": lambda: scenarios.dambreak(n_target=12000, seed=8),
    "channel_cellbed": lambda: _cell_bed_channel(),
    "channel_wind_cells": lambda: _wind_case(scenarios.channel(nx=40, ny=6), at_vertices=False),
    "meander_wind_vertices": lambda: _wind_case(scenarios.meander(n_target=6000, seed=3), at_vertices=True),
    "culvert_channel": lambda: scenarios.culvert_channel(),
}


def _wind_case(sc, at_vertices):
    return scenarios.with_wind(sc, scenarios.wind_fields(sc.problem, at_vertices))


def _cell_bed_channel():
    sc = scenarios.channel(nx=40, ny=6)
    p = sc.problem
    t = p.tri.reshape(-1, 3) - 1
    zc = p.zb[t].mean(axis=1)
    cdv = np.full(p.n_pts, 0.03)
    prob = abi.ProblemHolder(p.x, p.y, p.tri, zc, cdv, zb_at_vertices=False, cd_at_vertices=True,
                             inflow=p.inflow_spec, outflow=p.outflow_spec)
    sc.problem = prob
    return sc


@pytest.mark.parametrize("case", sorted(CASES))
def test_builder_matches_oracle(case, storm_lib, oracle_mod):
    sc = CASES[case]()
    o = oracle_mod.Oracle(sc.problem, sc.options)
    pm = fvt.build_mesh(sc.problem)
    mo = o.mesh_numpy()
    assert_mesh_equal(mo, pm.numpy())
    assert (mo["wcoef1"] is not None) == ("wind" in case)
    assert (mo["n_culvert"] > 0) == ("culvert" in case)


def test_channel_counts(storm_lib):
    """The 8,000-cell channel: N=4,221, E=12,220, 440 boundary edges (20 in, 20 out, 400 walls)."""
    sc = scenarios.channel()
    m = fvt.build_mesh(sc.problem).numpy()
    assert (m["n_pts"], m["n_elems"], m["n_edges"]) == (4221, 8000, 12220)
    assert m["wall_edges1"] == 400 and m["n_bcedges"] == 40
    assert m["flow_edges1"] == 12220 - 440


def test_builder_errors(storm_lib):
    sc = scenarios.channel(nx=10, ny=4)
    p = sc.problem
    bad = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, p.cd,
                            inflow=[{"type": 1, "nodes": [1, 7], "value": 1.0}],  # not an edge
                            outflow=p.outflow_spec)
    with pytest.raises(fvt.StormError) as e:
        fvt.build_mesh(bad)
    assert e.value.code == abi.STORM_ERR_MESH
    tri = p.tri.copy()
    tri[0] = p.n_pts + 5
    bad2 = abi.ProblemHolder(p.x, p.y, tri, p.zb, p.cd, inflow=p.inflow_spec, outflow=p.outflow_spec)
    with pytest.raises(fvt.StormError) as e:
        fvt.build_mesh(bad2)
    assert e.value.code == abi.STORM_ERR_MESH


def test_library_exports_every_declared_symbol(storm_lib):
    hdr = open(os.path.join(ROOT, "include", "storm_fvt.h")).read()
    declared = set(re.findall(r"STORM_FVT_API\s+[\w\s\*]+?\b(storm_fvt_\w+)\s*\(", hdr))
    assert declared == set(fvt.EXPORTS)
    lib = C.CDLL(fvt.lib_path())
    for name in declared:
        assert hasattr(lib, name), name


def test_library_exports_every_warm_start_symbol(storm_lib):
    from storm_b200 import gnn
    hdr = open(os.path.join(ROOT, "include", "storm_gnn.h")).read()
    declared = set(re.findall(r"STORM_FVT_API\s+[\w\s\*]+?\b(storm_gnn_\w+)\s*\(", hdr))
    assert declared == set(gnn.EXPORTS)
    lib = C.CDLL(fvt.lib_path())
    for name in declared:
        assert hasattr(lib, name), name
    L = gnn.lib()
    assert L.storm_gnn_grad_size(384, 128) == 128 * 384 + 128 + 128 * 128 + 128


def test_option_checks_run_before_device_use(storm_lib):
    """Invalid options are rejected on the host (STORM_ERR_ARG / UNSUPPORTED)."""
    sc = scenarios.channel(nx=10, ny=4)
    pm = fvt.build_mesh(sc.problem)
    for kw, code in [({"rkorder": 4}, abi.STORM_ERR_ARG), ({"opt_limiter": 3}, abi.STORM_ERR_ARG),
                     ({"opt_friction": 5}, abi.STORM_ERR_UNSUPPORTED), ({"flux": 7}, abi.STORM_ERR_ARG),
                     ({"precision": 7}, abi.STORM_ERR_ARG)]:
        with pytest.raises(fvt.StormError) as e:
            fvt.Solver(pm, fvt.default_options(**kw))
        assert e.value.code == code, kw


def test_default_options_match_reference_defaults(storm_lib):
    lo = fvt.default_options()
    po = abi.default_options()
    for name, _ in abi.Options._fields_:
        if name == "reserved":
            continue
        assert getattr(lo, name) == getattr(po, name), name


def test_fewer_than_four_triangles_rejected(storm_lib, oracle_mod):
    """read_data stops on a domain of fewer than 4 triangles; both builders do too."""
    x = np.array([0.0, 1.0, 1.0, 0.0])
    y = np.array([0.0, 0.0, 1.0, 1.0])
    p = abi.ProblemHolder(x, y, np.array([[1, 2, 3], [1, 3, 4]], dtype=np.int32), np.zeros(4), np.zeros(2))
    with pytest.raises(fvt.StormError) as e:
        fvt.build_mesh(p)
    assert e.value.code == abi.STORM_ERR_MESH
    with pytest.raises(oracle_mod.OracleError):
        oracle_mod.Oracle(p, abi.default_options())


def test_host_checks_of_the_newer_entry_points(storm_lib):
    """Argument checks that run before any device work: linking a null handle, and
    residual-smoothing options out of range."""
    L = fvt.lib()
    z = np.zeros(1, dtype=np.int32)
    rc = L.storm_fvt_link_partitions(None, 1, abi.iptr(z), abi.iptr(z), abi.iptr(z), abi.iptr(z), 0)
    assert rc == abi.STORM_ERR_ARG
    assert b"null handle" in L.storm_fvt_last_error()
    sc = scenarios.channel(nx=10, ny=4)
    pm = fvt.build_mesh(sc.problem)
    for kw in ({"rsavg_passes": -1}, {"rsavg_passes": 2, "rsavg_order": 1, "rsavg_eps": -0.5}):
        with pytest.raises(fvt.StormError) as e:
            fvt.Solver(pm, fvt.default_options(**kw))
        assert e.value.code == abi.STORM_ERR_ARG, kw


@pytest.mark.parametrize("make", [lambda: scenarios.meander(n_target=20000, seed=5),
                                  lambda: scenarios.dambreak(n_target=20000, seed=4),
                                  lambda: scenarios.channel(nx=60, ny=8)])
def test_lsq_coefficients_are_the_stencil_sums(make, storm_lib):
    """lsq_a/b/c/det of a prepared mesh are, bit for bit, the sums lsq_setup.f90:92-145
    forms from the stencil weights and offsets in stencil order (a = sum w dx dx, ...,
    det = a c - b b), which the FP64 gradient kernel relies on to form them itself
    (numpy float64 rounds each operation as the FMA-free device code does)."""
    sc = make()
    pm = fvt.PreparedMesh(sc.problem)
    try:
        m = pm.numpy()
        ncol = pm.mesh.t2t_ncol
        T = m["t2t"].size // ncol
        cnt = m["t2t"].reshape(ncol, T)[0]
        kl = max(ncol - 1, 1)
        w, dx, dy = (m[k].reshape(kl, T) for k in ("lsq_w", "lsq_dx", "lsq_dy"))
        a, b, c = np.zeros(T), np.zeros(T), np.zeros(T)
        for k in range(kl):
            on = cnt > k
            a = np.where(on, a + w[k] * dx[k] * dx[k], a)
            b = np.where(on, b + w[k] * dx[k] * dy[k], b)
            c = np.where(on, c + w[k] * dy[k] * dy[k], c)
        det = a * c - b * b
        for got, key in ((a, "lsq_a"), (b, "lsq_b"), (c, "lsq_c"), (det, "lsq_det")):
            assert np.array_equal(got.view(np.uint64), m[key].view(np.uint64)), key
    finally:
        pm.close()
