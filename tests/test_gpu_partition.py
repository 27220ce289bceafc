"""One mesh solved as linked parts of one batch handle (storm_fvt_link_partitions,
storm_b200/partition.py) against the undivided mesh on the same GPU: the owned cells
evolve bit for bit (state, dt, iteration count); the mass and residual sums, added
per part, agree to round-off."""
import numpy as np
import pytest

from storm_b200 import abi, fvt, partition, scenarios

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _opts(sc, **kw):
    o = abi.Options.from_buffer_copy(sc.options)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _compare(sc, opt, nparts, rounds, steps, keys=("h", "u", "v", "rkh", "rku", "rkv")):
    pm = fvt.build_mesh(sc.problem)
    with fvt.Solver(pm, opt, keep=pm) as whole, partition.PartitionedSolver(sc.problem, opt, nparts) as parts:
        for s in (whole, parts):
            s.set_state(sc.h0, sc.u0, sc.v0)
        for _ in range(rounds):
            a = whole.step(steps)
            b = parts.step(steps)
            assert a["iter"] == b["iter"]
            assert a["converged"] == b["converged"]
            assert _bits([a["delt"]]) == _bits([b["delt"]])
            assert b["tmass"] == pytest.approx(a["tmass"], rel=1e-12)
            assert b["rms_dh"] == pytest.approx(a["rms_dh"], rel=1e-9, abs=1e-300)
            sa, sb = whole.state(), parts.state()
            for k in keys:
                assert np.array_equal(_bits(sa[k]), _bits(sb[k])), k
            n_in = len(sc.problem.inflow_spec)
            np.testing.assert_array_equal(np.asarray(a["cqin3"][:n_in]), b["cqin3"])
        return parts


def test_meander_transient_three_parts(storm_lib):
    sc = scenarios.meander(n_target=12000, seed=5)
    parts = _compare(sc, sc.options, 3, rounds=2, steps=25)
    assert sum(int((~P.owned).sum()) for P in parts.parts) > 0


def test_dambreak_fronts_cross_five_parts(storm_lib):
    sc = scenarios.dambreak(n_target=9000, seed=3)
    _compare(sc, sc.options, 5, rounds=3, steps=20)


def test_steady_channel_four_parts_with_friction(storm_lib):
    """Local time steps, Manning friction (the friction dt is element n_elems's, taken
    from the part that owns it) and the stop test on the combined residual."""
    sc = scenarios.channel(nx=60, ny=10, rstop=1e-7, stop_cr=1)
    _compare(sc, sc.options, 4, rounds=3, steps=150)


def test_mixed_precision_meander(storm_lib):
    sc = scenarios.meander(n_target=9000, seed=8)
    _compare(sc, _opts(sc, precision=abi.PREC_MIXED), 3, rounds=1, steps=30)


def test_link_errors(storm_lib):
    sc = scenarios.meander(n_target=6000, seed=2)
    with pytest.raises(fvt.StormError) as e:
        partition.PartitionedSolver(sc.problem, _opts(sc, rsavg_passes=2, rsavg_order=1, rsavg_eps=0.5), 2)
    assert e.value.code == abi.STORM_ERR_UNSUPPORTED
    p = partition.PartitionedSolver(sc.problem, sc.options, 2)
    ds, de, ss, se = p.halo
    with pytest.raises(fvt.StormError) as e:  # linked already
        fvt._chk(fvt.lib().storm_fvt_link_partitions(p.batch._h, len(ds), abi.iptr(ds), abi.iptr(de),
                                                      abi.iptr(ss), abi.iptr(se), 0))
    assert e.value.code == abi.STORM_ERR_ARG
    p.close()
    pms = [fvt.build_mesh(P.problem) for P in p.parts]
    b = fvt.BatchSolver(pms, sc.options, keep=pms)
    bad = de.copy()
    bad[0] = 10 ** 8  # element out of range
    with pytest.raises(fvt.StormError) as e:
        fvt._chk(fvt.lib().storm_fvt_link_partitions(b._h, len(ds), abi.iptr(ds), abi.iptr(bad),
                                                      abi.iptr(ss), abi.iptr(se), 0))
    assert e.value.code == abi.STORM_ERR_ARG
    b.close()


def test_wind_meander_three_parts(storm_lib):
    """Wind terms at the vertices travel into every part with its nodes."""
    sc = scenarios.meander(n_target=9000, seed=6)
    sc.problem.cd[:] = 0.0
    sc = scenarios.with_wind(sc, scenarios.wind_fields(sc.problem, at_vertices=True, seed=3))
    _compare(sc, sc.options, 3, rounds=1, steps=30)


def _gpu_parts_rank(rank, world, port, which, steps, out):
    import os
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if which == "meander":
            sc = scenarios.meander(n_target=6000, seed=11)
        else:
            sc = scenarios.channel(nx=40, ny=6, rstop=2e-4, stop_cr=1)
        fused = lambda p, o, b: partition.GpuPartEngine(p, o, b, stage_path=fvt.STAGE_FUSED)  # noqa: E731
        dp = partition.DistributedPart(sc.problem, sc.options, rank, world, dist, fused)
        dp.set_state(sc.h0, sc.u0, sc.v0)
        st = dp.step(steps)
        pm = fvt.build_mesh(sc.problem)
        whole = fvt.Solver(pm, sc.options, keep=pm)
        whole.set_state(sc.h0, sc.u0, sc.v0)
        sw = whole.step(steps)
        mine, ref = dp.owned_state(), whole.state()
        c = mine["cells"]
        ok = {k: bool(np.array_equal(mine[k].view(np.uint64), ref[k][c].view(np.uint64)))
              for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        out.put((rank, ok, st["iter"], sw["iter"], bool(st["converged"]), bool(sw["converged"]),
                 st["tmass"], sw["tmass"], dp.engine.solver.stage_path()))
        dp.engine.close()
        whole.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("which,steps", [("meander", 30), ("channel", 3000)])
def test_one_part_per_process_gpu(which, steps, storm_lib):
    """The multi-process decomposition with each part in the CUDA library (fused stage
    kernel): two processes share this one GPU and exchange through the host over gloo
    (no kernel waits on another process).  Owned cells are bit for bit those of the
    undivided GPU run; both stop at the same iteration."""
    import socket
    import torch.multiprocessing as mp
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gpu_parts_rank, args=(r, 2, port, which, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    for rank, ok, it, it_ref, conv, conv_ref, tm, tm_ref, path in res:
        assert all(ok.values()), (rank, ok)
        assert it == it_ref and conv == conv_ref
        assert tm == pytest.approx(tm_ref, rel=1e-13)
        assert path in (fvt.STAGE_PHASES, fvt.STAGE_FUSED)
