"""Domain decomposition of one mesh (storm_b200/partition.py): owners, halo rings,
whole boundary strings, and that every part's own prepared mesh holds, for its owned
and first-ring cells and their nodes and edges, exactly the global prepared mesh's
values (so the linked parts can evolve bit for bit as the whole mesh), and that
`check_part` sees a difference when the halo is too thin."""
import numpy as np
import pytest

from storm_b200 import fvt, partition, scenarios


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


CASES = {
    "meander_3": (lambda: scenarios.meander(n_target=12000, seed=5), 3),
    "channel_4": (lambda: scenarios.channel(nx=60, ny=10), 4),
    "dambreak_5": (lambda: scenarios.dambreak(n_target=9000, seed=3), 5),
}


def _global(sc):
    gm = fvt.build_mesh(sc.problem)
    mn = gm.numpy()
    gm.close()
    return mn


@pytest.mark.parametrize("case", sorted(CASES))
def test_owners_rings_and_strings(storm_lib, case):
    mk, P = CASES[case]
    sc = mk()
    mn = _global(sc)
    T = int(mn["n_elems"])
    part = partition.partition_cells(sc.problem, mn, P)
    assert sorted(np.unique(part)) == list(range(P))
    parts = partition.extended_parts(sc.problem, mn, part)
    owned_count = np.zeros(T, dtype=int)
    tri0 = sc.problem.tri.reshape(T, 3).astype(np.int64) - 1
    adj = partition._Adjacency(tri0, int(mn["n_pts"]))
    for p, Pt in enumerate(parts):
        owned_count[Pt.cells[Pt.owned]] += 1
        assert np.all(part[Pt.cells[Pt.owned]] == p) and np.all(part[Pt.cells[~Pt.owned]] != p)
        own = np.zeros(T, dtype=bool)
        own[Pt.cells[Pt.owned]] = True
        three = adj.grow(adj.grow(adj.grow(own)))
        ext = np.zeros(T, dtype=bool)
        ext[Pt.cells] = True
        assert np.array_equal(three, ext)  # exactly three vertex rings around the owned cells
    assert np.all(owned_count == 1)
    # every open-boundary string, with the cells touching its nodes, lies in one part
    E = int(mn["n_edges"])
    ep = mn["edge_p"].reshape(E, 2).astype(np.int64) - 1
    for key, n, ld in (("bcedgesinflow", "n_inflowbdr", "bcin_ld"), ("bcedgesoutflow", "n_outflowbdr", "bcout_ld")):
        for edges in partition._string_edges(mn, key, int(mn[n]), int(mn[ld])):
            cells = adj.cells_of_nodes(np.unique(ep[edges - 1].reshape(-1)))
            assert len(np.unique(part[cells])) == 1


def _rows(a, T, ncol):
    return np.asarray(a).reshape(ncol, T).T if ncol else np.zeros((T, 0))


@pytest.mark.parametrize("case", sorted(CASES))
def test_part_meshes_equal_global_mesh_inside(storm_lib, case):
    mk, P = CASES[case]
    sc = mk()
    mn = _global(sc)
    T, N, E = int(mn["n_elems"]), int(mn["n_pts"]), int(mn["n_edges"])
    part = partition.partition_cells(sc.problem, mn, P)
    parts = partition.extended_parts(sc.problem, mn, part)
    tri0 = sc.problem.tri.reshape(T, 3).astype(np.int64) - 1
    adj = partition._Adjacency(tri0, N)
    g_ep = mn["edge_p"].reshape(E, 2).astype(np.int64)
    g_key = {(min(a, b), max(a, b)): k + 1 for k, (a, b) in enumerate(g_ep)}
    g_t2t = _rows(mn["t2t"], T, mn["t2t_ncol"])
    g_n2t = _rows(mn["n2t"], N, mn["n2t_ncol"])
    g_c2v = _rows(mn["c2v_w"], N, mn["c2v_ncol"])
    g_flow_pos = {int(k): i for i, k in enumerate(mn["flowedg1"])}
    g_wall_pos = {int(k): i for i, k in enumerate(mn["walledg1"])}
    for p, Pt in enumerate(parts):
        pm = fvt.build_mesh(Pt.problem)
        ml = pm.numpy()
        pm.close()
        Tl, Nl, El = int(ml["n_elems"]), int(ml["n_pts"]), int(ml["n_edges"])
        own = np.zeros(T, dtype=bool)
        own[Pt.cells[Pt.owned]] = True
        inner = adj.grow(own)[Pt.cells]          # owned + first ring, local mask
        g = Pt.cells                              # local element -> global (0-based)
        gn = Pt.nodes                             # local node -> global (0-based)
        li = np.nonzero(inner)[0]
        gi = g[li]
        for k in ("tri_area", "tri_perim", "tri_xc", "tri_yc", "z", "cd", "lsq_a", "lsq_b", "lsq_c", "lsq_det"):
            assert np.array_equal(_bits(ml[k][li]), _bits(mn[k][gi])), (p, k)
        for k in ("rc_x", "rc_y"):
            assert np.array_equal(_bits(_rows(ml[k], Tl, 3)[li]), _bits(_rows(mn[k], T, 3)[gi])), (p, k)
        # stencils: same neighbours (as global ids) in the same order, same weights
        l_t2t = _rows(ml["t2t"], Tl, ml["t2t_ncol"])
        for kk in ("lsq_dx", "lsq_dy", "lsq_w"):
            lw = _rows(ml[kk], Tl, max(ml["t2t_ncol"] - 1, 1))
            gw = _rows(mn[kk], T, max(mn["t2t_ncol"] - 1, 1))
            for a, b in zip(li, gi):
                n = int(l_t2t[a, 0])
                assert n == int(g_t2t[b, 0])
                assert np.array_equal(_bits(lw[a, :n]), _bits(gw[b, :n])), (p, kk)
        for a, b in zip(li, gi):
            n = int(l_t2t[a, 0])
            assert np.array_equal(g[l_t2t[a, 1:1 + n] - 1], g_t2t[b, 1:1 + n] - 1)
        l_t3 = ml["t2t3"].reshape(Tl, 3)
        g_t3 = mn["t2t3"].reshape(T, 3)
        m3 = np.where(l_t3[li] > 0, g[np.maximum(l_t3[li], 1) - 1] + 1, l_t3[li])
        assert np.array_equal(m3, g_t3[gi])
        assert np.array_equal(gn[ml["csortedz"].reshape(Tl, 3)[li] - 1] + 1, mn["csortedz"].reshape(T, 3)[gi])
        assert np.array_equal(gn[ml["tri_vertex"].reshape(Tl, 3)[li] - 1] + 1, mn["tri_vertex"].reshape(T, 3)[gi])
        # edges of the inner cells: same global edge, orientation, cells, normal, length
        l_ep = ml["edge_p"].reshape(El, 2).astype(np.int64)
        l_ee = ml["edge_e"].reshape(El, 2).astype(np.int64)
        g_ee = mn["edge_e"].reshape(E, 2).astype(np.int64)
        l_te = ml["tri_edge"].reshape(Tl, 3)
        g_te = mn["tri_edge"].reshape(T, 3)
        l2g_edge = np.zeros(El + 1, dtype=np.int64)
        for k in range(El):
            a, b = gn[l_ep[k] - 1] + 1
            l2g_edge[k + 1] = g_key[(min(a, b), max(a, b))]
        assert np.array_equal(np.sign(l_te[li]) * l2g_edge[np.abs(l_te[li])], g_te[gi])
        ie = np.unique(np.abs(l_te[li]).reshape(-1))
        ge = l2g_edge[ie]
        assert np.array_equal(gn[l_ep[ie - 1] - 1] + 1, g_ep[ge - 1])
        own_l = np.zeros(Tl, dtype=bool)
        own_l[np.nonzero(Pt.owned)[0]] = True
        for k_l, k_g in zip(ie, ge):
            le = l_ee[k_l - 1]
            gl = np.where(le > 0, g[np.maximum(le, 1) - 1] + 1, 0)
            ce = g_ee[k_g - 1]
            if np.all(le > 0) or np.any(own_l[np.maximum(le, 1) - 1] & (le > 0)):
                # an edge of an owned cell keeps both cells (or its boundary kind)
                if np.any((le > 0) & own_l[np.maximum(le, 1) - 1]):
                    assert np.array_equal(gl, np.where(ce > 0, ce, 0)), (p, k_l)
        for k in ("edge_length",):
            assert np.array_equal(_bits(ml[k][ie - 1]), _bits(mn[k][ge - 1]))
        for k in ("edge_normal", "edge_tang"):
            assert np.array_equal(_bits(ml[k].reshape(El, 2)[ie - 1]), _bits(mn[k].reshape(E, 2)[ge - 1]))
        # visiting orders: interior and wall edges of owned cells in the global order
        owned_edges = set(np.abs(l_te[own_l]).reshape(-1).tolist())
        lf = [int(l2g_edge[k]) for k in ml["flowedg1"] if int(k) in owned_edges]
        assert [g_flow_pos[k] for k in lf] == sorted(g_flow_pos[k] for k in lf)
        lw = [int(l2g_edge[k]) for k in ml["walledg1"] if int(k) in owned_edges]
        assert all(k in g_wall_pos for k in lw)
        assert [g_wall_pos[k] for k in lw] == sorted(g_wall_pos[k] for k in lw)
        assert partition.check_part(mn, ml, Pt, adj) == 0
        # nodes of the owned cells: elevation, incident cells and IDW weights
        nodes_l = np.unique(ml["tri_vertex"].reshape(Tl, 3)[own_l].reshape(-1)) - 1
        nodes_g = gn[nodes_l]
        assert np.array_equal(_bits(ml["zvtx"][nodes_l]), _bits(mn["zvtx"][nodes_g]))
        l_n2t = _rows(ml["n2t"], Nl, ml["n2t_ncol"])
        l_c2v = _rows(ml["c2v_w"], Nl, ml["c2v_ncol"])
        for a, b in zip(nodes_l, nodes_g):
            n = int(l_n2t[a, 0])
            assert n == int(g_n2t[b, 0])
            assert np.array_equal(g[l_n2t[a, 1:1 + n] - 1] + 1, g_n2t[b, 1:1 + n])
            assert np.array_equal(_bits(l_c2v[a, :n]), _bits(g_c2v[b, :n]))


def test_halo_pairs_point_at_owners(storm_lib):
    sc = scenarios.meander(n_target=8000, seed=4)
    mn = _global(sc)
    part = partition.partition_cells(sc.problem, mn, 3)
    parts = partition.extended_parts(sc.problem, mn, part)
    ds, de, ss, se = partition.halo_pairs(parts, part)
    assert len(ds) == sum(int((~P.owned).sum()) for P in parts)
    for a, b, c, d in zip(ds, de, ss, se):
        g_dst = parts[a].cells[b - 1]
        g_src = parts[c].cells[d - 1]
        assert g_dst == g_src and part[g_src] == c and parts[c].owned[d - 1]


def test_unsupported_inputs(storm_lib):
    sc = scenarios.culvert_channel()
    mn = _global(sc)
    part = partition.partition_cells(sc.problem, mn, 2)
    with pytest.raises(ValueError):
        partition.extended_parts(sc.problem, mn, part)
    sc2 = scenarios.channel(nx=8, ny=2)
    with pytest.raises(ValueError):
        partition.partition_cells(sc2.problem, _global(sc2), 40)


def test_check_part_sees_a_thin_halo(storm_lib):
    """With two rings a boundary cell of the first ring of the 12k meander misses a
    stencil member (its stencil reaches neighbours of neighbours): check_part counts it."""
    sc = scenarios.meander(n_target=12000, seed=5)
    mn = _global(sc)
    T, N = int(mn["n_elems"]), int(mn["n_pts"])
    part = partition.partition_cells(sc.problem, mn, 3)
    adj = partition._Adjacency(sc.problem.tri.reshape(T, 3).astype(np.int64) - 1, N)
    counts = []
    for rings in (2, 3):
        n = 0
        for Pt in partition.extended_parts(sc.problem, mn, part, rings=rings):
            pm = fvt.build_mesh(Pt.problem)
            n += partition.check_part(mn, pm.numpy(), Pt, adj)
            pm.close()
        counts.append(n)
    assert counts[0] > 0 and counts[1] == 0


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _exchange_rank(rank, world, port, out):
    import os
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = scenarios.meander(n_target=6000, seed=11)
        mn = _global(sc)
        T = int(mn["n_elems"])
        part = partition.partition_cells(sc.problem, mn, world)
        parts = partition.extended_parts(sc.problem, mn, part)
        plan = partition.exchange_plan(parts, part)
        rng = np.random.default_rng(0)
        glob = [rng.random(T), rng.random(T)]          # a whole-mesh state, the same on every rank
        P = parts[rank]
        mine = [np.where(P.owned, g[P.cells], np.nan) for g in glob]  # halo unknown before the exchange
        partition.exchange_halo(rank, plan, mine, dist)
        ok = all(np.array_equal(m, g[P.cells]) for m, g in zip(mine, glob))
        # the whole-mesh mass of this state from the owned cells of every rank
        import torch
        local = torch.tensor([float(np.sum(glob[0][P.cells[P.owned]] * mn["tri_area"][P.cells[P.owned]]))],
                             dtype=torch.float64)
        dist.all_reduce(local)
        out.put((rank, ok, float(local[0]), float(np.sum(glob[0] * mn["tri_area"]))))
    finally:
        dist.destroy_process_group()


def test_halo_exchange_over_two_gloo_ranks():
    """One part per process: after one exchange over gloo every rank's halo cells hold
    the owners' values, and the owned-cell sums add up to the whole mesh's."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    for rank, ok, total, whole in res:
        assert ok, rank
        assert total == pytest.approx(whole, rel=1e-13)


def _oracle_engine(problem, options, bch_max):
    from oracle.oracle import Oracle
    o = Oracle(problem, options)
    o.set_bch_max(bch_max)
    return o


def _parts_rank(rank, world, port, which, steps, out):
    """One rank of the one-part-per-process run: its part stepped through the oracle
    with the real exchanges over gloo, then its owned cells against an undivided
    oracle run of the same steps."""
    import os
    import torch.distributed as dist
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if which == "meander":
            sc = scenarios.meander(n_target=6000, seed=11)        # unsteady, CFL dt, wet/dry, Manning
        else:
            sc = scenarios.channel(nx=40, ny=6, rstop=2e-4, stop_cr=1)  # steady, stop test, friction dt
        dp = partition.DistributedPart(sc.problem, sc.options, rank, world, dist, _oracle_engine)
        dp.set_state(sc.h0, sc.u0, sc.v0)
        st = dp.step(steps)
        whole = Oracle(sc.problem, sc.options)
        whole.set_state(sc.h0, sc.u0, sc.v0)
        so = whole.step(steps)
        mine, ref = dp.owned_state(), whole.state()
        c = mine["cells"]
        ok = {k: bool(np.array_equal(mine[k].view(np.uint64), ref[k][c].view(np.uint64)))
              for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        out.put((rank, ok, st["iter"], so["iter"], bool(st["converged"]), bool(so["converged"]),
                 st["tmass"], so["tmass"], len(c), len(dp.halo_elems)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("which,steps", [("meander", 30), ("channel", 3000)])
def test_one_part_per_process_bitwise_vs_undivided(which, steps):
    """The multi-process decomposition over two gloo ranks: halo exchange after every
    stage and the friction step, global dt minimum, the friction dt of element
    n_elems, global sums for the stop test.  Owned cells are bit for bit those of the
    undivided run and both stop at the same iteration; the mass, summed per part,
    agrees to round-off."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_parts_rank, args=(r, 2, port, which, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    owned = 0
    for rank, ok, it, it_ref, conv, conv_ref, tm, tm_ref, n_own, n_halo in res:
        assert all(ok.values()), (rank, ok)
        assert it == it_ref and conv == conv_ref
        assert tm == pytest.approx(tm_ref, rel=1e-13)
        assert n_halo > 0
        owned += n_own
    if which == "channel":
        assert res[0][4]  # the steady run reached its stop test
    assert owned == scenarios.meander(n_target=6000, seed=11).n_elems if which == "meander" else owned == 480
