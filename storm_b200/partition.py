"""Domain decomposition of one mesh into parts with halos of vertex-adjacent rings.

One large mesh is cut into `nparts` parts along a Morton (Z-order) curve of the cell
centroids.  The update of a cell reads its face neighbours' reconstructed states
(their limited LSQ gradients over their own stencils), the vertex values around it
and the dry flags of its face neighbours; every value it reads comes from a cell of
the first ring (face neighbours and the cells at its nodes) or from the state of the
cells of those cells' stencils.  A boundary cell's LSQ stencil (elemnt_db.f90) reaches
neighbours of neighbours, so the halo is three rings of vertex-adjacent cells, and
each part is checked after it is prepared: every owned and first-ring cell must have
exactly the global mesh's stencil, LSQ coefficients, geometry, edges and node weights
(`check_part`); a part that fails gets another ring.  Each extended part is an
ordinary problem (local node and element numbers increasing with the global ones, so
edge orientation and every visiting order of the reference stay the same) prepared by
the library's own mesh builder.

The parts run as the scenarios of one batch handle linked by
``storm_fvt_link_partitions``: after each RK stage and after the friction step the
halo cells take their owners' values, halo cells stay out of the reductions, and the
parts share one dt and one stop test.  The owned cells then evolve bit for bit as in
the undivided mesh.  This is the single-device form of the multi-GPU decomposition;
with one part per GPU the exchange reads the owners' values from the peer GPUs.

Open-boundary strings are kept whole: every cell within two rings of a string's
nodes belongs to the part that owns the string, so no other part's owned or first-
ring cell touches a boundary node or edge.  Culverts (which couple distant cells)
and residual smoothing (an order-dependent sweep) are not supported.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import abi, fvt


def _part1by1(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0xFFFF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
    v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
    v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
    v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
    return v


def morton_order(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Cells sorted along a 16-bit-per-axis Z-order curve of their centroids."""
    def q(a):
        lo, hi = float(a.min()), float(a.max())
        return np.floor((a - lo) / max(hi - lo, 1e-300) * 65535.0).astype(np.int64)
    code = _part1by1(q(x)) | (_part1by1(q(y)) << np.uint64(1))
    return np.argsort(code, kind="stable")


class _Adjacency:
    """Node -> cells lists of a triangulation (0-based), for growing cell sets by one
    ring of vertex-adjacent cells."""

    def __init__(self, tri0: np.ndarray, n_pts: int):
        self.tri0 = tri0
        T = len(tri0)
        flat = tri0.reshape(-1)
        order = np.argsort(flat, kind="stable")
        self.cells = np.repeat(np.arange(T, dtype=np.int64), 3)[order]
        cnt = np.bincount(flat, minlength=n_pts)
        self.off = np.zeros(n_pts + 1, dtype=np.int64)
        np.cumsum(cnt, out=self.off[1:])

    def cells_of_nodes(self, nodes: np.ndarray) -> np.ndarray:
        starts, ends = self.off[nodes], self.off[nodes + 1]
        cnt = ends - starts
        base = np.repeat(starts - np.concatenate(([0], np.cumsum(cnt)[:-1])), cnt)
        return self.cells[base + np.arange(int(cnt.sum()))]

    def grow(self, mask: np.ndarray) -> np.ndarray:
        """The cells sharing a node with a cell of `mask` (the mask included)."""
        out = np.zeros_like(mask)
        nodes = np.unique(self.tri0[mask].reshape(-1))
        out[self.cells_of_nodes(nodes)] = True
        return out


@dataclasses.dataclass
class Part:
    cells: np.ndarray        # global cell ids (0-based, increasing) of the extended part
    owned: np.ndarray        # bool per entry of `cells`: owned (else halo)
    nodes: np.ndarray        # global node ids (0-based, increasing)
    problem: abi.ProblemHolder
    inflow_ids: list         # global indices of the inflow strings this part owns
    outflow_ids: list


def _string_edges(mn: dict, key: str, n: int, ld: int):
    if n == 0:
        return []
    a = mn[key].reshape(n, ld)
    return [a[k, 1:1 + int(a[k, 0])].astype(np.int64) for k in range(n)]


def partition_cells(problem: abi.ProblemHolder, mn: dict, nparts: int) -> np.ndarray:
    """Owner part of every cell: equal Morton-curve chunks, then every open-boundary
    string with its two-ring zone given whole to the part that holds most of the cells
    touching its nodes (zones that meet share one owner)."""
    T, N = int(mn["n_elems"]), int(mn["n_pts"])
    if nparts < 1 or nparts > T:
        raise ValueError("nparts out of range")
    order = morton_order(mn["tri_xc"], mn["tri_yc"])
    part = np.empty(T, dtype=np.int32)
    for p, ch in enumerate(np.array_split(order, nparts)):
        part[ch] = p
    adj = _Adjacency(problem.tri.reshape(T, 3).astype(np.int64) - 1, N)
    E = int(mn["n_edges"])
    ep = mn["edge_p"].reshape(E, 2).astype(np.int64) - 1
    strings = (_string_edges(mn, "bcedgesinflow", int(mn["n_inflowbdr"]), int(mn["bcin_ld"])) +
               _string_edges(mn, "bcedgesoutflow", int(mn["n_outflowbdr"]), int(mn["bcout_ld"])))
    zones = []
    for edges in strings:
        nodes = np.unique(ep[edges - 1].reshape(-1))
        z0 = np.zeros(T, dtype=bool)
        z0[adj.cells_of_nodes(nodes)] = True
        zones.append((z0, adj.grow(adj.grow(z0))))
    # zones that overlap are one group with one owner
    grp = list(range(len(zones)))

    def find(i):
        while grp[i] != i:
            grp[i] = grp[grp[i]]
            i = grp[i]
        return i
    for i in range(len(zones)):
        for j in range(i):
            if np.any(zones[i][1] & zones[j][1]):
                grp[find(i)] = find(j)
    for g in sorted({find(i) for i in range(len(zones))}):
        members = [i for i in range(len(zones)) if find(i) == g]
        z0 = np.logical_or.reduce([zones[i][0] for i in members])
        z2 = np.logical_or.reduce([zones[i][1] for i in members])
        owner = int(np.bincount(part[z0], minlength=nparts).argmax())
        part[z2] = owner
    if len(np.unique(part)) != nparts:
        raise ValueError(f"the mesh does not split into {nparts} non-empty parts with whole boundary strings")
    return part


def extended_parts(problem: abi.ProblemHolder, mn: dict, part: np.ndarray, rings: int = 3,
                   only=None) -> list[Part]:
    """Each part with `rings` rings of vertex-adjacent halo cells, as a problem of its
    own."""
    if problem.problem.n_edges != 0:
        raise ValueError("partitioning needs derived edges (no Triangle .edge input)")
    if problem.culverts:
        raise ValueError("culverts couple distant cells: partitioning does not support them")
    T, N = int(mn["n_elems"]), int(mn["n_pts"])
    tri0 = problem.tri.reshape(T, 3).astype(np.int64) - 1
    adj = _Adjacency(tri0, N)
    zb_v = bool(problem.problem.zb_at_vertices)
    cd_v = bool(problem.problem.cd_at_vertices)
    E = int(mn["n_edges"])
    ee = mn["edge_e"].reshape(E, 2).astype(np.int64)
    ins = _string_edges(mn, "bcedgesinflow", int(mn["n_inflowbdr"]), int(mn["bcin_ld"]))
    outs = _string_edges(mn, "bcedgesoutflow", int(mn["n_outflowbdr"]), int(mn["bcout_ld"]))

    def string_owner(edges):
        c = ee[edges - 1]
        c = np.where(c[:, 0] > 0, c[:, 0], c[:, 1]) - 1
        return int(part[c[0]])
    parts = []
    for p in (range(int(part.max()) + 1) if only is None else only):
        own = part == p
        ext = own
        for _ in range(rings):
            ext = adj.grow(ext)
        cells = np.nonzero(ext)[0]
        nodes = np.unique(tri0[cells].reshape(-1))
        nmap = np.full(N, -1, dtype=np.int64)
        nmap[nodes] = np.arange(len(nodes))
        tri_l = (nmap[tri0[cells]] + 1).astype(np.int32)
        in_ids = [k for k, e in enumerate(ins) if string_owner(e) == p]
        out_ids = [k for k, e in enumerate(outs) if string_owner(e) == p]

        def local_string(spec):
            s = dict(spec)
            ln = nmap[np.asarray(spec["nodes"], dtype=np.int64) - 1]
            if np.any(ln < 0):
                raise ValueError("a boundary string leaves its owning part")
            s["nodes"] = (ln + 1).astype(np.int32)
            return s
        wind = None
        if problem.wind is not None:
            sel = nodes if problem.wind.get("at_vertices", False) else cells
            wind = dict(c0=problem.wind_c0[sel], x=problem.wind_x[sel], y=problem.wind_y[sel],
                        at_vertices=bool(problem.wind.get("at_vertices", False)))
        prob = abi.ProblemHolder(
            problem.x[nodes], problem.y[nodes], tri_l,
            problem.zb[nodes] if zb_v else problem.zb[cells],
            problem.cd[nodes] if cd_v else problem.cd[cells],
            zb_at_vertices=zb_v, cd_at_vertices=cd_v,
            inflow=[local_string(problem.inflow_spec[k]) for k in in_ids],
            outflow=[local_string(problem.outflow_spec[k]) for k in out_ids], wind=wind)
        parts.append(Part(cells=cells, owned=own[cells], nodes=nodes, problem=prob,
                          inflow_ids=in_ids, outflow_ids=out_ids))
    return parts


def check_part(mn: dict, ml: dict, P: Part, adj: _Adjacency) -> int:
    """Number of the part's owned and first-ring cells (and nodes of those cells)
    whose prepared data differ from the global mesh's: stencil (as global ids, in
    order), LSQ weights and coefficients, rc, geometry, face neighbours, vertex order,
    node elevation, incident cells and IDW weights."""
    T, N = int(mn["n_elems"]), int(mn["n_pts"])
    Tl, Nl = int(ml["n_elems"]), int(ml["n_pts"])
    g, gn = P.cells, P.nodes
    own = np.zeros(T, dtype=bool)
    own[g[P.owned]] = True
    li = np.nonzero(adj.grow(own)[g])[0]
    gi = g[li]
    bad = np.zeros(len(li), dtype=bool)

    def cols(d, key, n_rows, ncol):
        return np.asarray(d[key]).reshape(ncol, n_rows).T
    for k in ("tri_area", "tri_perim", "tri_xc", "tri_yc", "z", "cd", "lsq_a", "lsq_b", "lsq_c", "lsq_det"):
        bad |= ml[k][li].view(np.uint64) != mn[k][gi].view(np.uint64)
    for k in ("rc_x", "rc_y"):
        bad |= np.any(cols(ml, k, Tl, 3)[li].view(np.uint64) != cols(mn, k, T, 3)[gi].view(np.uint64), axis=1)
    wl, wg = int(ml["t2t_ncol"]), int(mn["t2t_ncol"])
    lt, gt = cols(ml, "t2t", Tl, wl)[li], cols(mn, "t2t", T, wg)[gi]
    w = max(wl, wg)
    lt = np.pad(lt, ((0, 0), (0, w - wl)))
    gt = np.pad(gt, ((0, 0), (0, w - wg)))
    cnt = lt[:, 0]
    bad |= cnt != gt[:, 0]
    pos = np.arange(1, w)[None, :]
    valid = pos <= cnt[:, None]
    mapped = np.where(valid, g[np.maximum(lt[:, 1:], 1) - 1] + 1, 0)
    bad |= np.any(np.where(valid, mapped != gt[:, 1:], False), axis=1)
    for k in ("lsq_dx", "lsq_dy", "lsq_w"):
        a = np.pad(cols(ml, k, Tl, max(wl - 1, 1))[li], ((0, 0), (0, max(w - 1, 1) - max(wl - 1, 1))))
        b = np.pad(cols(mn, k, T, max(wg - 1, 1))[gi], ((0, 0), (0, max(w - 1, 1) - max(wg - 1, 1))))
        bad |= np.any(np.where(valid[:, :a.shape[1]], a.view(np.uint64) != b.view(np.uint64), False), axis=1)
    l3 = ml["t2t3"].reshape(Tl, 3)[li]
    bad |= np.any(np.where(l3 > 0, g[np.maximum(l3, 1) - 1] + 1, l3) != mn["t2t3"].reshape(T, 3)[gi], axis=1)
    for k in ("tri_vertex", "csortedz"):
        bad |= np.any(gn[ml[k].reshape(Tl, 3)[li] - 1] + 1 != mn[k].reshape(T, 3)[gi], axis=1)
    nl = np.unique(ml["tri_vertex"].reshape(Tl, 3)[li].reshape(-1)) - 1
    ng = gn[nl]
    nbad = ml["zvtx"][nl].view(np.uint64) != mn["zvtx"][ng].view(np.uint64)
    n2l, n2g = cols(ml, "n2t", Nl, int(ml["n2t_ncol"]))[nl], cols(mn, "n2t", N, int(mn["n2t_ncol"]))[ng]
    c2l, c2g = cols(ml, "c2v_w", Nl, int(ml["c2v_ncol"]))[nl], cols(mn, "c2v_w", N, int(mn["c2v_ncol"]))[ng]
    nbad |= n2l[:, 0] != n2g[:, 0]
    for j in range(1, n2l.shape[1]):
        v = j <= n2l[:, 0]
        nbad |= v & (g[np.maximum(n2l[:, j], 1) - 1] + 1 != (n2g[:, j] if j < n2g.shape[1] else 0))
        nbad |= v & (c2l[:, j - 1].view(np.uint64) != (c2g[:, j - 1].view(np.uint64) if j - 1 < c2g.shape[1] else 0))
    return int(bad.sum()) + int(nbad.sum())


def halo_pairs(parts: list[Part], part_of_cell: np.ndarray):
    """(dst part, dst element, src part, src element) of every halo cell, elements
    1-based in each part's own numbering."""
    ds, de, ss, se = [], [], [], []
    for p, P in enumerate(parts):
        halo = P.cells[~P.owned]
        owner = part_of_cell[halo]
        for q in np.unique(owner):
            g = halo[owner == q]
            ds.append(np.full(len(g), p))
            de.append(np.searchsorted(P.cells, g) + 1)
            ss.append(np.full(len(g), q))
            se.append(np.searchsorted(parts[q].cells, g) + 1)
    cat = (lambda a: np.concatenate(a).astype(np.int32) if a else np.zeros(0, np.int32))
    return cat(ds), cat(de), cat(ss), cat(se)


def exchange_plan(parts: list[Part], part_of_cell: np.ndarray) -> dict:
    """Per ordered pair (owner q, receiver p): the owner's local elements (1-based) to
    send and the receiver's local elements to fill, in the same order, for one part
    per process.  Every halo cell appears in exactly one receive list."""
    plan = {}
    for p, P in enumerate(parts):
        halo = P.cells[~P.owned]
        owner = part_of_cell[halo]
        for q in np.unique(owner):
            g = halo[owner == q]
            plan[(int(q), p)] = (np.searchsorted(parts[q].cells, g) + 1, np.searchsorted(P.cells, g) + 1)
    return plan


def exchange_halo(rank: int, plan: dict, fields: list, dist) -> None:
    """One halo exchange between processes (one part each) over a torch.distributed
    process group: every owner sends the values of its cells that other parts hold as
    halo, every part writes what it receives into its halo cells.  `fields` are this
    rank's per-cell arrays (numpy, or tensors on the process group's device).  The
    sends and receives are posted together in (owner, receiver) order, so every rank
    takes the same steps."""
    import torch
    reqs, inbox = [], []
    for (q, p), (src, dst) in sorted(plan.items()):
        if q == rank:
            for f in fields:
                t = torch.as_tensor(f)
                reqs.append(dist.isend(t[torch.as_tensor(src - 1)].contiguous(), dst=p))
        if p == rank:
            for f in fields:
                t = torch.as_tensor(f)
                buf = torch.empty(len(dst), dtype=t.dtype, device=t.device)
                reqs.append(dist.irecv(buf, src=q))
                inbox.append((f, dst, buf))
    for r in reqs:
        r.wait()
    for f, dst, buf in inbox:
        if isinstance(f, np.ndarray):
            f[dst - 1] = buf.numpy()
        else:
            f[torch.as_tensor(dst - 1, device=f.device)] = buf


class PartitionedSolver:
    """One mesh solved as `nparts` linked parts of one batch handle; state and
    statistics in the global element order, as ``fvt.Solver``."""

    def __init__(self, problem: abi.ProblemHolder, options: abi.Options, nparts: int):
        self.problem = problem
        self.options = options
        gm = fvt.build_mesh(problem)
        mn = gm.numpy()
        self.T, self.N = int(mn["n_elems"]), int(mn["n_pts"])
        self.part = partition_cells(problem, mn, nparts)
        tri0 = problem.tri.reshape(self.T, 3).astype(np.int64) - 1
        adj = _Adjacency(tri0, self.N)
        def prepare(p):
            for rings in range(3, 9):
                P = extended_parts(problem, mn, self.part, rings=rings, only=[p])[0]
                pm = fvt.build_mesh(P.problem)
                if check_part(mn, pm.numpy(), P, adj) == 0:
                    return P, pm
                pm.close()
            raise ValueError(f"part {p}: no halo depth reproduces the global mesh's data")
        # the parts are prepared side by side (the mesh builder runs outside the GIL)
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=min(nparts, 8)) as ex:
            done = list(ex.map(prepare, range(nparts)))
        self.parts = [P for P, _ in done]
        self.meshes = [pm for _, pm in done]
        for m in self.meshes:  # the inflow safety-net elevation is a whole-mesh figure
            m.mesh.bch_max = gm.mesh.bch_max
        gm.close()
        self.batch = fvt.BatchSolver(self.meshes, options, keep=self.meshes)
        self.halo = halo_pairs(self.parts, self.part)
        ds, de, ss, se = self.halo
        fric = int(self.part[self.T - 1])
        fvt._chk(fvt.lib().storm_fvt_link_partitions(self.batch._h, len(ds), abi.iptr(ds), abi.iptr(de),
                                                      abi.iptr(ss), abi.iptr(se), fric))

    def close(self):
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, h, u, v):
        h, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, u, v))
        for p, P in enumerate(self.parts):
            self.batch.set_scenario_state(p, h[P.cells], u[P.cells], v[P.cells])

    def step(self, n: int = 1) -> dict:
        st = self.batch.step(n)
        nin = len(self.problem.inflow_spec)
        nout = len(self.problem.outflow_spec)
        cqin = np.zeros(max(nin, 1))
        cqout = np.zeros(max(nout, 1))
        for p, P in enumerate(self.parts):
            sp = self.batch.scenario_stats(p)
            for j, k in enumerate(P.inflow_ids):
                cqin[k] = sp["cqin3"][j]
            for j, k in enumerate(P.outflow_ids):
                cqout[k] = sp["cqout3"][j]
        st["cqin3"] = cqin[:nin]
        st["cqout3"] = cqout[:nout]
        return st

    def state(self) -> dict:
        out = {k: np.empty(self.T) for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        for p, P in enumerate(self.parts):
            s = self.batch.scenario_state(p)
            own = P.cells[P.owned]
            for k in out:
                out[k][own] = s[k][P.owned]
        return out


class DistributedPart:
    """One part of a mesh per process: the multi-process form of the linked parts.

    Every rank holds one extended part (its owned cells plus the halo rings that make
    its prepared data equal to the whole mesh's, `check_part`) in its own `engine` and
    steps it with the exchanges an undivided iteration implies (solverFVT.f90:148-154
    for dt, :335-346 and :407-445 for the friction step, residual and stop test):

    * unsteady with the CFL dt: the iteration's dt is the minimum of the parts' CFL
      minima (all_reduce MIN), exactly the whole mesh's;
    * after every RK stage but the last, and after the friction step, the halo takes
      its owners' h, u, v and that RK level (`exchange_halo`, isend/irecv in (owner,
      receiver) order; NCCL puts the values in this GPU's own buffers);
    * steady: the friction step uses the local dt of element n_elems of the whole mesh
      (N3), broadcast from the part that owns it;
    * the residual sums, the mass (all_reduce SUM) and max |phi| (MAX) come from the
      owned cells of every part, so the stop test is the whole mesh's.

    The owned cells then read exactly the values they read undivided.  `engine` is
    made by make_engine(problem, options, bch_max) for this rank's part (bch_max: the
    whole mesh's inflow safety-net elevation) and provides set_state, iter_begin,
    iter_set_dt, iter_stage, iter_fric, iter_finish and state, and either get_level /
    put_level (host arrays; the state after the friction step is RK level K) or
    set_exchange / pack / unpack (device buffers, GpuPartEngine).  Every rank takes
    the same collective steps in the same order."""

    def __init__(self, problem: abi.ProblemHolder, options: abi.Options, rank: int, world: int, dist, make_engine):
        import torch
        self.rank, self.world, self.dist = rank, world, dist
        self.options = options
        self.K = int(options.rkorder)
        self.device = "cuda" if dist.get_backend() == "nccl" else "cpu"
        gm = fvt.build_mesh(problem)
        mn = gm.numpy()
        self.T = int(mn["n_elems"])
        self.part = partition_cells(problem, mn, world)
        adj = _Adjacency(problem.tri.reshape(self.T, 3).astype(np.int64) - 1, int(mn["n_pts"]))
        rings = 0
        for r in range(3, 9):  # the smallest halo that reproduces the whole mesh's data here
            P = extended_parts(problem, mn, self.part, rings=r, only=[rank])[0]
            pm = fvt.build_mesh(P.problem)
            ok = check_part(mn, pm.numpy(), P, adj) == 0
            pm.close()
            if ok:
                rings = r
                break
        allr = torch.zeros(world, dtype=torch.int64, device=self.device)
        allr[rank] = rings
        dist.all_reduce(allr)
        if int(allr.min()) == 0:
            raise ValueError("a part has no halo depth that reproduces the whole mesh's data")
        parts = [extended_parts(problem, mn, self.part, rings=int(allr[p]), only=[p])[0] for p in range(world)]
        self.P = parts[rank]
        self.plan = exchange_plan(parts, self.part)
        self.halo_elems = (np.nonzero(~self.P.owned)[0] + 1).astype(np.int32)
        self.fric_owner = int(self.part[self.T - 1])
        # the inflow safety net is a whole-mesh figure
        self.engine = make_engine(self.P.problem, options, float(gm.mesh.bch_max))
        gm.close()
        self.device_exchange = hasattr(self.engine, "pack")
        if self.device_exchange:
            # this rank's sends in (receiver) order and receives in (owner) order
            sends = [(p, src) for (q, p), (src, _) in sorted(self.plan.items()) if q == rank]
            recvs = [(q, dst) for (q, p), (_, dst) in sorted(self.plan.items()) if p == rank]
            self.send_off, self.recv_off, o = {}, {}, 0
            for p, src in sends:
                self.send_off[p] = (o, len(src))
                o += len(src)
            o = 0
            for q, dst in recvs:
                self.recv_off[q] = (o, len(dst))
                o += len(dst)
            cat = (lambda a: np.concatenate(a).astype(np.int32) if a else np.zeros(0, np.int32))
            self.send_elems = cat([src for _, src in sends])
            self.recv_elems = cat([dst for _, dst in recvs])
            self.engine.set_exchange(self.send_elems, self.recv_elems)
        self.converged = False

    def _reduce(self, vals, op):
        import torch
        t = torch.tensor(vals, dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return t.cpu().numpy()

    def _exchange(self, level: int, after_fric: bool = False):
        if self.device_exchange:
            return self._exchange_device(0 if after_fric else level, after_fric)
        f = self.engine.get_level(level)
        fields = [np.ascontiguousarray(f[k]) for k in range(6)]
        exchange_halo(self.rank, self.plan, fields, self.dist)
        he = self.halo_elems
        self.engine.put_level(level, he, np.stack([x[he - 1] for x in fields]))

    def _exchange_device(self, level: int, after_fric: bool):
        """Halo values packed on this GPU, sent per peer over the process group (device
        tensors with NCCL, staged through the host with gloo) and unpacked on the GPU."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        host = self.device == "cpu"
        sb = torch.empty((6, len(self.send_elems)), dtype=torch.float64, device=dev)
        self.engine.pack(level, after_fric, sb)
        if host:
            sb = sb.cpu()
        rb = torch.empty((6, len(self.recv_elems)), dtype=torch.float64, device="cpu" if host else dev)
        reqs, inbox = [], []
        for (q, p) in sorted(self.plan):
            if q == self.rank:
                o, n = self.send_off[p]
                reqs.append(self.dist.isend(sb[:, o:o + n].contiguous(), dst=p))
            if p == self.rank:
                o, n = self.recv_off[q]
                buf = torch.empty((6, n), dtype=torch.float64, device=rb.device)
                reqs.append(self.dist.irecv(buf, src=q))
                inbox.append((o, n, buf))
        for r in reqs:
            r.wait()
        for o, n, buf in inbox:
            rb[:, o:o + n] = buf
        if host:
            rb = rb.to(dev)
        torch.cuda.synchronize()
        self.engine.unpack(level, after_fric, rb)

    def set_state(self, h, u, v):
        c = self.P.cells
        self.engine.set_state(np.asarray(h)[c], np.asarray(u)[c], np.asarray(v)[c])
        self.converged = False

    def step(self, n: int = 1) -> dict:
        import torch
        R = self.dist.ReduceOp
        o = self.options
        st = {}
        for _ in range(n):
            if self.converged:
                break
            dt = self.engine.iter_begin()
            if not o.steady and o.dt_op != 0:
                dt = float(self._reduce([dt], R.MIN)[0])
            self.engine.iter_set_dt(dt)
            d_last = dt
            for s in range(1, self.K + 1):
                d_last = self.engine.iter_stage(s)
                if s < self.K:
                    self._exchange(s)
            if o.steady:
                t = torch.tensor([d_last], dtype=torch.float64, device=self.device)
                self.dist.broadcast(t, src=self.fric_owner)
                dfric = float(t.cpu()[0])
            else:
                dfric = dt
            sums = self.engine.iter_fric(dfric, self.P.owned)
            self._exchange(self.K, after_fric=True)
            tot = np.concatenate([self._reduce(list(sums[:3]), R.SUM), self._reduce([sums[3]], R.MAX)])
            st = self.engine.iter_finish(tot)
            self.converged = bool(st["converged"])
        return st

    def owned_state(self) -> dict:
        """The owned cells' state: global ids and h, u, v, rkh, rku, rkv."""
        s = self.engine.state()
        own = self.P.owned
        out = {k: np.asarray(s[k])[own] for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        out["cells"] = self.P.cells[own]
        return out


class GpuPartEngine:
    """A part on this process's GPU through the library's per-process entry points
    (storm_fvt_iter_*, storm_fvt_pack_halo / storm_fvt_unpack_halo)."""

    def __init__(self, problem: abi.ProblemHolder, options: abi.Options, bch_max: float, stage_path=None):
        import ctypes as C
        self._C = C
        self.pm = fvt.build_mesh(problem)
        self.pm.mesh.bch_max = bch_max
        self.solver = fvt.Solver(self.pm, options, keep=self.pm)
        if stage_path is not None:
            self.solver.set_stage_path(stage_path)
        self._h = self.solver._h

    def close(self):
        self.solver.close()

    def set_exchange(self, send_elems, recv_elems):
        s = np.ascontiguousarray(send_elems, dtype=np.int32)
        r = np.ascontiguousarray(recv_elems, dtype=np.int32)
        fvt._chk(fvt.lib().storm_fvt_set_exchange(self._h, len(s), abi.iptr(s), len(r), abi.iptr(r)))

    def set_state(self, h, u, v):
        self.solver.set_state(h, u, v)

    def iter_begin(self) -> float:
        d = self._C.c_double()
        fvt._chk(fvt.lib().storm_fvt_iter_begin(self._h, self._C.byref(d)))
        return d.value

    def iter_set_dt(self, dt: float):
        fvt._chk(fvt.lib().storm_fvt_iter_set_dt(self._h, float(dt)))

    def iter_stage(self, s: int) -> float:
        d = self._C.c_double()
        fvt._chk(fvt.lib().storm_fvt_iter_stage(self._h, int(s), self._C.byref(d)))
        return d.value

    def iter_fric(self, dt: float, owned) -> np.ndarray:
        sums = np.zeros(4)
        fvt._chk(fvt.lib().storm_fvt_iter_fric(self._h, float(dt), abi.dptr(sums)))
        return sums

    def iter_finish(self, sums) -> dict:
        s = np.ascontiguousarray(sums, dtype=np.float64)
        st = abi.StepStats()
        fvt._chk(fvt.lib().storm_fvt_iter_finish(self._h, abi.dptr(s), self._C.byref(st)))
        return st.as_dict()

    def pack(self, level: int, after_fric: bool, buf):
        fvt._chk(fvt.lib().storm_fvt_pack_halo(self._h, int(level), int(bool(after_fric)), buf.data_ptr()))

    def unpack(self, level: int, after_fric: bool, buf):
        fvt._chk(fvt.lib().storm_fvt_unpack_halo(self._h, int(level), int(bool(after_fric)), buf.data_ptr()))

    def state(self) -> dict:
        return self.solver.state()
