"""ctypes mirror of include/storm_fvt.h (the C-ABI of the FVT step library).

The structs here are byte-for-byte the ones a Fortran ISO_C_BINDING shim passes in
place of ``CALL solverFVT`` (Source_xsy-64bit/solver.f90:57).  They are shared by the
product binding (:mod:`storm_b200.fvt`) and by the test oracle's binding.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

STORM_OK = 0
STORM_ERR_ARG = -1
STORM_ERR_MESH = -2
STORM_ERR_CUDA = -3
STORM_ERR_NOMEM = -4
STORM_ERR_DEVICE = -5
STORM_ERR_UNSUPPORTED = -6

FLUX_ROE, FLUX_HLL, FLUX_RUSANOV = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
MAX_BDR = 16

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)


class Options(C.Structure):
    """MODULE options fields read by solverFVT (options.f90), plus flux/precision."""
    _fields_ = [
        ("h_dry", C.c_double), ("h_wet", C.c_double), ("cfl", C.c_double),
        ("vceiling", C.c_double), ("rstop", C.c_double), ("visc", C.c_double),
        ("steady", C.c_int32), ("dt_op", C.c_int32), ("rkorder", C.c_int32),
        ("opt_limiter", C.c_int32), ("btype", C.c_int32), ("hvalve", C.c_int32),
        ("vclip", C.c_int32), ("opt_friction", C.c_int32), ("stop_cr", C.c_int32),
        ("flux", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("rsavg_passes", C.c_int32), ("rsavg_order", C.c_int32), ("rsavg_eps", C.c_double),
        ("reserved", C.c_int32 * 2),
    ]


def default_options(**kw) -> Options:
    """Defaults of initialize_options.f90:23-141 (Roe flux, FP64), then overrides."""
    o = Options()
    o.h_dry = 0.001
    o.h_wet = 0.001
    o.cfl = 1.0
    o.vceiling = 35.0
    o.rstop = float(np.float32(1.0e-4))
    # viscosity(18 C), viscosity.f90: REAL(1.792e-6,mp)/(1 + 0.0337 t + 0.000221 t^2)
    t = 18.0
    o.visc = float(np.float32(1.792e-6)) / (1.0 + 0.0337 * t + 0.000221 * t * t)
    o.steady = 1
    o.dt_op = 0
    o.rkorder = 2
    o.opt_limiter = 2
    o.btype = 0
    o.hvalve = 1
    o.vclip = 0
    o.opt_friction = 0
    o.stop_cr = 0
    o.flux = FLUX_ROE
    o.precision = PREC_FP64
    o.device = 0
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


class Boundary(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("n_nodes", C.c_int32), ("nodes", _i),
        ("value", C.c_double), ("n_series", C.c_int32),
        ("series_t", _d), ("series_v", _d),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("n_pts", C.c_int32), ("n_elems", C.c_int32),
        ("x", _d), ("y", _d), ("tri", _i),
        ("n_edges", C.c_int32), ("edge_p", _i), ("edge_e", _i),
        ("zb", _d), ("zb_at_vertices", C.c_int32),
        ("cd", _d), ("cd_at_vertices", C.c_int32),
        ("n_inflow", C.c_int32), ("inflow", C.POINTER(Boundary)),
        ("n_outflow", C.c_int32), ("outflow", C.POINTER(Boundary)),
        ("wind_c0", _d), ("wind_x", _d), ("wind_y", _d), ("wind_at_vertices", C.c_int32),
        ("n_culvert", C.c_int32), ("cv_ld", C.c_int32), ("cvptoin", _d), ("cvptoout", _d),
        ("ncvtable", _i), ("cvhead", _d), ("cvq", _d),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("n_pts", C.c_int32), ("n_elems", C.c_int32), ("n_edges", C.c_int32),
        ("node_x", _d), ("node_y", _d),
        ("tri_vertex", _i), ("tri_edge", _i),
        ("tri_area", _d), ("tri_perim", _d), ("tri_xc", _d), ("tri_yc", _d),
        ("edge_p", _i), ("edge_e", _i), ("edge_normal", _d), ("edge_tang", _d),
        ("edge_length", _d),
        ("rc_x", _d), ("rc_y", _d),
        ("t2t_ncol", C.c_int32), ("t2t", _i),
        ("lsq_dx", _d), ("lsq_dy", _d), ("lsq_w", _d),
        ("lsq_a", _d), ("lsq_b", _d), ("lsq_c", _d), ("lsq_det", _d),
        ("t2t3", _i),
        ("n2t_ncol", C.c_int32), ("n2t", _i),
        ("c2v_ncol", C.c_int32), ("c2v_w", _d),
        ("csortedz", _i),
        ("flow_edges1", C.c_int32), ("flowedg1", _i),
        ("wall_edges1", C.c_int32), ("walledg1", _i),
        ("n_bcedges", C.c_int32), ("bcedges", _i), ("hbar", _i),
        ("z", _d), ("zvtx", _d), ("cd", _d),
        ("n_inflowbdr", C.c_int32), ("vtype", _i), ("qin", _d),
        ("bcin_ld", C.c_int32), ("bcedgesinflow", _i),
        ("tsq_ld", C.c_int32), ("n_timeserq", _i), ("timelocq", _d), ("timeserq", _d),
        ("n_outflowbdr", C.c_int32), ("htype", _i), ("hbc", _d),
        ("bcout_ld", C.c_int32), ("bcedgesoutflow", _i),
        ("hbc_ld", C.c_int32), ("n_hbc", _i), ("hbc_nodes", _i),
        ("tsh_ld", C.c_int32), ("n_timeserh", _i), ("timeloch", _d), ("timeserh", _d),
        ("bch_max", C.c_double),
        ("wcoef1", _d), ("wcoef2", _d),
        ("n_culvert", C.c_int32), ("cv_ld", C.c_int32), ("cvtrigin", _i), ("cvtrigout", _i),
        ("cvptoin", _d), ("cvrin", _d), ("ncvtable", _i), ("cvhead", _d), ("cvq", _d),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("iter", C.c_int32), ("converged", C.c_int32),
        ("ttime", C.c_double), ("stime", C.c_double), ("delt", C.c_double),
        ("rmax", C.c_double), ("rms_dh", C.c_double), ("tmass", C.c_double),
        ("cqin3", C.c_double * MAX_BDR), ("cqout3", C.c_double * MAX_BDR),
        ("device_status", C.c_int32), ("reserved", C.c_int32 * 7),
    ]

    def as_dict(self) -> dict:
        return {
            "iter": self.iter, "converged": bool(self.converged), "ttime": self.ttime,
            "stime": self.stime, "delt": self.delt, "rmax": self.rmax,
            "rms_dh": self.rms_dh, "tmass": self.tmass,
            "cqin3": list(self.cqin3), "cqout3": list(self.cqout3),
            "device_status": self.device_status,
        }


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_d)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_i)


class ProblemHolder:
    """Owns the numpy arrays behind a :class:`Problem` so the pointers stay valid.

    Inputs mirror what read_data reads: nodes, 1-based CCW triangles, optional
    Triangle .edge/.v.edge data, bed and roughness, and the boundary node strings.
    ``inflow``/``outflow`` are lists of dicts ``{type, nodes, value, series}``
    with ``series`` an optional ``(t, v)`` pair of arrays.
    """

    def __init__(self, x, y, tri, zb, cd, *, zb_at_vertices=True, cd_at_vertices=False,
                 inflow=(), outflow=(), edge_p=None, edge_e=None, wind=None, culverts=()):
        self._keep = []
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.tri = np.ascontiguousarray(tri, dtype=np.int32).reshape(-1)
        self.zb = np.ascontiguousarray(zb, dtype=np.float64)
        self.cd = np.ascontiguousarray(cd, dtype=np.float64)
        self.inflow_spec = [dict(b) for b in inflow]
        self.outflow_spec = [dict(b) for b in outflow]
        p = Problem()
        p.n_pts = len(self.x)
        p.n_elems = len(self.tri) // 3
        p.x, p.y, p.tri = dptr(self.x), dptr(self.y), iptr(self.tri)
        if edge_p is not None:
            self.edge_p = np.ascontiguousarray(edge_p, dtype=np.int32).reshape(-1)
            self.edge_e = np.ascontiguousarray(edge_e, dtype=np.int32).reshape(-1)
            p.n_edges = len(self.edge_p) // 2
            p.edge_p, p.edge_e = iptr(self.edge_p), iptr(self.edge_e)
        else:
            p.n_edges = 0
        p.zb, p.zb_at_vertices = dptr(self.zb), int(zb_at_vertices)
        p.cd, p.cd_at_vertices = dptr(self.cd), int(cd_at_vertices)
        p.n_inflow, p.inflow = self._bdr(self.inflow_spec)
        p.n_outflow, p.outflow = self._bdr(self.outflow_spec)
        # wind: dict(c0=..., x=..., y=..., at_vertices=bool), the windforcing.f90 input
        self.wind = wind
        if wind is not None:
            self.wind_c0 = np.ascontiguousarray(wind["c0"], dtype=np.float64)
            self.wind_x = np.ascontiguousarray(wind["x"], dtype=np.float64)
            self.wind_y = np.ascontiguousarray(wind["y"], dtype=np.float64)
            p.wind_c0, p.wind_x, p.wind_y = dptr(self.wind_c0), dptr(self.wind_x), dptr(self.wind_y)
            p.wind_at_vertices = int(bool(wind.get("at_vertices", False)))
        # culverts: list of dicts(inlet=(x, y, invert), outlet=(x, y), head=[...], q=[...]),
        # the ioculvert.f90 input (performance curve in ascending head)
        self.culverts = [dict(c) for c in culverts]
        if self.culverts:
            n = len(self.culverts)
            ld = max(len(c["head"]) for c in self.culverts)
            self.cvptoin = np.ascontiguousarray([c["inlet"] for c in self.culverts], dtype=np.float64).reshape(-1)
            self.cvptoout = np.ascontiguousarray([c["outlet"] for c in self.culverts], dtype=np.float64).reshape(-1)
            self.ncvtable = np.array([len(c["head"]) for c in self.culverts], dtype=np.int32)
            self.cvhead = np.zeros(ld * n)
            self.cvq = np.zeros(ld * n)
            for i, c in enumerate(self.culverts):
                self.cvhead[i * ld:i * ld + len(c["head"])] = c["head"]
                self.cvq[i * ld:i * ld + len(c["q"])] = c["q"]
            p.n_culvert, p.cv_ld = n, ld
            p.cvptoin, p.cvptoout, p.ncvtable = dptr(self.cvptoin), dptr(self.cvptoout), iptr(self.ncvtable)
            p.cvhead, p.cvq = dptr(self.cvhead), dptr(self.cvq)
        self.problem = p

    def _bdr(self, specs):
        n = len(specs)
        arr = (Boundary * max(n, 1))()
        for i, b in enumerate(specs):
            nodes = np.ascontiguousarray(b["nodes"], dtype=np.int32)
            self._keep.append(nodes)
            arr[i].type = int(b["type"])
            arr[i].n_nodes = len(nodes)
            arr[i].nodes = iptr(nodes)
            arr[i].value = float(b.get("value", 0.0))
            ser = b.get("series")
            if ser is not None:
                t = np.ascontiguousarray(ser[0], dtype=np.float64)
                v = np.ascontiguousarray(ser[1], dtype=np.float64)
                self._keep += [t, v]
                arr[i].n_series = len(t)
                arr[i].series_t, arr[i].series_v = dptr(t), dptr(v)
        self._keep.append(arr)
        return n, arr

    @property
    def n_elems(self) -> int:
        return self.problem.n_elems

    @property
    def n_pts(self) -> int:
        return self.problem.n_pts


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def mesh_to_numpy(m: Mesh) -> dict:
    """Copy every array of a prepared :class:`Mesh` into numpy (for comparisons)."""
    N, T, E = m.n_pts, m.n_elems, m.n_edges
    d = {"n_pts": N, "n_elems": T, "n_edges": E}
    f64, i32 = np.float64, np.int32
    spec = [
        ("node_x", N, f64), ("node_y", N, f64), ("tri_vertex", 3 * T, i32),
        ("tri_edge", 3 * T, i32), ("tri_area", T, f64), ("tri_perim", T, f64),
        ("tri_xc", T, f64), ("tri_yc", T, f64), ("edge_p", 2 * E, i32), ("edge_e", 2 * E, i32),
        ("edge_normal", 2 * E, f64), ("edge_tang", 2 * E, f64), ("edge_length", E, f64),
        ("rc_x", 3 * T, f64), ("rc_y", 3 * T, f64), ("t2t", T * m.t2t_ncol, i32),
        ("lsq_dx", T * max(m.t2t_ncol - 1, 1), f64), ("lsq_dy", T * max(m.t2t_ncol - 1, 1), f64),
        ("lsq_w", T * max(m.t2t_ncol - 1, 1), f64), ("lsq_a", T, f64), ("lsq_b", T, f64),
        ("lsq_c", T, f64), ("lsq_det", T, f64), ("t2t3", 3 * T, i32),
        ("n2t", N * m.n2t_ncol, i32), ("c2v_w", N * m.c2v_ncol, f64), ("csortedz", 3 * T, i32),
        ("flowedg1", m.flow_edges1, i32), ("walledg1", m.wall_edges1, i32),
        ("bcedges", m.n_bcedges, i32), ("hbar", m.n_bcedges, i32),
        ("z", T, f64), ("zvtx", N, f64), ("cd", T, f64),
        ("vtype", m.n_inflowbdr, i32), ("qin", m.n_inflowbdr, f64),
        ("bcedgesinflow", m.bcin_ld * m.n_inflowbdr, i32),
        ("n_timeserq", m.n_inflowbdr, i32), ("timelocq", m.tsq_ld * m.n_inflowbdr, f64),
        ("timeserq", m.tsq_ld * m.n_inflowbdr, f64),
        ("htype", m.n_outflowbdr, i32), ("hbc", m.n_outflowbdr, f64),
        ("bcedgesoutflow", m.bcout_ld * m.n_outflowbdr, i32),
        ("n_hbc", m.n_outflowbdr, i32), ("hbc_nodes", m.hbc_ld * m.n_outflowbdr, i32),
        ("n_timeserh", m.n_outflowbdr, i32), ("timeloch", m.tsh_ld * m.n_outflowbdr, f64),
        ("timeserh", m.tsh_ld * m.n_outflowbdr, f64),
    ]
    for name, n, dt in spec:
        d[name] = _arr(getattr(m, name), n, dt)
    for name in ("wcoef1", "wcoef2"):
        d[name] = _arr(getattr(m, name), T, f64) if getattr(m, name) else None
    n, ld = m.n_culvert, m.cv_ld
    for name, k, dt in (("cvtrigin", n, i32), ("cvtrigout", n, i32), ("cvptoin", 3 * n, f64),
                        ("cvrin", 2 * n, f64), ("ncvtable", n, i32), ("cvhead", ld * n, f64),
                        ("cvq", ld * n, f64)):
        d[name] = _arr(getattr(m, name), k, dt) if n > 0 else None
    d["n_culvert"], d["cv_ld"] = (n, ld) if n > 0 else (0, 0)
    for name in ("t2t_ncol", "n2t_ncol", "c2v_ncol", "flow_edges1", "wall_edges1", "n_bcedges",
                 "n_inflowbdr", "n_outflowbdr", "bcin_ld", "bcout_ld", "hbc_ld", "tsq_ld",
                 "tsh_ld", "bch_max"):
        d[name] = getattr(m, name)
    return d


class OutputBoundary(C.Structure):
    """StormFvtOutputBoundary: boundary arrays of the output-time vertex pass."""
    _fields_ = [
        ("n_wall", C.c_int32), ("wall_pts", _i), ("wtangs", _d), ("qin_ld", C.c_int32),
        ("n_qin", _i), ("qin_nodes", _i), ("pnormals", _d), ("l_inflow", _d), ("qin2", _d),
        ("hbc_ld", C.c_int32), ("hnormals", _d),
    ]


class OutputBoundaryHolder:
    """The arrays the reference builds after read_data for enforce_bcs at output time,
    from a prepared mesh (``mesh_to_numpy``) and the problem's boundary strings:

    * ``wall_pts`` -- walls.f90:170-195: the nodes of the wall edges, in walledg1
      order, without repetitions and without nodes of any boundary string;
    * ``pnormals``/``l_inflow`` -- ibc_arrays.f90:59-135: per inflow string, the
      inward normal of edge i (between nodes i and i+1), moved to the nodes (node n
      takes edge n-1; node i, 1 < i < n, the sum of edges i-1 and i), normalised;
    * ``hnormals`` -- ibc_arrays.f90:181-252 and ``wtangs`` -- :266-345: the sum of
      the outward normals of the two boundary edges at the node, normalised (for
      walls then turned by 90 degrees into a tangent).

    ibc_arrays runs before dataprepFVT normalises the edge normals, so the sums use
    normals of edge-length magnitude; the prepared mesh stores unit normals, which
    are scaled back by the edge length here."""

    def __init__(self, problem: "ProblemHolder", mn: dict):
        T, E = int(mn["n_elems"]), int(mn["n_edges"])
        ep = mn["edge_p"].reshape(E, 2).astype(np.int64)
        ee = mn["edge_e"].reshape(E, 2).astype(np.int64)
        nrm = mn["edge_normal"].reshape(E, 2) * mn["edge_length"][:, None]
        tedge = mn["tri_edge"].reshape(T, 3).astype(np.int64)
        key = {}
        for e in range(E):
            a, b = int(ep[e, 0]), int(ep[e, 1])
            key.setdefault((min(a, b), max(a, b)), e + 1)

        def elem_of(e):
            t = int(ee[e - 1, 0])
            return t if t > 0 else int(ee[e - 1, 1])

        def sign_in(e, t):
            for k in tedge[t - 1]:
                if abs(int(k)) == e:
                    return 1 if k > 0 else -1
            raise ValueError("edge not in its element")

        def unit(v):
            length = np.sqrt(v[0] * v[0] + v[1] * v[1])
            return np.array([v[0] / length, v[1] / length])

        # boundary edges and, per node, the first two of them (bpolygon order: edge id)
        bnd = [e + 1 for e in range(E) if ee[e, 0] <= 0 or ee[e, 1] <= 0]
        at_node = {}
        for e in bnd:
            for p in ep[e - 1]:
                lst = at_node.setdefault(int(p), [])
                if len(lst) < 2:
                    lst.append(e)

        def outward_sum(p):
            es = at_node.get(int(p), [])
            if len(es) < 2:
                es = (es + es)[:2] if es else []
            if not es:
                return np.zeros(2)
            s = np.zeros(2)
            acc = []
            for e in es:
                sg = sign_in(e, elem_of(e))
                acc.append(nrm[e - 1] * (1.0 if sg > 0 else -1.0))
            s = np.array([acc[0][0] + acc[1][0], acc[0][1] + acc[1][1]])
            return unit(s)

        ins = problem.inflow_spec
        qin_nodes_all = set(int(p) for b in ins for p in b["nodes"])
        n_out = int(mn["n_outflowbdr"])
        hld = max(int(mn["hbc_ld"]), 1)
        hbc_nodes = mn["hbc_nodes"].reshape(max(n_out, 0), -1) if n_out else np.zeros((0, hld), np.int32)
        n_hbc = mn["n_hbc"]
        hbc_all = set(int(hbc_nodes[b, i]) for b in range(n_out) for i in range(int(n_hbc[b])))
        # walls.f90:170-195
        wall = []
        seen = set()
        for e in mn["walledg1"]:
            for p in ep[int(e) - 1]:
                p = int(p)
                if p not in seen and p not in qin_nodes_all and p not in hbc_all:
                    seen.add(p)
                    wall.append(p)
        self.wall_pts = np.array(wall, dtype=np.int32)
        wt = np.zeros((len(wall), 2))
        for i, p in enumerate(wall):
            u = outward_sum(p)
            wt[i] = [-u[1], u[0]]
        self.wtangs = np.ascontiguousarray(wt.reshape(-1))
        # ibc_arrays.f90:59-135
        n_in = len(ins)
        self.qin_ld = max([len(b["nodes"]) for b in ins] + [1])
        self.n_qin = np.array([len(b["nodes"]) for b in ins] + [0], dtype=np.int32)[:max(n_in, 1)]
        qn = np.zeros((max(n_in, 1), self.qin_ld), dtype=np.int32)
        pn = np.zeros((max(n_in, 1), self.qin_ld, 2))
        lin = np.zeros((max(n_in, 1), self.qin_ld))
        for b, spec in enumerate(ins):
            nodes = [int(p) for p in spec["nodes"]]
            n = len(nodes)
            qn[b, :n] = nodes
            for i in range(n - 1):
                a, c = nodes[i], nodes[i + 1]
                e = key[(min(a, c), max(a, c))]
                sg = sign_in(e, elem_of(e))
                pn[b, i] = -nrm[e - 1] if sg > 0 else nrm[e - 1]
                lin[b, i] = mn["edge_length"][e - 1]
            if n > 1:
                pn[b, n - 1] = pn[b, n - 2]
            for i in range(n - 2, 0, -1):
                pn[b, i] = [pn[b, i, 0] + pn[b, i - 1, 0], pn[b, i, 1] + pn[b, i - 1, 1]]
            for i in range(n):
                pn[b, i] = unit(pn[b, i])
        self.qin_nodes = np.ascontiguousarray(qn.reshape(-1))
        self.pnormals = np.ascontiguousarray(pn.reshape(-1))
        self.l_inflow = np.ascontiguousarray(lin.reshape(-1))
        self.qin2 = np.zeros(max(n_in, 1))
        # ibc_arrays.f90:181-252
        self.hbc_ld = hld
        hn = np.zeros((max(n_out, 1), hld, 2))
        for b in range(n_out):
            for i in range(int(n_hbc[b])):
                hn[b, i] = outward_sum(hbc_nodes[b, i])
        self.hnormals = np.ascontiguousarray(hn.reshape(-1))
        s = OutputBoundary()
        s.n_wall = len(wall)
        s.wall_pts = iptr(self.wall_pts) if len(wall) else None
        s.wtangs = dptr(self.wtangs) if len(wall) else None
        s.qin_ld = self.qin_ld
        s.n_qin, s.qin_nodes = iptr(self.n_qin), iptr(self.qin_nodes)
        s.pnormals, s.l_inflow, s.qin2 = dptr(self.pnormals), dptr(self.l_inflow), dptr(self.qin2)
        s.hbc_ld, s.hnormals = self.hbc_ld, dptr(self.hnormals)
        self.struct = s
