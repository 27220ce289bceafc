"""Seeded synthetic scenarios for the FVT step (the benchmark workloads).

No public benchmark or dataset exists for the reference (SToRM ships one iRIC case,
tests/Tutorial_1, whose CGNS/HDF5 input holds no solution).  These generators build
stand-ins with the shapes the benchmark configurations name:

* :func:`channel`     -- straight rectangular channel split into triangles (config of
  8,000 cells: 100 m x 10 m, 200 x 20 quads of 0.5 m);
* :func:`meander`     -- Delaunay triangulation of a seeded jittered lattice on a
  floodplain carrying a sine-meandering incised channel, sloped bed plus a seeded
  Gaussian random field (the 2,000,000-triangle transient case);
* :func:`dambreak`    -- Delaunay triangulation of a jittered lattice in a disk, all
  walls, a central water column over a dry bed with seeded Gaussian mounds (the
  1,000,000-triangle wet/dry case).

Each returns a :class:`Scenario`: the raw problem (nodes, CCW triangles, bed,
roughness, boundary node strings), the initial cell state and the solver options.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import abi


@dataclasses.dataclass
class Scenario:
    name: str
    problem: abi.ProblemHolder
    h0: np.ndarray
    u0: np.ndarray
    v0: np.ndarray
    options: abi.Options
    info: dict

    @property
    def n_elems(self) -> int:
        return self.problem.n_elems


def _orient_ccw(x, y, tri):
    """Return 1-based triangles ordered counter-clockwise, zero-area ones dropped."""
    a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
    cross = (x[b] - x[a]) * (y[c] - y[a]) - (x[c] - x[a]) * (y[b] - y[a])
    keep = np.abs(cross) > 1e-12 * (np.abs(x).max() + np.abs(y).max()) ** 2
    tri = tri[keep].copy()
    cross = cross[keep]
    neg = cross < 0
    tri[neg, 1], tri[neg, 2] = tri[neg, 2].copy(), tri[neg, 1].copy()
    return (tri + 1).astype(np.int32)


def _renumber(x, y, tri0):
    """Drop unreferenced nodes; tri0 is 0-based."""
    used = np.zeros(len(x), dtype=bool)
    used[tri0.reshape(-1)] = True
    newid = -np.ones(len(x), dtype=np.int64)
    newid[used] = np.arange(used.sum())
    return x[used], y[used], newid[tri0], newid


def channel(nx: int = 200, ny: int = 20, length: float = 100.0, width: float = 10.0,
            slope: float = 0.001, noise: float = 0.01, manning: float = 0.03, q: float = 10.0,
            depth: float = 1.0, seed: int = 1, **opt) -> Scenario:
    """Straight channel of nx x ny quads, each split along its lower-left to
    upper-right diagonal into two CCW triangles.  Bed (at nodes) is a plane of the
    given slope, z = slope*(length - x), plus seeded uniform noise in
    [-noise, noise].  Inflow discharge q at x = 0 (vtype 1), stage outflow at
    x = length with WSE `depth` above the outlet bed plane (htype 1), walls
    elsewhere.  Initial state: depth `depth`, still water.

    Defaults reproduce the 8,000-cell CPU-runnable configuration: HLL flux, LSQ +
    Barth-Jespersen, SSP-RK3, CFL 0.9, steady to RMS dh 1e-8 or 20,000 steps."""
    rng = np.random.default_rng(seed)
    dx, dy = length / nx, width / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    x = (ii * dx).astype(np.float64).reshape(-1)
    y = (jj * dy).astype(np.float64).reshape(-1)
    nid = lambda i, j: i * (ny + 1) + j  # noqa: E731  (0-based node id, x-major)
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I, J = I.reshape(-1), J.reshape(-1)
    p00, p10, p11, p01 = nid(I, J), nid(I + 1, J), nid(I + 1, J + 1), nid(I, J + 1)
    tri = np.empty((2 * nx * ny, 3), dtype=np.int64)
    tri[0::2] = np.stack([p00, p10, p11], axis=1)
    tri[1::2] = np.stack([p00, p11, p01], axis=1)
    tri = (tri + 1).astype(np.int32)
    zb = slope * (length - x) + rng.uniform(-noise, noise, size=x.shape)
    T = len(tri)
    cd = np.full(T, manning)
    inflow_nodes = np.array([nid(0, j) + 1 for j in range(ny + 1)], dtype=np.int32)
    outflow_nodes = np.array([nid(nx, j) + 1 for j in range(ny + 1)], dtype=np.int32)
    hbc = depth + 0.0  # WSE `depth` above the outlet bed plane (z_plane(length) = 0)
    prob = abi.ProblemHolder(
        x, y, tri, zb, cd, zb_at_vertices=True, cd_at_vertices=False,
        inflow=[{"type": 1, "nodes": inflow_nodes, "value": q}],
        outflow=[{"type": 1, "nodes": outflow_nodes, "value": hbc}])
    o = dict(rkorder=3, opt_limiter=2, flux=abi.FLUX_HLL, cfl=0.9, steady=1, stop_cr=1,
             rstop=1e-8, btype=0, hvalve=1, h_dry=1e-3, h_wet=1e-3, opt_friction=0)
    o.update(opt)
    options = abi.default_options(**o)
    h0 = np.full(T, depth)
    return Scenario("channel", prob, h0, np.zeros(T), np.zeros(T), options,
                    {"nx": nx, "ny": ny, "diagonal": "lower-left to upper-right", "seed": seed,
                     "istop": 20000})


def _grf(x, y, sigma, ell, rng, modes=256):
    """Gaussian random field with Gaussian covariance sigma^2 exp(-r^2/(2 ell^2)),
    by a sum of random Fourier modes (wave vectors drawn from the spectral density)."""
    k = rng.normal(0.0, 1.0 / ell, size=(modes, 2))
    ph = rng.uniform(0.0, 2 * np.pi, size=modes)
    out = np.zeros_like(x)
    chunk = 1 << 16
    amp = sigma * np.sqrt(2.0 / modes)
    for s in range(0, len(x), chunk):
        xs, ys = x[s:s + chunk, None], y[s:s + chunk, None]
        out[s:s + chunk] = amp * np.cos(xs * k[:, 0] + ys * k[:, 1] + ph).sum(axis=1)
    return out


def _delaunay(x, y):
    from scipy.spatial import Delaunay
    return Delaunay(np.stack([x, y], axis=1)).simplices.astype(np.int64)


def _boundary_string(x, y, tri1, sel):
    """Nodes on the mesh boundary selected by `sel` (bool per node), ordered as a
    chain of boundary edges.  tri1 is 1-based."""
    t = tri1.astype(np.int64) - 1
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    key = np.minimum(e[:, 0], e[:, 1]) * (len(x) + 1) + np.maximum(e[:, 0], e[:, 1])
    uk, cnt = np.unique(key, return_counts=True)
    bkeys = uk[cnt == 1]
    a, b = bkeys // (len(x) + 1), bkeys % (len(x) + 1)
    m = sel[a] & sel[b]
    a, b = a[m], b[m]
    adj = {}
    for p, q in zip(a.tolist(), b.tolist()):
        adj.setdefault(p, []).append(q)
        adj.setdefault(q, []).append(p)
    ends = [p for p, n in adj.items() if len(n) == 1]
    if not ends:
        raise ValueError("boundary selection is not an open chain")
    start = min(ends, key=lambda p: (y[p], x[p]))
    chain, prev, cur = [start], -1, start
    while True:
        nxt = [q for q in adj[cur] if q != prev]
        if not nxt:
            break
        prev, cur = cur, nxt[0]
        chain.append(cur)
    if len(chain) != len(adj):
        raise ValueError("boundary selection is not a single chain")
    return np.array(chain, dtype=np.int32) + 1


def meander(n_target: int = 2_000_000, length: float = 4000.0, valley: float = 200.0,
            wavelength: float = 400.0, amplitude: float = 60.0, chan_width: float = 40.0,
            chan_depth: float = 2.0, slope: float = 0.0005, grf_sigma: float = 0.5,
            grf_ell: float = 20.0, jitter: float = 0.3, q: float = 200.0, dry_frac: float = 0.30,
            seed: int = 2, **opt) -> Scenario:
    """Large transient case: a floodplain valley `length` x `valley` carrying a
    sine-meandering channel (centreline y = amplitude*sin(2 pi x/wavelength),
    `chan_width` wide, incised `chan_depth` with a parabolic section).  Nodes are a
    seeded jittered lattice (interior jitter `jitter` x spacing; boundary nodes slide
    along the boundary only), triangulated by Delaunay.  Bed = slope*(length - x)
    + GRF(sigma 0.5 m, correlation length 20 m) + channel incision.  Manning n is
    U[0.02, 0.06] per cell.  The initial water surface is the bed plane plus the
    constant that leaves `dry_frac` of the cells with h < 1e-4 m.  Inflow Q at
    x = 0 across the valley (vtype 1); stage outflow at x = length holding the
    initial water surface there (htype 1).  Fixed, recorded choices: valley width
    200 m, incision 2 m, outflow stage = initial WSE."""
    rng = np.random.default_rng(seed)
    aspect = length / valley
    ny = max(2, int(round(np.sqrt(n_target / (2 * aspect)))))
    nx = max(2, int(round(n_target / (2 * ny))))
    hx, hy = length / nx, valley / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    x = ii.reshape(-1) * hx
    y = jj.reshape(-1) * hy - valley / 2
    jx = rng.uniform(-jitter, jitter, size=x.shape) * hx
    jy = rng.uniform(-jitter, jitter, size=x.shape) * hy
    ib = (ii.reshape(-1) == 0) | (ii.reshape(-1) == nx)
    jb = (jj.reshape(-1) == 0) | (jj.reshape(-1) == ny)
    x = x + np.where(ib, 0.0, jx)
    y = y + np.where(jb, 0.0, jy)
    tri0 = _delaunay(x, y)
    tri1 = _orient_ccw(x, y, tri0)
    x, y, renum, _ = _renumber(x, y, tri1 - 1)
    tri1 = (renum + 1).astype(np.int32)
    yc = amplitude * np.sin(2 * np.pi * x / wavelength)
    d = np.abs(y - yc) / (chan_width / 2)
    incision = -chan_depth * np.clip(1.0 - d * d, 0.0, None)
    zb = slope * (length - x) + _grf(x, y, grf_sigma, grf_ell, rng) + incision
    T = len(tri1)
    cd = rng.uniform(0.02, 0.06, size=T)
    t0 = tri1 - 1
    zc = (zb[t0[:, 0]] + zb[t0[:, 1]] + zb[t0[:, 2]]) / 3.0
    xc = (x[t0[:, 0]] + x[t0[:, 1]] + x[t0[:, 2]]) / 3.0
    rel = zc - slope * (length - xc)
    c = float(np.quantile(rel, 1.0 - dry_frac))
    h0 = np.maximum(slope * (length - xc) + c - zc, 0.0)
    h0[h0 < 1e-4] = 0.0
    tol = 1e-9 * length
    inflow = _boundary_string(x, y, tri1, np.abs(x) < tol)
    outflow = _boundary_string(x, y, tri1, np.abs(x - length) < tol)
    hbc = c  # initial WSE at x = length (bed plane is 0 there)
    prob = abi.ProblemHolder(x, y, tri1, zb, cd, zb_at_vertices=True, cd_at_vertices=False,
                             inflow=[{"type": 1, "nodes": inflow, "value": q}],
                             outflow=[{"type": 1, "nodes": outflow, "value": hbc}])
    o = dict(rkorder=3, opt_limiter=2, flux=abi.FLUX_ROE, cfl=0.9, steady=0, dt_op=1,
             btype=0, hvalve=1, h_dry=1e-4, h_wet=1e-4, opt_friction=0)
    o.update(opt)
    options = abi.default_options(**o)
    return Scenario("meander", prob, h0, np.zeros(T), np.zeros(T), options,
                    {"nx": nx, "ny": ny, "seed": seed, "valley": valley,
                     "dry_fraction": float(np.mean(h0 < 1e-4)), "hbc": hbc})


def dambreak(n_target: int = 1_000_000, radius: float = 500.0, col_radius: float = 50.0,
             col_depth: float = 10.0, n_mounds: int = 10, manning: float = 0.025,
             jitter: float = 0.3, seed: int = 3, **opt) -> Scenario:
    """Circular dam break on a disk of `radius`, all boundary edges walls (no
    inflow/outflow strings).  Nodes: a seeded jittered square lattice inside the disk
    plus equally spaced nodes on the circle, triangulated by Delaunay.  Bed: flat
    plus `n_mounds` seeded Gaussian mounds (height U[0.5,2] m, radius U[10,40] m).
    Initial depth `col_depth` inside r < col_radius, dry elsewhere.  Rusanov flux,
    unsteady with the CFL dt (CFL 0.9); the full case runs 60 s simulated."""
    rng = np.random.default_rng(seed)
    area = np.pi * radius * radius
    h = np.sqrt(area / (n_target / 2.0))
    n = int(np.ceil(radius / h))
    g1 = (np.arange(-n, n + 1) * h)
    X, Y = np.meshgrid(g1, g1, indexing="ij")
    X = X.reshape(-1) + rng.uniform(-jitter, jitter, size=X.size) * h
    Y = Y.reshape(-1) + rng.uniform(-jitter, jitter, size=Y.size) * h
    keep = np.hypot(X, Y) < radius - 0.6 * h
    nb = int(np.ceil(2 * np.pi * radius / h))
    th = np.arange(nb) * (2 * np.pi / nb)
    x = np.concatenate([X[keep], radius * np.cos(th)])
    y = np.concatenate([Y[keep], radius * np.sin(th)])
    tri1 = _orient_ccw(x, y, _delaunay(x, y))
    x, y, renum, _ = _renumber(x, y, tri1 - 1)
    tri1 = (renum + 1).astype(np.int32)
    zb = np.zeros_like(x)
    for _ in range(n_mounds):
        r0 = rng.uniform(0.1, 0.9) * radius
        a0 = rng.uniform(0, 2 * np.pi)
        hm = rng.uniform(0.5, 2.0)
        rm = rng.uniform(10.0, 40.0)
        cx, cy = r0 * np.cos(a0), r0 * np.sin(a0)
        zb += hm * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * rm * rm))
    T = len(tri1)
    t0 = tri1 - 1
    xc = (x[t0[:, 0]] + x[t0[:, 1]] + x[t0[:, 2]]) / 3.0
    yc = (y[t0[:, 0]] + y[t0[:, 1]] + y[t0[:, 2]]) / 3.0
    h0 = np.where(np.hypot(xc, yc) < col_radius, col_depth, 0.0)
    cd = np.full(T, manning)
    prob = abi.ProblemHolder(x, y, tri1, zb, cd, zb_at_vertices=True, cd_at_vertices=False)
    o = dict(rkorder=3, opt_limiter=2, flux=abi.FLUX_RUSANOV, cfl=0.9, steady=0, dt_op=1,
             btype=0, hvalve=1, h_dry=1e-3, h_wet=1e-3, opt_friction=0)
    o.update(opt)
    options = abi.default_options(**o)
    return Scenario("dambreak", prob, h0, np.zeros(T), np.zeros(T), options,
                    {"seed": seed, "spacing": h, "t_end": 60.0})


def wind_fields(problem, at_vertices: bool, seed: int = 11, c0=(1.0e-3, 1.6e-3), wx=(-20.0, 20.0),
                wy=(-5.0, 5.0)) -> dict:
    """A spatially varying wind in the windforcing.f90 text-input form: drag
    coefficient c0 and wind velocity (x, y) in m/s, uniform random in the given
    ranges, on the vertices or the cells of a problem."""
    n = problem.n_pts if at_vertices else problem.n_elems
    rng = np.random.default_rng(seed)
    return dict(c0=rng.uniform(*c0, n), x=rng.uniform(*wx, n), y=rng.uniform(*wy, n), at_vertices=at_vertices)


def with_wind(sc: Scenario, wind: dict) -> Scenario:
    """The same scenario with wind forcing terms."""
    p = sc.problem
    sc.problem = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, p.cd, inflow=p.inflow_spec, outflow=p.outflow_spec,
                                   wind=wind, culverts=p.culverts)
    return sc


def with_culverts(sc: Scenario, culverts) -> Scenario:
    """The same scenario with culverts (ioculvert.f90 input, see ProblemHolder)."""
    p = sc.problem
    sc.problem = abi.ProblemHolder(p.x, p.y, p.tri, p.zb, p.cd, inflow=p.inflow_spec, outflow=p.outflow_spec,
                                   wind=p.wind, culverts=culverts)
    return sc


def culvert_channel(nx: int = 60, ny: int = 8, q: float = 2.0, crest: float = 1.5, **kw) -> Scenario:
    """A 60 x 8 m channel crossed by an embankment (bed raised by `crest` m for
    28 m <= x <= 32 m) with two culverts through it: water ponds upstream, the
    culverts carry it across by their performance curves (head above the invert
    -> discharge), and it flows on to the outlet."""
    sc = channel(nx=nx, ny=ny, length=60.0, width=8.0, q=q, **kw)
    p = sc.problem
    zb = p.zb.copy()
    zb[(p.x >= 28.0) & (p.x <= 32.0)] += crest
    sc.problem = abi.ProblemHolder(p.x, p.y, p.tri, zb, p.cd, inflow=p.inflow_spec, outflow=p.outflow_spec)
    # dry embankment cells at the start (their bed is above the initial surface)
    xc = p.x[p.tri.reshape(-1, 3) - 1].mean(axis=1)
    sc.h0 = np.where((xc > 28.0) & (xc < 32.0), 0.0, sc.h0)
    zin = 0.001 * (60.0 - 25.0) - 0.05  # invert just below the bed plane at x = 25
    curve = dict(head=[0.1, 0.5, 1.0, 2.0], q=[0.0, 0.6, 1.5, 3.5])
    cvs = [dict(inlet=(25.1, 2.05, zin), outlet=(35.2, 2.1), **curve),
           dict(inlet=(25.3, 5.95, zin), outlet=(35.1, 6.0), head=[0.2, 1.2], q=[0.1, 1.1])]
    return with_culverts(sc, cvs)


def algorithmic_bytes_per_cell_stage(n_elems: int, n_edges: int, n_pts: int,
                                     mean_valence: float | None = None) -> float:
    """Compulsory HBM bytes of one perfectly fused FP64 RK stage per cell:
    B = 232 + 42 E/T + 20 N/T + 12 vbar N/T  (vbar N = 3T makes the last term 36)."""
    T, E, N = float(n_elems), float(n_edges), float(n_pts)
    vbar = 3.0 * T / N if mean_valence is None else mean_valence
    return 232.0 + 42.0 * E / T + 20.0 * N / T + 12.0 * vbar * N / T


def meander_channel(n_cells: int, width: float, q: float, manning: float, stage: float, seed: int,
                    slope: float = 0.001, cells_across: int = 0, cover_inlet: bool = True,
                    **opt) -> Scenario:
    """One steady ensemble member: a sine-meandering channel with the proportions and
    bed of the straight 100 m x 10 m channel (length 10 widths, square quads each split
    along one diagonal, bed slope 0.001 plus seeded noise of +-1 cm), bent along a
    sine centreline of seeded wavelength (8-15 widths) and amplitude (0.5-1.5 widths);
    about `n_cells` triangles.  Manning n and inflow Q (vtype 1) as given.  The
    downstream water surface (htype 1) stands `stage` m above the Manning normal depth
    of the member, h_n = (n Q / (W sqrt(S)))^(3/5), so the outlet stays subcritical:
    with the stage counted from the bed, members with a large unit discharge put a
    stage boundary on supercritical outflow, where the reference scheme (and this
    port, bit for bit) diverges.  Cold start: still water with a flat surface at the
    outlet level, raised where needed so the inlet carries at least h_n."""
    rng = np.random.default_rng(seed)
    ny = cells_across or int(np.clip(round(np.sqrt(n_cells / 20.0)), 6, 200))
    nx = max(4, int(round(n_cells / (2 * ny))))
    ds = width / ny
    length = nx * ds
    lam = rng.uniform(8.0, 15.0) * width
    amp = rng.uniform(0.5, 1.5) * width
    # centreline by arc length: y = amp sin(2 pi x / lam), sampled finely then resampled
    xf = np.linspace(0.0, length * 1.5, 20 * nx + 1)
    yf = amp * np.sin(2 * np.pi * xf / lam)
    sf = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xf), np.diff(yf)))])
    s = np.arange(nx + 1) * ds
    cx = np.interp(s, sf, xf)
    cy = np.interp(s, sf, yf)
    tx = np.gradient(cx)
    ty = np.gradient(cy)
    tn = np.hypot(tx, ty)
    nxv, nyv = -ty / tn, tx / tn
    off = (np.arange(ny + 1) / ny - 0.5) * width
    X = (cx[:, None] + off[None, :] * nxv[:, None]).reshape(-1)
    Y = (cy[:, None] + off[None, :] * nyv[:, None]).reshape(-1)
    S = np.repeat(s, ny + 1)
    nid = lambda i, j: i * (ny + 1) + j  # noqa: E731
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I, J = I.reshape(-1), J.reshape(-1)
    p00, p10, p11, p01 = nid(I, J), nid(I + 1, J), nid(I + 1, J + 1), nid(I, J + 1)
    tri = np.empty((2 * nx * ny, 3), dtype=np.int64)
    tri[0::2] = np.stack([p00, p10, p11], axis=1)
    tri[1::2] = np.stack([p00, p11, p01], axis=1)
    tri1 = _orient_ccw(X, Y, tri)
    zb = slope * (length - S) + rng.uniform(-0.01, 0.01, size=S.shape)
    T = len(tri1)
    h_normal = (manning * q / (width * np.sqrt(slope))) ** 0.6
    hbc = h_normal + stage  # outlet bed plane is at 0
    t0 = tri1.astype(np.int64) - 1
    zc = (zb[t0[:, 0]] + zb[t0[:, 1]] + zb[t0[:, 2]]) / 3.0
    wse0 = hbc
    if cover_inlet:
        wse0 = max(hbc, float(zb[: ny + 1].max()) + h_normal)
    h0 = np.maximum(wse0 - zc, 0.0)
    prob = abi.ProblemHolder(
        X, Y, tri1, zb, np.full(T, manning), zb_at_vertices=True, cd_at_vertices=False,
        inflow=[{"type": 1, "nodes": np.array([nid(0, j) + 1 for j in range(ny + 1)]), "value": q}],
        outflow=[{"type": 1, "nodes": np.array([nid(nx, j) + 1 for j in range(ny + 1)]), "value": hbc}])
    o = dict(rkorder=3, opt_limiter=2, flux=abi.FLUX_HLL, cfl=0.9, steady=1, stop_cr=1, rstop=1e-6,
             btype=0, hvalve=1, h_dry=1e-3, h_wet=1e-3, opt_friction=0)
    o.update(opt)
    return Scenario("meander_channel", prob, h0, np.zeros(T), np.zeros(T), abi.default_options(**o),
                    {"seed": seed, "width": width, "q": q, "manning": manning, "stage": stage,
                     "h_normal": h_normal, "hbc": hbc, "wse0": wse0, "slope": slope, "nx": nx, "ny": ny,
                     "wavelength": lam, "amplitude": amp})


def batch_channel_params(n_scen: int = 256, lo: int = 20_000, hi: int = 400_000, seed: int = 4) -> list:
    """Parameters of the ensemble members (no meshes built): sizes log-uniform in
    [lo, hi] triangles, width U[20,80] m, Q U[20,500] m^3/s, n U[0.02,0.06],
    downstream stage U[0.5,3] m above normal depth, one mesh seed per member."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_scen):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        out.append(dict(n_cells=n, width=rng.uniform(20, 80), q=rng.uniform(20, 500),
                        manning=rng.uniform(0.02, 0.06), stage=rng.uniform(0.5, 3.0),
                        seed=int(rng.integers(1 << 30))))
    return out


def batch_channels(n_scen: int = 256, lo: int = 20_000, hi: int = 400_000, seed: int = 4, only=None,
                   **opt) -> list:
    """The batched steady ensemble: one :func:`meander_channel` per member of
    :func:`batch_channel_params`; `only` (indices) builds a subset, in that order."""
    params = batch_channel_params(n_scen, lo, hi, seed)
    idx = range(n_scen) if only is None else only
    return [meander_channel(**params[i], **opt) for i in idx]
