"""Python host binding of the FVT step library (ctypes over include/storm_fvt.h).

This mirrors the reference's call sequence at Source_xsy-64bit/solver.f90:50-57:
``read_data`` + ``dataprepFVT`` (here :func:`build_mesh`, or a prepared
:class:`~storm_b200.abi.Mesh` supplied by the caller), then ``solverFVT`` (here
:class:`Solver`: ``set_state`` once, ``step`` as often as output is wanted).  Errors
are raised as :class:`StormError` carrying the library's status code and message,
where the reference would call ``byebye`` and stop.

There is no CPU fallback: loading fails loudly if ``libstorm_fvt.so`` was not built
(``python -m storm_b200.build``) and creating a solver fails without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libstorm_fvt.so")
_lib = None

EXPORTS = (
    "storm_fvt_default_options", "storm_fvt_last_error", "storm_fvt_mesh_build", "storm_fvt_mesh_free",
    "storm_fvt_create", "storm_fvt_set_state", "storm_fvt_step", "storm_fvt_get_state",
    "storm_fvt_get_drycell", "storm_fvt_kernel_launches", "storm_fvt_set_kernel_timing",
    "storm_fvt_last_timing", "storm_fvt_kernel_times", "storm_fvt_destroy",
    "storm_fvt_cfl_dt_noalloc", "storm_fvt_create_batch", "storm_fvt_num_scenarios",
    "storm_fvt_set_scenario_state", "storm_fvt_get_scenario_state", "storm_fvt_scenario_stats",
    "storm_fvt_autotune", "storm_fvt_output_vertices", "storm_fvt_link_partitions",
    "storm_fvt_set_stage_path", "storm_fvt_stage_path", "storm_fvt_tile_check",
    "storm_fvt_set_exchange", "storm_fvt_iter_begin", "storm_fvt_iter_set_dt", "storm_fvt_iter_stage",
    "storm_fvt_iter_fric", "storm_fvt_iter_finish", "storm_fvt_pack_halo", "storm_fvt_unpack_halo",
)

KERNEL_CLASSES = ("node", "grad", "bc", "flux", "fric", "final", "eflux", "tile")
STAGE_PHASES, STAGE_FUSED, STAGE_FUSED_NODE_KERNEL = 0, 1, 2


class StormError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib_path() -> str:
    return _LIB_PATH


def lib():
    """Load libstorm_fvt.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is not built; run `python -m storm_b200.build`")
    L = C.CDLL(_LIB_PATH)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    L.storm_fvt_default_options.argtypes = [C.POINTER(abi.Options)]
    L.storm_fvt_default_options.restype = None
    L.storm_fvt_last_error.restype = C.c_char_p
    L.storm_fvt_mesh_build.argtypes = [C.POINTER(abi.Problem), C.POINTER(C.POINTER(abi.Mesh))]
    L.storm_fvt_mesh_free.argtypes = [C.POINTER(abi.Mesh)]
    L.storm_fvt_mesh_free.restype = None
    L.storm_fvt_create.argtypes = [C.POINTER(abi.Mesh), C.POINTER(abi.Options), C.POINTER(C.c_void_p)]
    L.storm_fvt_set_state.argtypes = [C.c_void_p, dp, dp, dp]
    L.storm_fvt_step.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.StepStats)]
    L.storm_fvt_get_state.argtypes = [C.c_void_p] + [dp] * 7
    L.storm_fvt_get_drycell.argtypes = [C.c_void_p, ip]
    L.storm_fvt_kernel_launches.argtypes = [C.c_void_p]
    L.storm_fvt_kernel_launches.restype = C.c_int64
    L.storm_fvt_set_kernel_timing.argtypes = [C.c_void_p, C.c_int32]
    L.storm_fvt_last_timing.argtypes = [C.c_void_p, dp, dp, C.POINTER(C.c_int64)]
    L.storm_fvt_kernel_times.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int64)]
    L.storm_fvt_destroy.argtypes = [C.c_void_p]
    L.storm_fvt_cfl_dt_noalloc.argtypes = [C.c_void_p] * 5 + [C.c_int32, C.c_double, C.c_double, C.c_double,
                                                                C.c_void_p, C.c_void_p]
    L.storm_fvt_create_batch.argtypes = [C.POINTER(C.POINTER(abi.Mesh)), C.c_int32, C.POINTER(abi.Options),
                                         C.POINTER(C.c_void_p)]
    L.storm_fvt_num_scenarios.argtypes = [C.c_void_p]
    L.storm_fvt_num_scenarios.restype = C.c_int32
    L.storm_fvt_set_scenario_state.argtypes = [C.c_void_p, C.c_int32, dp, dp, dp]
    L.storm_fvt_get_scenario_state.argtypes = [C.c_void_p, C.c_int32] + [dp] * 7
    L.storm_fvt_scenario_stats.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.StepStats)]
    L.storm_fvt_autotune.argtypes = [C.c_void_p, C.c_int32, ip]
    L.storm_fvt_output_vertices.argtypes = [C.c_void_p, C.POINTER(abi.OutputBoundary), C.c_int32] + [dp] * 5
    L.storm_fvt_link_partitions.argtypes = [C.c_void_p, C.c_int32, ip, ip, ip, ip, C.c_int32]
    L.storm_fvt_set_stage_path.argtypes = [C.c_void_p, C.c_int32]
    L.storm_fvt_stage_path.argtypes = [C.c_void_p]
    L.storm_fvt_stage_path.restype = C.c_int32
    L.storm_fvt_tile_check.argtypes = [C.POINTER(C.POINTER(abi.Mesh)), C.c_int32, C.c_int32,
                                       C.POINTER(C.c_int64)]
    L.storm_fvt_set_exchange.argtypes = [C.c_void_p, C.c_int32, ip, C.c_int32, ip]
    L.storm_fvt_iter_begin.argtypes = [C.c_void_p, dp]
    L.storm_fvt_iter_set_dt.argtypes = [C.c_void_p, C.c_double]
    L.storm_fvt_iter_stage.argtypes = [C.c_void_p, C.c_int32, dp]
    L.storm_fvt_iter_fric.argtypes = [C.c_void_p, C.c_double, dp]
    L.storm_fvt_iter_finish.argtypes = [C.c_void_p, dp, C.POINTER(abi.StepStats)]
    L.storm_fvt_pack_halo.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
    L.storm_fvt_unpack_halo.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
    _lib = L
    return L


def _chk(rc: int):
    if rc != 0:
        raise StormError(rc, lib().storm_fvt_last_error().decode())


def tile_check(meshes, tile_cells: int = 256) -> dict:
    """Host-only build and check of the fused kernel's tile plan (storm_fvt_tile_check)."""
    ms = [m.mesh if isinstance(m, PreparedMesh) else m for m in meshes]
    arr = (C.POINTER(abi.Mesh) * len(ms))(*[C.pointer(m) for m in ms])
    st = (C.c_int64 * 8)()
    _chk(lib().storm_fvt_tile_check(arr, len(ms), int(tile_cells), st))
    keys = ("tiles", "ns_max", "ng_max", "ne_max", "h1_cells", "h2_cells", "back_edges", "check")
    return dict(zip(keys, [int(x) for x in st]))


def default_options(**kw) -> abi.Options:
    """The library's defaults (initialize_options.f90) with keyword overrides."""
    o = abi.Options()
    lib().storm_fvt_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


class PreparedMesh:
    """A prepared mesh built by the library (owns the C allocation)."""

    def __init__(self, problem: abi.ProblemHolder):
        self.problem = problem  # keep the input arrays alive
        p = C.POINTER(abi.Mesh)()
        _chk(lib().storm_fvt_mesh_build(C.byref(problem.problem), C.byref(p)))
        self._p = p

    @property
    def mesh(self) -> abi.Mesh:
        return self._p.contents

    def numpy(self) -> dict:
        return abi.mesh_to_numpy(self.mesh)

    def close(self):
        if self._p:
            lib().storm_fvt_mesh_free(self._p)
            self._p = C.POINTER(abi.Mesh)()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_mesh(problem: abi.ProblemHolder) -> PreparedMesh:
    return PreparedMesh(problem)


class Solver:
    """One FVT solver on one GPU (``storm_fvt_create``)."""

    def __init__(self, mesh, options: abi.Options, *, keep=None):
        self._keep = keep  # e.g. the PreparedMesh / oracle owning `mesh`'s arrays
        m = mesh.mesh if isinstance(mesh, PreparedMesh) else mesh
        self.T = m.n_elems
        self.N = m.n_pts
        self.options = options
        h = C.c_void_p()
        _chk(lib().storm_fvt_create(C.byref(m), C.byref(options), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().storm_fvt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, h, u, v):
        h, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, u, v))
        if not (len(h) == len(u) == len(v) == self.T):
            raise ValueError("state arrays must have n_elems entries")
        _chk(lib().storm_fvt_set_state(self._h, abi.dptr(h), abi.dptr(u), abi.dptr(v)))

    def step(self, n: int = 1) -> dict:
        st = abi.StepStats()
        _chk(lib().storm_fvt_step(self._h, int(n), C.byref(st)))
        return st.as_dict()

    def state(self, keys=("h", "u", "v", "rkh", "rku", "rkv", "hvtx")) -> dict:
        """The state in element order; `keys` selects the arrays read back (the
        others are not copied)."""
        out = {k: np.empty(self.N if k == "hvtx" else self.T) for k in keys}
        ptr = lambda k: abi.dptr(out[k]) if k in out else None  # noqa: E731
        _chk(lib().storm_fvt_get_state(self._h, *(ptr(k) for k in ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"))))
        return out

    def output_vertices(self, ob: "abi.OutputBoundaryHolder", in_loop: bool = True) -> dict:
        """The reference's output step (to_vertices, ctr2vtx(cd), error_est(2)) on the
        device; zeroes u,v of wet cells with a dry vertex in the solution, as the
        reference does (``storm_fvt_output_vertices``)."""
        out = {k: np.empty(self.N) for k in ("hvtx", "uvtx", "vvtx", "cdvtx")}
        out["e_est"] = np.empty(self.T)
        _chk(lib().storm_fvt_output_vertices(self._h, C.byref(ob.struct), int(bool(in_loop)),
                                             *(abi.dptr(out[k]) for k in ("hvtx", "uvtx", "vvtx", "cdvtx", "e_est"))))
        return out

    def drycell(self) -> np.ndarray:
        d = np.empty(self.T, dtype=np.int32)
        _chk(lib().storm_fvt_get_drycell(self._h, abi.iptr(d)))
        return d

    def kernel_launches(self) -> int:
        return int(lib().storm_fvt_kernel_launches(self._h))

    def set_kernel_timing(self, on: bool):
        _chk(lib().storm_fvt_set_kernel_timing(self._h, int(bool(on))))

    def last_timing(self) -> dict:
        a, b = C.c_double(), C.c_double()
        n = C.c_int64()
        _chk(lib().storm_fvt_last_timing(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return {"step_ms": a.value, "flux_ms": b.value, "flux_launches": n.value}

    def autotune(self, iters: int = 2) -> dict:
        """Pick block sizes by timing (state restored afterwards)."""
        ch = np.zeros(4, dtype=np.int32)
        _chk(lib().storm_fvt_autotune(self._h, int(iters), abi.iptr(ch)))
        return dict(zip(("node", "grad", "eflux", "flux"), ch.tolist()))

    def set_stage_path(self, path: int):
        """STAGE_PHASES (k_node, k_grad, k_eflux, k_flux: the default) or STAGE_FUSED /
        STAGE_FUSED_NODE_KERNEL (one tile kernel per stage); results are bitwise the
        same in FP64; re-captures the iteration graph."""
        _chk(lib().storm_fvt_set_stage_path(self._h, int(path)))

    def stage_path(self) -> int:
        return int(lib().storm_fvt_stage_path(self._h))

    def kernel_times(self) -> dict:
        """Per-kernel device ms and launch counts of the last step in timing mode."""
        ms = (C.c_double * 8)()
        n = (C.c_int64 * 8)()
        _chk(lib().storm_fvt_kernel_times(self._h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(KERNEL_CLASSES)}


class BatchSolver(Solver):
    """Many independent scenarios advanced together (``storm_fvt_create_batch``): one
    launch per kernel covers every mesh; each scenario has its own dt, clocks, stop
    test and statistics."""

    def __init__(self, meshes, options: abi.Options, *, keep=None):
        self._keep = keep
        ms = [m.mesh if isinstance(m, PreparedMesh) else m for m in meshes]
        self.sizes = [(m.n_elems, m.n_pts) for m in ms]
        self.T = sum(t for t, _ in self.sizes)
        self.N = sum(n for _, n in self.sizes)
        self.options = options
        arr = (C.POINTER(abi.Mesh) * len(ms))(*[C.pointer(m) for m in ms])
        h = C.c_void_p()
        _chk(lib().storm_fvt_create_batch(arr, len(ms), C.byref(options), C.byref(h)))
        self._h = h

    @property
    def n(self) -> int:
        return int(lib().storm_fvt_num_scenarios(self._h))

    def set_scenario_state(self, i: int, h, u, v):
        T = self.sizes[i][0]
        h, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, u, v))
        if not (len(h) == len(u) == len(v) == T):
            raise ValueError("state arrays must have n_elems entries of the scenario")
        _chk(lib().storm_fvt_set_scenario_state(self._h, i, abi.dptr(h), abi.dptr(u), abi.dptr(v)))

    def scenario_stats(self, i: int) -> dict:
        st = abi.StepStats()
        _chk(lib().storm_fvt_scenario_stats(self._h, i, C.byref(st)))
        return st.as_dict()

    def scenario_state(self, i: int) -> dict:
        T, N = self.sizes[i]
        out = {k: np.empty(T) for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        out["hvtx"] = np.empty(N)
        _chk(lib().storm_fvt_get_scenario_state(self._h, i, *(abi.dptr(out[k]) for k in
                                                              ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"))))
        return out
