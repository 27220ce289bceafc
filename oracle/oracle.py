"""ctypes binding of the CPU FP64 oracle (oracle/libstorm_oracle.so).

TEST INFRASTRUCTURE ONLY: a restatement of the reference Fortran solverFVT path
(see storm_oracle.c for the routine-by-routine file:line citations).  Imported by
tests/, the smoke check and bench.py's CPU-baseline leg, never by the product
package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from storm_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libstorm_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(_LIB_PATH)
    return any(os.path.getmtime(os.path.join(_HERE, f)) > t
               for f in ("storm_oracle.c", "storm_oracle.h"))


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.argtypes = [C.POINTER(abi.Problem), C.POINTER(abi.Options), C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_export_mesh.argtypes = [C.c_void_p, C.POINTER(abi.Mesh)]
        L.orc_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_state.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
        L.orc_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(abi.StepStats)]
        L.orc_get_state.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 7
        L.orc_get_drycell.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        L.orc_stage_probe.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32)] + \
            [C.POINTER(C.c_double)] * 4
        L.orc_output_vertices.argtypes = [C.c_void_p, C.POINTER(abi.OutputBoundary), C.c_int] + \
            [C.POINTER(C.c_double)] * 5
        dp = C.POINTER(C.c_double)
        L.orc_iter_begin.argtypes = [C.c_void_p, dp]
        L.orc_iter_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.orc_iter_set_dt.restype = None
        L.orc_iter_stage.argtypes = [C.c_void_p, C.c_int, dp, C.POINTER(C.c_int)]
        L.orc_iter_fric.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_uint8), dp]
        L.orc_iter_finish.argtypes = [C.c_void_p, dp, C.POINTER(abi.StepStats)]
        L.orc_get_level.argtypes = [C.c_void_p, C.c_int, dp]
        L.orc_put_level.argtypes = [C.c_void_p, C.c_int, C.c_int32, C.POINTER(C.c_int32), dp]
        L.orc_set_bch_max.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_bch_max.restype = None
        L.orc_get_bch_max.argtypes = [C.c_void_p]
        L.orc_get_bch_max.restype = C.c_double
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _chk(rc):
    if rc != 0:
        raise OracleError(f"oracle error {rc}: {lib().orc_last_error().decode()}")


class Oracle:
    """The reference algorithm on the CPU: prepare(read_data+dataprepFVT) then step."""

    def __init__(self, problem: abi.ProblemHolder, options: abi.Options, threads: int = 1):
        self.problem = problem
        self.options = options
        h = C.c_void_p()
        _chk(lib().orc_create(C.byref(problem.problem), C.byref(options), C.byref(h)))
        self._h = h
        self.T = problem.n_elems
        self.N = problem.n_pts
        lib().orc_set_threads(self._h, int(threads))

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mesh(self) -> abi.Mesh:
        """The prepared mesh (pointers into the oracle; valid while it lives)."""
        m = abi.Mesh()
        _chk(lib().orc_export_mesh(self._h, C.byref(m)))
        return m

    def mesh_numpy(self) -> dict:
        return abi.mesh_to_numpy(self.mesh())

    def set_threads(self, n: int):
        lib().orc_set_threads(self._h, int(n))

    def set_state(self, h, u, v):
        h, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, u, v))
        _chk(lib().orc_set_state(self._h, abi.dptr(h), abi.dptr(u), abi.dptr(v)))

    def step(self, n: int = 1) -> dict:
        st = abi.StepStats()
        _chk(lib().orc_step(self._h, int(n), C.byref(st)))
        return st.as_dict()

    def state(self) -> dict:
        T, N = self.T, self.N
        out = {k: np.empty(T) for k in ("h", "u", "v", "rkh", "rku", "rkv")}
        out["hvtx"] = np.empty(N)
        _chk(lib().orc_get_state(self._h, *(abi.dptr(out[k]) for k in
                                           ("h", "u", "v", "rkh", "rku", "rkv", "hvtx"))))
        return out

    def output_vertices(self, ob: abi.OutputBoundaryHolder, in_loop: bool = True) -> dict:
        """The reference's output step (orc_output_vertices); zeroes u,v of wet cells
        with a dry vertex, as the reference does."""
        out = {k: np.empty(self.N) for k in ("hvtx", "uvtx", "vvtx", "cdvtx")}
        out["e_est"] = np.empty(self.T)
        _chk(lib().orc_output_vertices(self._h, C.byref(ob.struct), int(bool(in_loop)),
                                       *(abi.dptr(out[k]) for k in ("hvtx", "uvtx", "vvtx", "cdvtx", "e_est"))))
        return out

    def drycell(self) -> np.ndarray:
        d = np.empty(self.T, dtype=np.int32)
        _chk(lib().orc_get_drycell(self._h, abi.iptr(d)))
        return d

    # ---- one iteration in steps (one part of a mesh split over processes) ----
    def iter_begin(self) -> float:
        dt = C.c_double()
        _chk(lib().orc_iter_begin(self._h, C.byref(dt)))
        return dt.value

    def iter_set_dt(self, dt: float):
        lib().orc_iter_set_dt(self._h, float(dt))

    def iter_stage(self, rkstep: int) -> float:
        d, bad = C.c_double(), C.c_int(0)
        _chk(lib().orc_iter_stage(self._h, int(rkstep), C.byref(d), C.byref(bad)))
        return d.value

    def iter_fric(self, dt: float, owned: np.ndarray) -> np.ndarray:
        own = np.ascontiguousarray(owned, dtype=np.uint8)
        sums = np.zeros(4)
        _chk(lib().orc_iter_fric(self._h, float(dt), own.ctypes.data_as(C.POINTER(C.c_uint8)), abi.dptr(sums)))
        return sums

    def iter_finish(self, sums) -> dict:
        s = np.ascontiguousarray(sums, dtype=np.float64)
        st = abi.StepStats()
        _chk(lib().orc_iter_finish(self._h, abi.dptr(s), C.byref(st)))
        return st.as_dict()

    def get_level(self, level: int) -> np.ndarray:
        out = np.empty((6, self.T))
        _chk(lib().orc_get_level(self._h, int(level), abi.dptr(out)))
        return out

    def put_level(self, level: int, elems, values):
        e = np.ascontiguousarray(elems, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64)
        _chk(lib().orc_put_level(self._h, int(level), len(e), abi.iptr(e), abi.dptr(v)))

    def set_bch_max(self, v: float):
        lib().orc_set_bch_max(self._h, float(v))

    def bch_max(self) -> float:
        return float(lib().orc_get_bch_max(self._h))

    def stage_probe(self, rkstep: int = 1, upto: int = 4) -> dict:
        T, N = self.T, self.N
        dry = np.empty(T, dtype=np.int32)
        grads = np.empty(6 * T)
        uv = np.empty(2 * T)
        hv = np.empty(N)
        phi = np.empty(3 * T)
        _chk(lib().orc_stage_probe(self._h, rkstep, upto, abi.iptr(dry), abi.dptr(grads),
                                   abi.dptr(uv), abi.dptr(hv), abi.dptr(phi)))
        return {"dry": dry, "grads": grads.reshape(T, 6), "uv": uv.reshape(T, 2), "hvtx": hv,
                "phi": phi.reshape(T, 3)}
