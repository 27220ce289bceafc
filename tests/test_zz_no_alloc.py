"""The allocation-free CFL time step (storm_fvt_cfl_dt_noalloc) against storm_fvt_step.

Callers that cannot allocate device memory (an external memory pool owns the GPU,
or the loop cannot take an allocation's implicit synchronisation) use
storm_fvt_cfl_dt_noalloc, whose scratch is a static device
array.  This test allocates the input/output buffers itself (the caller's side),
then checks that two calls in a row give exactly the dt that storm_fvt_step reports
for the next iteration (dt_op = 1): the CFL minimum is order independent and both
kernels evaluate the same per-cell expression, so the tolerance is zero.  The file
is collected last so a failure here cannot hide an earlier one.
"""
import ctypes as C

import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios

pytestmark = pytest.mark.gpu


class Cudart:
    def __init__(self):
        self.rt = None
        for name in ("libcudart.so", "libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"):
            try:
                self.rt = C.CDLL(name)
                break
            except OSError:
                continue
        if self.rt is None:
            pytest.fail("no libcudart could be loaded to allocate the caller's buffers")
        self.rt.cudaMemGetInfo.argtypes = [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        self.rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        self.rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        self.rt.cudaFree.argtypes = [C.c_void_p]
        self.rt.cudaDeviceSynchronize.argtypes = []
        self.bufs = []

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        p = C.c_void_p()
        assert self.rt.cudaMalloc(C.byref(p), max(a.nbytes, 8)) == 0
        assert self.rt.cudaMemcpy(p, a.ctypes.data, a.nbytes, 1) == 0  # host to device
        self.bufs.append(p)
        return p

    def empty(self, n):
        return self.upload(np.zeros(n))

    def download(self, p, n):
        out = np.empty(n)
        assert self.rt.cudaDeviceSynchronize() == 0
        assert self.rt.cudaMemcpy(out.ctypes.data, p, out.nbytes, 2) == 0  # device to host
        return out

    def free_bytes(self):
        assert self.rt.cudaDeviceSynchronize() == 0
        free, total = C.c_size_t(), C.c_size_t()
        assert self.rt.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
        return free.value

    def free(self):
        for p in self.bufs:
            self.rt.cudaFree(p)
        self.bufs = []


def _noalloc_dt(rt, state, area, perim, o, check_free=False):
    """One call on buffers the caller allocated beforehand.  With check_free, the
    device's free memory is read right before and after the call (synchronised): an
    entry point that allocates nothing leaves it unchanged."""
    d = [rt.upload(state["h"]), rt.upload(state["u"]), rt.upload(state["v"]), rt.upload(area), rt.upload(perim)]
    out = rt.empty(1)
    f0 = rt.free_bytes() if check_free else None
    rc = fvt.lib().storm_fvt_cfl_dt_noalloc(*d, len(area), o.cfl, o.h_dry, o.h_wet, out, None)
    assert rc == 0, fvt.lib().storm_fvt_last_error().decode()
    if check_free:
        assert rt.free_bytes() == f0, "the allocation-free entry point changed the device's free memory"
    return rt.download(out, 1)[0]


def test_noalloc_cfl_dt_matches_step(storm_lib):
    sc = scenarios.meander(n_target=20000, seed=21)  # unsteady, dt_op = 1, wet/dry
    assert sc.options.steady == 0 and sc.options.dt_op == 1
    pm = fvt.build_mesh(sc.problem)
    m = pm.numpy()
    area, perim = m["tri_area"], m["tri_perim"]
    g = fvt.Solver(pm, sc.options, keep=pm)
    g.set_state(sc.h0, sc.u0, sc.v0)
    rt = Cudart()
    try:
        st = g.step(3)
        dt1 = _noalloc_dt(rt, g.state(), area, perim, sc.options)  # first call
        assert dt1 == st["delt"], (dt1, st["delt"])
        st = g.step(2)
        dt2 = _noalloc_dt(rt, g.state(), area, perim, sc.options, check_free=True)  # second call, same scratch
        assert dt2 == st["delt"], (dt2, st["delt"])
        assert dt1 != dt2
        # a smaller input after a larger one: stale partials of the earlier call are not read
        k = len(area) // 3
        s = g.state()
        sub = {key: s[key][:k] for key in ("h", "u", "v")}
        dt3 = _noalloc_dt(rt, sub, area[:k], perim[:k], sc.options)
        h, u, v = sub["h"], sub["u"], sub["v"]
        um = np.where(h < sc.options.h_dry, 0.0, np.sqrt(u * u + v * v))
        dry = (h < sc.options.h_dry) | ((h < sc.options.h_wet) & (um == 0.0))
        wc = np.where(dry, 0.0, np.sqrt(9.81 * h))
        ref = np.min(sc.options.cfl * area[:k] / ((um + wc + float(np.float32(1e-9))) * perim[:k]))
        assert dt3 == pytest.approx(ref, rel=1e-14)
    finally:
        rt.free()
        g.close()


def test_noalloc_rejects_oversized_input(storm_lib):
    rt = Cudart()
    try:
        p = rt.empty(4)
        n = 1_048_577
        rc = fvt.lib().storm_fvt_cfl_dt_noalloc(p, p, p, p, p, n, 0.9, 1e-3, 1e-3, p, None)
        assert rc == abi.STORM_ERR_ARG
        assert "exceeds" in fvt.lib().storm_fvt_last_error().decode()
    finally:
        rt.free()
