"""Learned warm start for steady runs: a message-passing network on the cell-dual
graph, trained and run on the GPU by the library's own tcgen05 kernels
(include/storm_gnn.h).

SToRM has no such component: a steady run (solverFVT.f90:129-478 with ``steady``)
starts from the initial condition the user supplies.  Here the network predicts an
initial h, hu, hv from the bed, roughness, cell geometry and the boundary discharge
and stage; the solver then runs from that field to its own stop test, so the solver
remains both the fallback and the arbiter of the result.

Architecture (encode / process / decode):

* node input (64 features, zero padded) -> node encoder MLP 64 -> 128 -> 128;
* edge input (64 features) -> edge encoder MLP 64 -> 128 -> 128;
* 8 processor layers, each ``e' = e + MLP_e([e, h_src, h_dst])`` (384 -> 128 -> 128)
  then ``h' = h + MLP_n([h, sum_k e'_k])`` (256 -> 128 -> 128);
* decoder MLP 128 -> 128 -> 64 whose first three outputs are the targets.

Every MLP is ``W2 relu(W1 x + b1) + b2`` with bf16 weights and activations and fp32
accumulation in TMEM.  PyTorch is used only to hold device memory; every operation
on the network's data is a kernel of libstorm_fvt.so.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import fvt

HID = 128
N_LAYERS = 8
IN_NODE = 64
IN_EDGE = 64
N_OUT_PAD = 64
N_TARGET = 3

_vp = C.c_void_p
_ip = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)


class Seg(C.Structure):
    _fields_ = [("src", _vp), ("idx", _vp), ("width", C.c_int32), ("agg", C.c_int32),
                ("agg_stride", C.c_int32), ("nbr", _vp)]


class MlpFwd(C.Structure):
    _fields_ = [("rows", C.c_int32), ("nseg", C.c_int32), ("k_in", C.c_int32), ("n_out", C.c_int32),
                ("seg", Seg * 3), ("w1", _vp), ("b1", _vp), ("w2", _vp), ("b2", _vp), ("res", _vp),
                ("out", _vp), ("out_f32", _vp), ("a1_save", _vp)]


class MlpBwdData(C.Structure):
    _fields_ = [("rows", C.c_int32), ("nseg", C.c_int32), ("k_in", C.c_int32), ("n_out", C.c_int32),
                ("seg_width", C.c_int32 * 3), ("dseg", _vp * 3), ("dseg_add", _vp * 3), ("dy", _vp),
                ("a1", _vp), ("w1", _vp), ("w2", _vp), ("dz1_save", _vp)]


class MlpBwdWeight(C.Structure):
    _fields_ = [("rows", C.c_int32), ("nseg", C.c_int32), ("k_in", C.c_int32), ("n_out", C.c_int32),
                ("seg", Seg * 3), ("dy", _vp), ("a1", _vp), ("dz1", _vp)]


EXPORTS = ("storm_gnn_grad_size", "storm_gnn_weight_scratch_bytes", "storm_gnn_mlp_forward",
           "storm_gnn_mlp_backward_data", "storm_gnn_mlp_backward_weight", "storm_gnn_agg_backward",
           "storm_gnn_node_backward", "storm_gnn_mse", "storm_gnn_adam", "storm_gnn_sumsq",
           "storm_gnn_kernel_launches")

_bound = False


def lib():
    global _bound
    L = fvt.lib()
    if not _bound:
        L.storm_gnn_grad_size.argtypes = [C.c_int32, C.c_int32]
        L.storm_gnn_grad_size.restype = C.c_int32
        L.storm_gnn_weight_scratch_bytes.argtypes = [C.c_int32, C.c_int32]
        L.storm_gnn_weight_scratch_bytes.restype = C.c_size_t
        L.storm_gnn_mlp_forward.argtypes = [C.POINTER(MlpFwd), _vp, _vp]
        L.storm_gnn_mlp_backward_data.argtypes = [C.POINTER(MlpBwdData), _vp, _vp]
        L.storm_gnn_mlp_backward_weight.argtypes = [C.POINTER(MlpBwdWeight), _vp, _vp, C.c_size_t, _vp, _vp]
        L.storm_gnn_agg_backward.argtypes = [_vp, _vp, _vp, C.c_int32, _vp, _vp]
        L.storm_gnn_node_backward.argtypes = [_vp, _vp, _vp, _vp, C.c_int32, _vp, _vp]
        L.storm_gnn_mse.argtypes = [_vp, C.c_int32, _vp, _vp, C.c_int32, C.c_int32, C.c_float, _vp, _vp, _vp]
        L.storm_gnn_adam.argtypes = [_vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_float, C.c_float, C.c_float,
                                     C.c_float, C.c_int32, C.c_float, C.c_float, _vp]
        L.storm_gnn_sumsq.argtypes = [_vp, C.c_int32, _vp, _vp]
        L.storm_gnn_kernel_launches.restype = C.c_int64
        _bound = True
    return L


def _chk(rc):
    if rc != 0:
        raise fvt.StormError(rc, fvt.lib().storm_fvt_last_error().decode())


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def kernel_launches() -> int:
    return int(lib().storm_gnn_kernel_launches())


# ---- parameters ---------------------------------------------------------------------

@dataclasses.dataclass
class MlpSpec:
    name: str
    k_in: int
    n_out: int
    offset: int = 0  # into the flat parameter vector

    @property
    def size(self) -> int:
        return HID * self.k_in + HID + self.n_out * HID + self.n_out

    def views(self, flat):
        o = self.offset
        w1 = flat[o:o + HID * self.k_in]
        b1 = flat[o + HID * self.k_in:o + HID * self.k_in + HID]
        o2 = o + HID * self.k_in + HID
        w2 = flat[o2:o2 + self.n_out * HID]
        b2 = flat[o2 + self.n_out * HID:o2 + self.n_out * HID + self.n_out]
        return w1, b1, w2, b2


def network_specs(n_layers: int = N_LAYERS):
    specs = [MlpSpec("enc_node", IN_NODE, HID), MlpSpec("enc_edge", IN_EDGE, HID)]
    for l in range(n_layers):
        specs.append(MlpSpec(f"edge{l}", 3 * HID, HID))
        specs.append(MlpSpec(f"node{l}", 2 * HID, HID))
    specs.append(MlpSpec("dec", HID, N_OUT_PAD))
    off = 0
    for s in specs:
        s.offset = off
        off += (s.size + 63) // 64 * 64
    return specs, off


def init_params(specs, total, seed: int = 0, out_scale: float = 1.0) -> np.ndarray:
    """He-uniform first layers, scaled-down second layers (residual branches start
    small), zero biases.  Decoder output rows beyond the targets are zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(total, dtype=np.float32)
    for s in specs:
        w1, b1, w2, b2 = s.views(p)
        lim1 = math.sqrt(6.0 / s.k_in)
        w1[:] = rng.uniform(-lim1, lim1, size=w1.shape)
        lim2 = math.sqrt(6.0 / HID) * (0.25 if s.name.startswith(("edge", "node")) else 1.0) * (
            0.1 * out_scale if s.name == "dec" else 1.0)
        w2v = rng.uniform(-lim2, lim2, size=(s.n_out, HID)).astype(np.float32)
        if s.name == "dec":
            w2v[N_TARGET:] = 0.0
        w2[:] = w2v.reshape(-1)
    return p


# ---- graph ------------------------------------------------------------------------------

@dataclasses.dataclass
class Graph:
    """Disjoint union of cell-dual graphs, cells padded to Tp = 128 * k."""
    T: int
    Tp: int
    nbr: np.ndarray        # [3*Tp] int32 source cell of edge row k*Tp + c, or -1
    dst: np.ndarray        # [3*Tp] int32 c, or -1 for padding cells
    rev: np.ndarray        # [3*Tp] int32 edge row where cell c is the source (k-th such), or -1
    x_node: np.ndarray     # [Tp, 64] float32
    x_edge: np.ndarray     # [3*Tp, 64] float32
    cell_off: np.ndarray   # [G+1] offsets of the member graphs


def build_graph(t2t3_list, xnode_list, xedge_list) -> Graph:
    """t2t3_list: per member [3, T] neighbour ids (0-based, -1 none) in the member's
    cell order; features per member [T, 64] and [3, T, 64]."""
    Ts = [int(t.shape[1]) for t in t2t3_list]
    T = int(sum(Ts))
    Tp = (T + 127) // 128 * 128
    nbr = -np.ones((3, Tp), dtype=np.int32)
    off = np.concatenate([[0], np.cumsum(Ts)]).astype(np.int64)
    xn = np.zeros((Tp, IN_NODE), dtype=np.float32)
    xe = np.zeros((3, Tp, IN_EDGE), dtype=np.float32)
    for g, t in enumerate(t2t3_list):
        o = off[g]
        n = Ts[g]
        tt = np.asarray(t, dtype=np.int64)
        nbr[:, o:o + n] = np.where(tt >= 0, tt + o, -1)
        xn[o:o + n] = xnode_list[g]
        xe[:, o:o + n] = xedge_list[g]
    dst = np.tile(np.arange(Tp, dtype=np.int32), 3)
    dst[np.tile(np.arange(Tp) >= T, 3)] = -1
    flat = nbr.reshape(-1)
    rev = -np.ones((3, Tp), dtype=np.int32)
    cnt = np.zeros(Tp, dtype=np.int32)
    for e in np.nonzero(flat >= 0)[0]:  # edge row e carries src -> dst; rows in increasing order
        s = flat[e]
        if cnt[s] >= 3:
            raise ValueError("a cell is the source of more than three edge rows")
        rev[cnt[s], s] = e
        cnt[s] += 1
    x_edge = xe.reshape(3 * Tp, IN_EDGE)
    return Graph(T, Tp, flat.copy(), dst, rev.reshape(-1), xn, x_edge, off)


def build_graph_fast(t2t3_list, xnode_list, xedge_list) -> Graph:
    """Vectorised :func:`build_graph` (same result)."""
    Ts = [int(t.shape[1]) for t in t2t3_list]
    T = int(sum(Ts))
    Tp = (T + 127) // 128 * 128
    off = np.concatenate([[0], np.cumsum(Ts)]).astype(np.int64)
    nbr = -np.ones((3, Tp), dtype=np.int64)
    xn = np.zeros((Tp, IN_NODE), dtype=np.float32)
    xe = np.zeros((3, Tp, IN_EDGE), dtype=np.float32)
    for g, t in enumerate(t2t3_list):
        o, n = off[g], Ts[g]
        tt = np.asarray(t, dtype=np.int64)
        nbr[:, o:o + n] = np.where(tt >= 0, tt + o, -1)
        xn[o:o + n] = xnode_list[g]
        xe[:, o:o + n] = xedge_list[g]
    flat = nbr.reshape(-1)
    e = np.nonzero(flat >= 0)[0]
    s = flat[e]
    order = np.lexsort((e, s))  # by source, then edge row
    e, s = e[order], s[order]
    first = np.searchsorted(s, s, side="left")
    k = np.arange(len(s)) - first
    if len(k) and k.max() >= 3:
        raise ValueError("a cell is the source of more than three edge rows")
    rev = -np.ones((3, Tp), dtype=np.int64)
    rev[k, s] = e
    dst = np.tile(np.arange(Tp, dtype=np.int64), 3)
    dst[np.tile(np.arange(Tp) >= T, 3)] = -1
    return Graph(T, Tp, flat.astype(np.int32), dst.astype(np.int32), rev.reshape(-1).astype(np.int32), xn,
                 xe.reshape(3 * Tp, IN_EDGE), off)


# ---- device network -----------------------------------------------------------------------

class DeviceGraph:
    """A Graph resident on the GPU (bf16 features, int32 tables)."""

    def __init__(self, g: Graph, device):
        import torch
        self.g = g
        self.T, self.Tp = g.T, g.Tp
        self.nbr = torch.from_numpy(g.nbr).to(device)
        self.dst = torch.from_numpy(g.dst).to(device)
        self.rev = torch.from_numpy(g.rev).to(device)
        self.x_node = torch.from_numpy(g.x_node).to(device=device, dtype=torch.bfloat16)
        self.x_edge = torch.from_numpy(g.x_edge).to(device=device, dtype=torch.bfloat16)


class WarmStartNet:
    """The network's parameters and optimiser state on one GPU, with forward,
    backward and Adam steps built from the library's kernels."""

    def __init__(self, device="cuda:0", n_layers: int = N_LAYERS, seed: int = 0, params: np.ndarray | None = None):
        import torch
        self.device = torch.device(device)
        self.n_layers = n_layers
        self.specs, self.total = network_specs(n_layers)
        self.by_name = {s.name: s for s in self.specs}
        p = init_params(self.specs, self.total, seed) if params is None else np.asarray(params, np.float32)
        self.w = torch.from_numpy(p.copy()).to(self.device)
        self.wb = self.w.to(torch.bfloat16)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.grad = torch.zeros_like(self.w)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.step_count = 0
        self._scratch = None
        self._parts = torch.zeros(148, dtype=torch.float32, device=self.device)
        self.norm_stats = None  # feature/target scaling, set by the trainer

    # -- helpers
    def params_numpy(self) -> np.ndarray:
        return self.w.cpu().numpy()

    def _wv(self, name):
        s = self.by_name[name]
        o = s.offset
        w1 = self.wb[o:]
        b1 = self.w[o + HID * s.k_in:]
        o2 = o + HID * s.k_in + HID
        w2 = self.wb[o2:]
        b2 = self.w[o2 + s.n_out * HID:]
        return s, w1, b1, w2, b2

    def _check_err(self):
        e = int(self.err.item())
        if e:
            raise fvt.StormError(-5, f"warm-start kernel reported device status {e}")

    def _fwd(self, name, rows, segs, out, res=None, out_f32=None, a1_save=None):
        s, w1, b1, w2, b2 = self._wv(name)
        a = MlpFwd()
        a.rows, a.nseg, a.k_in, a.n_out = rows, len(segs), s.k_in, s.n_out
        for i, sg in enumerate(segs):
            a.seg[i] = sg
        a.w1, a.b1, a.w2, a.b2 = _ptr(w1), _ptr(b1), _ptr(w2), _ptr(b2)
        a.res, a.out, a.out_f32, a.a1_save = _ptr(res), _ptr(out), _ptr(out_f32), _ptr(a1_save)
        _chk(lib().storm_gnn_mlp_forward(C.byref(a), _ptr(self.err), _stream()))

    def _bwd_data(self, name, rows, widths, dy, a1, dz1, dseg, dadd):
        s, w1, b1, w2, b2 = self._wv(name)
        a = MlpBwdData()
        a.rows, a.nseg, a.k_in, a.n_out = rows, len(widths), s.k_in, s.n_out
        for i, w in enumerate(widths):
            a.seg_width[i] = w
            a.dseg[i] = _ptr(dseg[i]) if dseg[i] is not None else None
            a.dseg_add[i] = _ptr(dadd[i]) if dadd[i] is not None else None
        a.dy, a.a1, a.w1, a.w2, a.dz1_save = _ptr(dy), _ptr(a1), _ptr(w1), _ptr(w2), _ptr(dz1)
        _chk(lib().storm_gnn_mlp_backward_data(C.byref(a), _ptr(self.err), _stream()))

    def _bwd_weight(self, name, rows, segs, dy, a1, dz1):
        import torch
        s = self.by_name[name]
        a = MlpBwdWeight()
        a.rows, a.nseg, a.k_in, a.n_out = rows, len(segs), s.k_in, s.n_out
        for i, sg in enumerate(segs):
            a.seg[i] = sg
        a.dy, a.a1, a.dz1 = _ptr(dy), _ptr(a1), _ptr(dz1)
        need = int(lib().storm_gnn_weight_scratch_bytes(s.k_in, s.n_out))
        if self._scratch is None or self._scratch.numel() * 4 < need:
            self._scratch = torch.empty((need + 3) // 4, dtype=torch.float32, device=self.device)
        g = self.grad[s.offset:]
        _chk(lib().storm_gnn_mlp_backward_weight(C.byref(a), _ptr(g), _ptr(self._scratch), need, _ptr(self.err),
                                                 _stream()))

    @staticmethod
    def _seg(src, width=HID, idx=None, agg=False, stride=0, nbr=None) -> Seg:
        s = Seg()
        s.src = _ptr(src)
        s.idx = _ptr(idx) if idx is not None else None
        s.width = width
        s.agg = 1 if agg else 0
        s.agg_stride = stride
        s.nbr = _ptr(nbr) if nbr is not None else None
        return s

    # -- forward
    def forward(self, dg: DeviceGraph, save: bool = False):
        """Returns the decoder output (fp32 [Tp, 64]); with save=True keeps the
        activations for :meth:`backward`."""
        import torch
        Tp, E = dg.Tp, 3 * dg.Tp
        bf = torch.bfloat16
        dev = self.device
        L = self.n_layers
        hs = [torch.empty((Tp, HID), dtype=bf, device=dev) for _ in range(L + 1 if save else 2)]
        es = [torch.empty((E, HID), dtype=bf, device=dev) for _ in range(L + 1 if save else 2)]
        acts = {}

        def a1buf(name, rows):
            if not save:
                return None
            t = torch.empty((rows, HID), dtype=bf, device=dev)
            acts[name] = t
            return t

        self._fwd("enc_node", Tp, [self._seg(dg.x_node, IN_NODE)], hs[0], a1_save=a1buf("enc_node", Tp))
        self._fwd("enc_edge", E, [self._seg(dg.x_edge, IN_EDGE)], es[0], a1_save=a1buf("enc_edge", E))
        for l in range(L):
            hi, ho = (l, l + 1) if save else (l % 2, (l + 1) % 2)
            h, e = hs[hi], es[hi]
            self._fwd(f"edge{l}", E, [self._seg(e), self._seg(h, idx=dg.nbr), self._seg(h, idx=dg.dst)], es[ho],
                      res=e, a1_save=a1buf(f"edge{l}", E))
            self._fwd(f"node{l}", Tp, [self._seg(h), self._seg(es[ho], agg=True, stride=Tp, nbr=dg.nbr)], hs[ho],
                      res=h, a1_save=a1buf(f"node{l}", Tp))
        hl = hs[L] if save else hs[L % 2]
        y = torch.empty((Tp, N_OUT_PAD), dtype=bf, device=dev)
        y32 = torch.empty((Tp, N_OUT_PAD), dtype=torch.float32, device=dev)
        self._fwd("dec", Tp, [self._seg(hl)], y, out_f32=y32, a1_save=a1buf("dec", Tp))
        if save:
            self._saved = (dg, hs, es, acts)
        return y32

    # -- loss
    def mse(self, y32, target, wmask, norm):
        """Loss sum over the first 3 outputs (weights wmask), and dy."""
        import torch
        Tp = y32.shape[0]
        dy = torch.empty_like(y32)
        _chk(lib().storm_gnn_mse(_ptr(y32), N_OUT_PAD, _ptr(target), _ptr(wmask), Tp, N_TARGET, float(norm),
                                 _ptr(dy), _ptr(self._parts), _stream()))
        return dy, self._parts

    # -- backward (after forward(save=True)); fills self.grad
    def backward(self, dy_dec):
        import torch
        dg, hs, es, acts = self._saved
        Tp, E = dg.Tp, 3 * dg.Tp
        dev = self.device
        f32 = torch.float32
        L = self.n_layers
        dz_n = torch.empty((Tp, HID), dtype=torch.bfloat16, device=dev)
        dz_e = torch.empty((E, HID), dtype=torch.bfloat16, device=dev)
        dh = torch.empty((Tp, HID), dtype=f32, device=dev)
        dh_next = torch.empty_like(dh)
        dagg = torch.empty_like(dh)
        de = torch.zeros((E, HID), dtype=f32, device=dev)
        de_tot = torch.empty_like(de)
        de_next = torch.empty_like(de)
        dsrc = torch.empty_like(de)
        ddst = torch.empty_like(de)
        # decoder
        self._bwd_data("dec", Tp, [HID], dy_dec, acts["dec"], dz_n, [dh], [None])
        self._bwd_weight("dec", Tp, [self._seg(hs[L])], dy_dec, acts["dec"], dz_n)
        first = True
        for l in reversed(range(L)):
            h, e, e1 = hs[l], es[l], es[l + 1]
            # node update h_{l+1} = h_l + MLP_n([h_l, agg(e_{l+1})])
            self._bwd_data(f"node{l}", Tp, [HID, HID], dh, acts[f"node{l}"], dz_n, [dh_next, dagg], [dh, None])
            self._bwd_weight(f"node{l}", Tp, [self._seg(h), self._seg(e1, agg=True, stride=Tp, nbr=dg.nbr)], dh,
                             acts[f"node{l}"], dz_n)
            _chk(lib().storm_gnn_agg_backward(None if first else _ptr(de), _ptr(dagg), _ptr(dg.nbr), Tp,
                                              _ptr(de_tot), _stream()))
            first = False
            # edge update e_{l+1} = e_l + MLP_e([e_l, h_l[src], h_l[dst]])
            self._bwd_data(f"edge{l}", E, [HID, HID, HID], de_tot, acts[f"edge{l}"], dz_e,
                           [de_next, dsrc, ddst], [de_tot, None, None])
            self._bwd_weight(f"edge{l}", E, [self._seg(e), self._seg(h, idx=dg.nbr), self._seg(h, idx=dg.dst)],
                             de_tot, acts[f"edge{l}"], dz_e)
            _chk(lib().storm_gnn_node_backward(_ptr(dh_next), _ptr(ddst), _ptr(dsrc), _ptr(dg.rev), Tp, _ptr(dh),
                                               _stream()))
            de, de_next = de_next, de
        # encoders (weights only)
        self._bwd_data("enc_node", Tp, [IN_NODE], dh, acts["enc_node"], dz_n, [None], [None])
        self._bwd_weight("enc_node", Tp, [self._seg(dg.x_node, IN_NODE)], dh, acts["enc_node"], dz_n)
        self._bwd_data("enc_edge", E, [IN_EDGE], de, acts["enc_edge"], dz_e, [None], [None])
        self._bwd_weight("enc_edge", E, [self._seg(dg.x_edge, IN_EDGE)], de, acts["enc_edge"], dz_e)
        self._saved = None

    def grad_norm(self) -> float:
        _chk(lib().storm_gnn_sumsq(_ptr(self.grad), self.total, _ptr(self._parts), _stream()))
        return float(math.sqrt(float(self._parts.cpu().numpy().astype(np.float64).sum())))

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, grad_scale=1.0):
        self.step_count += 1
        _chk(lib().storm_gnn_adam(_ptr(self.w), _ptr(self.m), _ptr(self.v), _ptr(self.grad), _ptr(self.wb),
                                  self.total, float(lr), float(beta1), float(beta2), float(eps), self.step_count,
                                  float(weight_decay), float(grad_scale), _stream()))


def neighbour_table(mesh_np: dict) -> np.ndarray:
    """[3, T] 0-based neighbour across each local face of every cell (-1: boundary),
    from the prepared mesh's t2t3 table (Fortran t2t3(3, n_elems), the cell itself
    where the face has no neighbour; dataprepFVT.f90)."""
    T = int(mesh_np["n_elems"])
    t = mesh_np["t2t3"].reshape(T, 3).T.astype(np.int64) - 1
    own = np.arange(T)[None, :]
    return np.where((t >= 0) & (t != own), t, -1).astype(np.int32)
