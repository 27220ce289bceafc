"""CPU oracle of the warm-start network (numpy): forward and backward of the same
encode / process / decode message-passing network the GPU kernels compute
(storm_b200/gnn.py, storm_b200/csrc/gnn_kernels.cu).

Test infrastructure only: the tests use it to check the GPU forward pass and the
GPU gradients.  It has no counterpart in the reference (SToRM has no learned
component).

With ``bf16=True`` the oracle rounds to bfloat16 at the points where the kernels
store bf16 (inputs, weights, hidden activations, layer outputs, aggregated messages,
the staged dy and dz1) and computes everything else in float64, so the remaining
difference to the GPU is the fp32 accumulation order of the tensor cores.  The
backward pass treats each rounding as the identity (as the kernels do).  With
``bf16=False`` it is the exact float64 network, whose gradient the finite-difference
test pins.
"""
from __future__ import annotations

import numpy as np

HID = 128


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round float values to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


class GnnOracle:
    def __init__(self, specs, params: np.ndarray, n_layers: int, bf16: bool = True):
        self.specs = {s.name: s for s in specs}
        self.p = np.asarray(params, dtype=np.float64)
        self.L = n_layers
        self.bf = bf16

    def r(self, x):
        return to_bf16(x) if self.bf else np.asarray(x, dtype=np.float64)

    def weights(self, name):
        s = self.specs[name]
        o = s.offset
        w1 = self.p[o:o + HID * s.k_in].reshape(HID, s.k_in)
        b1 = self.p[o + HID * s.k_in:o + HID * s.k_in + HID]
        o2 = o + HID * s.k_in + HID
        w2 = self.p[o2:o2 + s.n_out * HID].reshape(s.n_out, HID)
        b2 = self.p[o2 + s.n_out * HID:o2 + s.n_out * HID + s.n_out]
        return s, self.r(w1), b1, self.r(w2), b2

    def mlp(self, name, A, res=None):
        """A: [rows, k_in] (already rounded).  Returns (out_bf16, out_f, a1)."""
        s, w1, b1, w2, b2 = self.weights(name)
        z1 = A @ w1.T + b1
        a1 = self.r(np.maximum(z1, 0.0))
        y = a1 @ w2.T
        if res is not None:
            y = y + res
        y = y + b2
        return self.r(y), y, a1

    @staticmethod
    def gather(x, idx):
        out = np.zeros((len(idx), x.shape[1]))
        m = idx >= 0
        out[m] = x[idx[m]]
        return out

    def agg(self, e, nbr, Tp):
        e3 = e.reshape(3, Tp, -1)
        m = (nbr.reshape(3, Tp) >= 0)[:, :, None]
        return self.r((e3 * m).sum(axis=0))

    def forward(self, g):
        """g: storm_b200.gnn.Graph.  Returns the decoder output (fp, [Tp, 64]) and a tape."""
        Tp = g.Tp
        xn = self.r(g.x_node)
        xe = self.r(g.x_edge)
        tape = {"xn": xn, "xe": xe}
        h, _, tape["a_enc_node"] = self.mlp("enc_node", xn)
        e, _, tape["a_enc_edge"] = self.mlp("enc_edge", xe)
        hs, es = [h], [e]
        for l in range(self.L):
            A = np.concatenate([e, self.gather(h, g.nbr), self.gather(h, g.dst)], axis=1)
            e, _, tape[f"a_edge{l}"] = self.mlp(f"edge{l}", A, res=e)
            tape[f"A_edge{l}"] = A
            B = np.concatenate([h, self.agg(e, g.nbr, Tp)], axis=1)
            h, _, tape[f"a_node{l}"] = self.mlp(f"node{l}", B, res=h)
            tape[f"A_node{l}"] = B
            hs.append(h)
            es.append(e)
        _, y, tape["a_dec"] = self.mlp("dec", h)
        tape["hs"], tape["es"] = hs, es
        return y, tape

    def mlp_backward(self, name, A, a1, dy, grads):
        """Returns dA; accumulates the weight gradient of `name` into grads."""
        s, w1, b1, w2, b2 = self.weights(name)
        dyr = self.r(dy)
        dz1 = self.r((dyr @ w2) * (a1 > 0))
        gw1 = dz1.T @ A
        gb1 = dz1.sum(axis=0)
        gw2 = dyr.T @ a1
        gb2 = dy.sum(axis=0)
        o = s.offset
        grads[o:o + HID * s.k_in] += gw1.reshape(-1)
        grads[o + HID * s.k_in:o + HID * s.k_in + HID] += gb1
        o2 = o + HID * s.k_in + HID
        grads[o2:o2 + s.n_out * HID] += gw2.reshape(-1)
        grads[o2 + s.n_out * HID:o2 + s.n_out * HID + s.n_out] += gb2
        return dz1 @ w1

    def backward(self, g, tape, dy_dec):
        Tp, E = g.Tp, 3 * g.Tp
        grads = np.zeros_like(self.p)
        hs, es = tape["hs"], tape["es"]
        L = self.L
        dh = self.mlp_backward("dec", hs[L], tape["a_dec"], dy_dec, grads)
        de = np.zeros((E, HID))
        m = (g.nbr.reshape(3, Tp) >= 0)[:, :, None]
        for l in reversed(range(L)):
            dB = self.mlp_backward(f"node{l}", tape[f"A_node{l}"], tape[f"a_node{l}"], dh, grads)
            dh_next = dh + dB[:, :HID]
            dagg = dB[:, HID:]
            de_tot = de + (m * dagg[None]).reshape(E, HID)
            dA = self.mlp_backward(f"edge{l}", tape[f"A_edge{l}"], tape[f"a_edge{l}"], de_tot, grads)
            de = de_tot + dA[:, :HID]
            dsrc, ddst = dA[:, HID:2 * HID], dA[:, 2 * HID:]
            dh = dh_next.copy()
            dh += ddst.reshape(3, Tp, HID).sum(axis=0)
            valid = g.nbr >= 0
            np.add.at(dh, g.nbr[valid], dsrc[valid])
        self.mlp_backward("enc_node", tape["xn"], tape["a_enc_node"], dh, grads)
        self.mlp_backward("enc_edge", tape["xe"], tape["a_enc_edge"], de, grads)
        return grads

    def loss(self, y, target, w, norm):
        d = y[:, :3] - target
        loss = float((w[:, None] * d * d).sum() / norm)
        dy = np.zeros_like(y)
        dy[:, :3] = 2.0 * w[:, None] * d / norm
        return loss, dy
