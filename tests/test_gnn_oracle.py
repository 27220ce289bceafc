"""CPU checks of the warm-start network's oracle and graph builder (no GPU)."""
import numpy as np

from oracle.gnn_oracle import GnnOracle, to_bf16
from storm_b200 import gnn


def _ring_graph(T=40, seed=0):
    """Cells on a strip: each cell's neighbours are its predecessor and successor
    (face 2 has none), features random."""
    rng = np.random.default_rng(seed)
    t = -np.ones((3, T), dtype=np.int32)
    t[0, 1:] = np.arange(T - 1)
    t[1, :-1] = np.arange(1, T)
    xn = rng.normal(size=(T, gnn.IN_NODE)).astype(np.float32)
    xe = rng.normal(size=(3, T, gnn.IN_EDGE)).astype(np.float32)
    return t, xn, xe


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.0e38])
    r = to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5 and r[4] == 0.0


def test_graph_builders_agree():
    parts = [_ring_graph(37, 1), _ring_graph(100, 2)]
    a = gnn.build_graph([p[0] for p in parts], [p[1] for p in parts], [p[2] for p in parts])
    b = gnn.build_graph_fast([p[0] for p in parts], [p[1] for p in parts], [p[2] for p in parts])
    assert a.Tp == b.Tp == 256 and a.T == b.T == 137
    for f in ("nbr", "dst", "rev"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    # rev lists, for every cell, exactly the edge rows whose source it is
    for c in range(a.T):
        rows = sorted(int(e) for e in a.rev.reshape(3, -1)[:, c] if e >= 0)
        assert rows == sorted(np.nonzero(a.nbr == c)[0].tolist())
    assert (a.nbr[a.nbr >= 0] < a.T).all()


def test_oracle_gradient_matches_finite_differences():
    """The oracle's backward pass (float64, no rounding) against central differences
    of its own loss, along random directions, on a 2-layer network."""
    t, xn, xe = _ring_graph(30, 3)
    g = gnn.build_graph_fast([t], [xn], [xe])
    specs, total = gnn.network_specs(2)
    rng = np.random.default_rng(5)
    p = gnn.init_params(specs, total, seed=1).astype(np.float64)
    for s in specs:
        w1, b1, w2, b2 = s.views(p)
        b1[:] = rng.normal(scale=0.1, size=b1.shape)
        b2[:] = rng.normal(scale=0.1, size=b2.shape)
        if s.name == "dec":
            w2[:] = rng.normal(scale=0.05, size=w2.shape)
    target = rng.normal(size=(g.Tp, 3))
    w = (np.arange(g.Tp) < g.T).astype(np.float64)

    def loss_at(q):
        o = GnnOracle(specs, q, 2, bf16=False)
        y, _ = o.forward(g)
        return o.loss(y, target, w, 3.0 * g.T)[0]

    o = GnnOracle(specs, p, 2, bf16=False)
    y, tape = o.forward(g)
    _, dy = o.loss(y, target, w, 3.0 * g.T)
    grad = o.backward(g, tape, dy)
    for k in range(3):
        d = rng.normal(size=p.shape)
        eps = 1e-6
        fd = (loss_at(p + eps * d) - loss_at(p - eps * d)) / (2 * eps)
        an = float(grad @ d)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
