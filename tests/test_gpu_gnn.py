"""Warm-start network kernels (tcgen05 MLPs, gathers, aggregation, Adam) against the
numpy oracle (oracle/gnn_oracle.py) that rounds to bf16 at the same points.

Tolerances: the remaining difference is the fp32 accumulation order inside the
tensor cores, which flips single bf16 roundings (relative 2^-8) that then propagate;
single MLPs must agree to 1e-2 relative L2, the 8-layer network's output to 3e-2
and every parameter block's gradient to 5e-2 relative L2 with cosine >= 0.998."""
import numpy as np
import pytest

from oracle.gnn_oracle import GnnOracle, to_bf16
from storm_b200 import gnn, scenarios

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _cos(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def torch_cuda(storm_lib):
    import torch
    return torch


def _tiny_graph(seed=0, n_members=2):
    """A union of small channel meshes with random features."""
    from storm_b200 import fvt
    rng = np.random.default_rng(seed)
    nb, xn, xe = [], [], []
    for m in range(n_members):
        sc = scenarios.channel(nx=6 + 2 * m, ny=4, seed=seed + m)
        pm = fvt.build_mesh(sc.problem)
        mn = pm.numpy()
        nb.append(gnn.neighbour_table(mn))
        T = mn["n_elems"]
        xn.append(rng.normal(size=(T, gnn.IN_NODE)).astype(np.float32))
        xe.append(rng.normal(size=(3, T, gnn.IN_EDGE)).astype(np.float32))
    return gnn.build_graph_fast(nb, xn, xe)


def test_mlp_forward_segments(torch_cuda):
    torch = torch_cuda
    net = gnn.WarmStartNet(seed=3)
    rng = np.random.default_rng(1)
    rows = 384
    e = to_bf16(rng.normal(size=(rows, 128)))
    h = to_bf16(rng.normal(size=(rows // 3, 128)))
    idx = rng.integers(-1, rows // 3, size=rows).astype(np.int32)
    dev = net.device
    e_t = torch.tensor(e, dtype=torch.bfloat16, device=dev)
    h_t = torch.tensor(h, dtype=torch.bfloat16, device=dev)
    idx_t = torch.tensor(idx, device=dev)
    out = torch.empty((rows, 128), dtype=torch.bfloat16, device=dev)
    a1 = torch.empty((rows, 128), dtype=torch.bfloat16, device=dev)
    net._fwd("edge0", rows, [net._seg(e_t), net._seg(h_t, idx=idx_t), net._seg(e_t)], out, res=e_t, a1_save=a1)
    torch.cuda.synchronize()
    net._check_err()
    orc = GnnOracle(net.specs, net.params_numpy(), net.n_layers)
    A = np.concatenate([e, GnnOracle.gather(h, idx), e], axis=1)
    ref, _, ref_a1 = orc.mlp("edge0", A, res=e)
    assert _rel(a1.float().cpu().numpy(), ref_a1) < 1e-2
    assert _rel(out.float().cpu().numpy(), ref) < 1e-2
    # 64-wide input, 64-wide output (decoder shape) with fp32 copy
    x = to_bf16(rng.normal(size=(256, 128)))
    x_t = torch.tensor(x, dtype=torch.bfloat16, device=dev)
    y = torch.empty((256, 64), dtype=torch.bfloat16, device=dev)
    y32 = torch.empty((256, 64), dtype=torch.float32, device=dev)
    net._fwd("dec", 256, [net._seg(x_t)], y, out_f32=y32)
    torch.cuda.synchronize()
    _, ref32, _ = orc.mlp("dec", x)
    assert _rel(y32.cpu().numpy(), ref32) < 1e-2
    xi = to_bf16(rng.normal(size=(256, 64)))
    xi_t = torch.tensor(xi, dtype=torch.bfloat16, device=dev)
    z = torch.empty((256, 128), dtype=torch.bfloat16, device=dev)
    net._fwd("enc_node", 256, [net._seg(xi_t, 64)], z)
    torch.cuda.synchronize()
    refz, _, _ = orc.mlp("enc_node", xi)
    assert _rel(z.float().cpu().numpy(), refz) < 1e-2


def test_aggregation_segment(torch_cuda):
    torch = torch_cuda
    g = _tiny_graph(seed=5)
    net = gnn.WarmStartNet(seed=4)
    dg = gnn.DeviceGraph(g, net.device)
    rng = np.random.default_rng(2)
    e = to_bf16(rng.normal(size=(3 * g.Tp, 128)))
    h = to_bf16(rng.normal(size=(g.Tp, 128)))
    e_t = torch.tensor(e, dtype=torch.bfloat16, device=net.device)
    h_t = torch.tensor(h, dtype=torch.bfloat16, device=net.device)
    out = torch.empty((g.Tp, 128), dtype=torch.bfloat16, device=net.device)
    net._fwd("node0", g.Tp, [net._seg(h_t), net._seg(e_t, agg=True, stride=g.Tp, nbr=dg.nbr)], out, res=h_t)
    torch.cuda.synchronize()
    orc = GnnOracle(net.specs, net.params_numpy(), net.n_layers)
    B = np.concatenate([h, orc.agg(e, g.nbr, g.Tp)], axis=1)
    ref, _, _ = orc.mlp("node0", B, res=h)
    assert _rel(out.float().cpu().numpy(), ref) < 1e-2


def test_mlp_backward(torch_cuda):
    torch = torch_cuda
    net = gnn.WarmStartNet(seed=5)
    rng = np.random.default_rng(3)
    rows = 512
    dev = net.device
    x = [to_bf16(rng.normal(size=(rows, 128))) for _ in range(2)]
    xt = [torch.tensor(a, dtype=torch.bfloat16, device=dev) for a in x]
    out = torch.empty((rows, 128), dtype=torch.bfloat16, device=dev)
    a1 = torch.empty((rows, 128), dtype=torch.bfloat16, device=dev)
    net._fwd("node1", rows, [net._seg(xt[0]), net._seg(xt[1])], out, a1_save=a1)
    dy = rng.normal(size=(rows, 128)).astype(np.float32)
    add = rng.normal(size=(rows, 128)).astype(np.float32)
    dy_t = torch.tensor(dy, device=dev)
    add_t = torch.tensor(add, device=dev)
    dz = torch.empty((rows, 128), dtype=torch.bfloat16, device=dev)
    d0 = torch.empty((rows, 128), dtype=torch.float32, device=dev)
    d1 = torch.empty((rows, 128), dtype=torch.float32, device=dev)
    net._bwd_data("node1", rows, [128, 128], dy_t, a1, dz, [d0, d1], [add_t, None])
    net.grad.zero_()
    net._bwd_weight("node1", rows, [net._seg(xt[0]), net._seg(xt[1])], dy_t, a1, dz)
    torch.cuda.synchronize()
    net._check_err()
    orc = GnnOracle(net.specs, net.params_numpy(), net.n_layers)
    A = np.concatenate(x, axis=1)
    a1_np = a1.float().cpu().numpy()  # the GPU's own activation (isolates the backward)
    grads = np.zeros(net.total)
    dA = orc.mlp_backward("node1", A, a1_np, dy.astype(np.float64), grads)
    assert _rel(d0.cpu().numpy(), dA[:, :128] + add) < 1e-2
    assert _rel(d1.cpu().numpy(), dA[:, 128:]) < 1e-2
    s = net.by_name["node1"]
    g_gpu = net.grad.cpu().numpy()[s.offset:s.offset + s.size]
    g_ref = grads[s.offset:s.offset + s.size]
    for lo, hi in ((0, 128 * 256), (128 * 256, 128 * 257), (128 * 257, 128 * 257 + 128 * 128),
                   (128 * 257 + 128 * 128, s.size)):
        assert _rel(g_gpu[lo:hi], g_ref[lo:hi]) < 1e-2, (lo, hi)


def test_network_forward_and_gradients(torch_cuda):
    torch = torch_cuda
    g = _tiny_graph(seed=7, n_members=3)
    net = gnn.WarmStartNet(seed=11)
    # non-zero biases so that every bias path is exercised
    p = net.params_numpy()
    rng = np.random.default_rng(9)
    for s in net.specs:
        w1, b1, w2, b2 = s.views(p)
        b1[:] = rng.normal(scale=0.1, size=b1.shape)
        b2[:] = rng.normal(scale=0.1, size=b2.shape)
    net = gnn.WarmStartNet(params=p)
    dg = gnn.DeviceGraph(g, net.device)
    y32 = net.forward(dg, save=True)
    target = rng.normal(size=(g.Tp, 3)).astype(np.float32)
    w = (np.arange(g.Tp) < g.T).astype(np.float32)
    norm = 3.0 * g.T
    t_t = torch.tensor(target, device=net.device)
    w_t = torch.tensor(w, device=net.device)
    dy, parts = net.mse(y32, t_t, w_t, norm)
    loss_gpu = float(parts.cpu().numpy().astype(np.float64).sum())
    net.grad.zero_()
    net.backward(dy)
    torch.cuda.synchronize()
    net._check_err()
    orc = GnnOracle(net.specs, p, net.n_layers)
    y_ref, tape = orc.forward(g)
    assert _rel(y32.cpu().numpy()[:g.T, :3], y_ref[:g.T, :3]) < 3e-2
    loss_ref, dy_ref = orc.loss(y_ref, target.astype(np.float64), w.astype(np.float64), norm)
    assert abs(loss_gpu - loss_ref) < 3e-2 * abs(loss_ref)
    grads = orc.backward(g, tape, dy_ref)
    g_gpu = net.grad.cpu().numpy().astype(np.float64)
    for s in net.specs:
        a = g_gpu[s.offset:s.offset + s.size]
        b = grads[s.offset:s.offset + s.size]
        assert _rel(a, b) < 5e-2, s.name
        assert _cos(a, b) > 0.998, s.name


def test_adam_training_reduces_loss(torch_cuda):
    torch = torch_cuda
    g = _tiny_graph(seed=13, n_members=2)
    net = gnn.WarmStartNet(seed=2)
    dg = gnn.DeviceGraph(g, net.device)
    rng = np.random.default_rng(4)
    target = np.tanh(g.x_node[:, :3]).astype(np.float32)
    w = (np.arange(g.Tp) < g.T).astype(np.float32)
    t_t = torch.tensor(target, device=net.device)
    w_t = torch.tensor(w, device=net.device)
    losses = []
    for it in range(40):
        y32 = net.forward(dg, save=True)
        dy, parts = net.mse(y32, t_t, w_t, 3.0 * g.T)
        losses.append(float(parts.cpu().numpy().sum()))
        net.backward(dy)
        net.adam_step(lr=1e-3)
    torch.cuda.synchronize()
    net._check_err()
    assert losses[-1] < 0.5 * losses[0], losses
    n0 = gnn.kernel_launches()
    assert n0 > 0
