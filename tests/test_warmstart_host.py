"""Host side of the warm start (no GPU): scenario features, target transforms,
normalisation and batching."""
import numpy as np

from storm_b200 import fvt, gnn, scenarios, warmstart


def _sample(seed, n=2500):
    sc = scenarios.batch_channels(1, n, n + 1, seed=seed, opt_limiter=0)[0]
    pm = fvt.build_mesh(sc.problem)
    q, hbc = warmstart.scenario_q_hbc(sc)
    inp = warmstart.scenario_inputs(pm.numpy(), q, hbc, sc.options.h_dry)
    return sc, inp


def test_features_are_finite_and_describe_the_channel(storm_lib):
    sc, inp = _sample(3)
    T = sc.n_elems
    assert inp.x_node.shape == (T, gnn.IN_NODE) and inp.x_edge.shape == (3, T, gnn.IN_EDGE)
    assert np.isfinite(inp.x_node).all() and np.isfinite(inp.x_edge).all()
    assert (inp.d0 >= 0).all()
    # exactly one inflow and one outflow string of cells, walls elsewhere on the boundary
    fin, fout = inp.x_node[:, 7], inp.x_node[:, 8]
    assert 0 < fin.sum() < T and 0 < fout.sum() < T and not (fin * fout).any()
    # along-channel distance: 0 at the outflow, about the channel length at the inflow
    s = inp.x_node[:, 10]
    assert s[fout > 0].max() < 0.05 and abs(s[fin > 0].mean() - 1.0) < 1e-6
    # normal-depth estimate from the mesh close to the generator's own value
    h_n = inp.x_node[0, 14] * 5.0
    assert abs(h_n - sc.info["h_normal"]) < 0.35 * sc.info["h_normal"]
    # edge rows without a neighbour carry no features
    assert not inp.x_edge[inp.nbr < 0].any()


def test_target_roundtrip():
    sc, inp = _sample(4)
    rng = np.random.default_rng(0)
    h = inp.d0 + rng.uniform(-0.2, 0.2, size=len(inp.d0))
    h = np.maximum(h, 0.01)
    u = rng.normal(size=len(h))
    v = rng.normal(size=len(h))
    t = warmstart.targets(inp, h, u, v)
    h2, u2, v2 = warmstart.state_from_prediction(inp, t)
    assert np.allclose(h2, h, atol=1e-5)
    assert np.allclose(u2, u, atol=1e-4 * np.abs(u).max() / np.maximum(h, 0.01).min())


def test_normalizer_and_grouping():
    samples = []
    for seed in (5, 6, 7):
        sc, inp = _sample(seed, n=2000 + 300 * seed)
        samples.append(warmstart.Sample(inp, warmstart.targets(inp, sc.h0, sc.u0, sc.v0)))
    norm = warmstart.Normalizer.fit(samples)
    xs = np.concatenate([norm.inputs(s.inp).x_node for s in samples])
    used = norm.node_std != 1.0
    assert np.allclose(xs[:, used].mean(axis=0), 0.0, atol=1e-4)
    assert np.allclose(xs[:, used].std(axis=0), 1.0, atol=1e-3)
    assert not xs[:, 30:].any()  # padding columns stay zero
    t = samples[0].target
    assert np.allclose(norm.untarget(norm.target(t)), t, atol=1e-4)
    groups = warmstart.group_samples(samples, cells_per_batch=5000)
    assert sum(len(g) for g in groups) == 3 and all(len(g) >= 1 for g in groups)
