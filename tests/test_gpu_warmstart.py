"""The trained warm start against the method without it: on held-out ensemble
members (seeds disjoint from the training data) the solver, started from the
network's prediction, reaches the same stop test (RMS dh < 1e-6) in fewer iterations
than from the cold start, and its steady depth agrees with the cold run's."""
import os

import numpy as np
import pytest

from storm_b200 import abi, fvt, scenarios, warmstart

pytestmark = pytest.mark.gpu

MODEL = os.path.join(os.path.dirname(warmstart.__file__), "models", "warmstart_channels.npz")


@pytest.mark.skipif(not os.path.exists(MODEL), reason="no trained model in the package")
def test_warm_start_needs_fewer_iterations(storm_lib):
    net, norm = warmstart.load_model(MODEL)
    scs = scenarios.batch_channels(6, 2000, 5000, seed=424_242, opt_limiter=0)
    inps = []
    for sc in scs:
        pm = fvt.build_mesh(sc.problem)
        q, hbc = warmstart.scenario_q_hbc(sc)
        inps.append(warmstart.scenario_inputs(pm.numpy(), q, hbc, sc.options.h_dry))
    preds = warmstart.predict(net, norm, inps, "cuda:0")
    states = [warmstart.state_from_prediction(i, p) for i, p in zip(inps, preds)]
    for h, u, v in states:
        assert np.isfinite(h).all() and (h >= 0).all() and np.isfinite(u).all() and np.isfinite(v).all()
    cold = warmstart.run_steady_batch(scs, istop=40000, precision=abi.PREC_MIXED)
    warm = warmstart.run_steady_batch(scs, states=states, istop=40000, precision=abi.PREC_MIXED)
    assert cold["converged"].all() and warm["converged"].all()
    assert warm["iters"].mean() < 0.67 * cold["iters"].mean(), (warm["iters"], cold["iters"])
    # what the network adds over its analytic prior (zero network output through the
    # same mapping to h, hu, hv): fewer iterations to the same stop test
    prior = [warmstart.state_from_prediction(i, np.zeros((len(i.d0), 3), dtype=np.float32)) for i in inps]
    pri = warmstart.run_steady_batch(scs, states=prior, istop=40000, precision=abi.PREC_MIXED)
    assert pri["converged"].all()
    assert warm["iters"].mean() < 0.8 * pri["iters"].mean(), (warm["iters"], pri["iters"])
    for a, b in zip(warm["states"], cold["states"]):
        # both runs stop at RMS dh < 1e-6, a few cm short of the steady state
        assert np.abs(a["h"] - b["h"]).max() < 0.25


MODEL_20K = os.path.join(os.path.dirname(warmstart.__file__), "models", "warmstart_channels_20k-40k.npz")


@pytest.mark.skipif(not os.path.exists(MODEL_20K), reason="no 20k-40k model in the package")
def test_warm_start_20k_40k_beats_cold_and_prior(storm_lib):
    """The 20k-40k-cell model on four held-out members of that band (seeds disjoint
    from its training data): fewer iterations to RMS dh < 1e-6 than the cold start
    and than the analytic prior alone (zero network output, same mapping)."""
    net, norm = warmstart.load_model(MODEL_20K)
    scs = scenarios.batch_channels(4, 20_000, 40_000, seed=515_151, opt_limiter=0)
    inps = []
    for sc in scs:
        pm = fvt.build_mesh(sc.problem)
        q, hbc = warmstart.scenario_q_hbc(sc)
        inps.append(warmstart.scenario_inputs(pm.numpy(), q, hbc, sc.options.h_dry))
    preds = warmstart.predict(net, norm, inps, "cuda:0")
    warm = [warmstart.state_from_prediction(i, p) for i, p in zip(inps, preds)]
    prior = [warmstart.state_from_prediction(i, np.zeros((len(i.d0), 3), dtype=np.float32)) for i in inps]
    runs = {name: warmstart.run_steady_batch(scs, states=st, istop=60000, precision=abi.PREC_MIXED,
                                             keep_states=False)
            for name, st in (("cold", None), ("prior", prior), ("warm", warm))}
    assert all(r["converged"].all() for r in runs.values()), {k: r["iters"] for k, r in runs.items()}
    assert runs["warm"]["iters"].mean() < 0.8 * runs["cold"]["iters"].mean(), runs["warm"]["iters"]
    assert runs["warm"]["iters"].mean() < 0.8 * runs["prior"]["iters"].mean(), runs["prior"]["iters"]
