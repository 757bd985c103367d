"""Learned surrogate end to end on a reduced surrogate set: targets from the
ensemble solver, a committee trained on the GPU, held-out error against the
solver, what the trained network gains over predicting without it, and the
disagreement fallback."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_pipeline_reduced(gpu_lib):
    from cosenu_b200.surrogate import Surrogate, features, solve_pee, surrogate_instances
    # reduced: nz 256 on [-600, 600], runs to t = 250 / mu, nvz 128 as the full surrogate workload
    train = surrogate_instances(192, seed=11, nz=256, t_factor=250.0)
    test = surrogate_instances(48, seed=12, nz=256, t_factor=250.0)
    t0 = time.perf_counter()
    y_train = solve_pee(train)
    y_test = solve_pee(test)
    t_solver = (time.perf_counter() - t0) * len(test) / (len(train) + len(test))
    assert np.isfinite(y_train).all() and y_train.min() > 0 and y_train.max() <= 1.05
    x_train = np.stack([features(i) for i in train])
    x_test = np.stack([features(i) for i in test])
    sur = Surrogate(n_models=3)
    losses = sur.fit(x_train, y_train, epochs=150, batch=64, lr=1e-3)
    for ls in losses:
        assert ls[-1] < ls[0] / 5
    t1 = time.perf_counter()
    mean, spread = sur.committee(x_test)
    t_net = time.perf_counter() - t1
    err_net = np.abs(mean - y_test).mean()
    # the same question answered without the trained network
    err_mean = np.abs(y_train.mean(axis=0) - y_test).mean()   # training-set average
    err_none = np.abs(1.0 - y_test).mean()                    # no flavour conversion
    assert err_net < 0.5 * err_mean and err_net < 0.5 * err_none, (err_net, err_mean, err_none)
    assert t_net < t_solver / 100
    # out of distribution (alpha far outside [0.6, 1.2]): the committee
    # disagrees more than on the held-out set
    import dataclasses
    ood = [dataclasses.replace(test[0], alpha=3.0)]
    _, s_ood = sur.committee(np.stack([features(i) for i in ood]))
    assert s_ood[0] > np.median(spread)
    # fallback path: with a zero threshold every instance goes to the solver
    pred = sur.predict(test[:4], threshold=0.0)
    assert pred.fallback.all()
    assert np.abs(pred.pee - y_test[:4]).max() <= 1e-10
    sur.close()
