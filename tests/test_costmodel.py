"""The learned DFT pass-cost model on the CPU: the gradient oracle against
finite differences, the pass features, and the committed model (trained on the
GPU by the library's own kernels from the committed pass timings) against the
timing probe it replaces, on held-out LDE shapes."""
import json
import os

import numpy as np
import pytest

from oracle import mlp as OM
from lambda_vm_b200 import costmodel as CM
from lambda_vm_b200 import native


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = CM.init_params(3).astype(np.float64) + rng.normal(0, 0.05, OM.NP)
    X = rng.uniform(-1, 1, (40, OM.IN))
    y = rng.normal(0, 1, 40)
    _, g = OM.loss_grad(p, X, y)
    idx = rng.choice(OM.NP, 120, replace=False)
    for i in idx:
        e = np.zeros(OM.NP)
        e[i] = 1e-6
        fd = (OM.loss_grad(p + e, X, y)[0] - OM.loss_grad(p - e, X, y)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_pass_features():
    rec = {"log_len": 10, "tiles": 1024, "m": 9, "reps": 4, "inverse": 0, "pre": 1, "post": 1, "canon": 0}
    f = CM.features(rec, 4)
    assert f.shape == (native.MLP_IN,)
    assert f[0] == pytest.approx(2 / 3) and f[1] == pytest.approx(10 / 14)
    assert list(f[3:6]) == [1, 0, 0]
    assert f[6] == pytest.approx(np.log2(3) / 7) and f[7] == pytest.approx(12 / 9 - 1)
    assert f[8] == pytest.approx(2 / 3) and f[9] == 0 and f[10] == 1 and f[11] == 1 and f[12] == 0
    assert f[15] == pytest.approx(np.log2(1024 * 1024 * 12 * 4) / 32)
    assert list(CM.features(rec, 16)[3:6]) == [0, 0, 1]


def test_probe_rule_restates_the_tile_chooser():
    probe = {"10": {"4": 1.20, "8": 1.03, "16": 1.0}, "11": {"4": 1.0, "8": 0.99}}
    assert CM.probe_pick(probe, 10, 256) == 16
    assert CM.probe_pick(probe, 10, 3) == 4      # 4 x 1.20 < 16 x 1.0
    assert CM.probe_pick(probe, 11, 64) == 8     # 4-col 1 % cheaper: default kept
    assert CM.probe_pick(probe, 9, 40) == 16     # no probe data: the default


@pytest.mark.skipif(not os.path.exists(CM.MODEL), reason="no committed model")
def test_committed_model_beats_the_probe_on_heldout_shapes():
    params, meta = CM.load_model()
    data = CM.load_dataset()
    _, test = CM.split(data["records"])
    ev = CM.evaluate(test, params, data["probe"])
    assert ev["shapes"] >= 50
    # the model's picks cost no more in total than the probe's, and less than always using the default
    assert ev["ms"]["model"] <= ev["ms"]["probe"] * 1.0005
    assert ev["mean_regret"]["model"] <= ev["mean_regret"]["probe"]
    assert ev == meta["heldout"]
    # the host forward pass the tile chooser runs is the oracle's network
    X, _ = CM.design(test[:64])
    assert np.allclose(CM.predict_host(params, X), OM.forward(params, X)[0], rtol=1e-4, atol=1e-4)
