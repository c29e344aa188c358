"""The pass-cost MLP's GPU kernels (csrc/mlp.cu) against the float64 oracle
(oracle/mlp.py): loss and gradient of one forward/backward pass, predictions,
training; then the model trained by these kernels on the committed pass
timings against the timing probe on held-out LDE shapes, and a context that
chooses its tile widths with the model (same LDE, no probe launches)."""
import json
import os

import numpy as np
import pytest

from oracle import mlp as OM
from lambda_vm_b200 import costmodel as CM
from lambda_vm_b200 import native

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    p = (CM.init_params(seed) + rng.normal(0, 0.02, OM.NP)).astype(np.float32)
    X = rng.uniform(-1, 1, (n, OM.IN)).astype(np.float32)
    y = (np.sin(X[:, 0] * 2) + X[:, 1] * X[:, 2] + 0.1 * rng.normal(size=n)).astype(np.float32)
    return p, X, y


@pytest.mark.parametrize("n", [1, 127, 300])
def test_loss_and_gradient_match_the_oracle(be, n):
    p, X, y = _data(n, n)
    loss, g = CM.loss_grad(be, X, y, p)
    want_loss, want_g = OM.loss_grad(p.astype(np.float64), X, y)
    assert loss == pytest.approx(want_loss, rel=1e-5, abs=1e-6)
    scale = max(1e-6, float(np.abs(want_g).max()))
    assert np.abs(g - want_g).max() <= 2e-5 * scale + 1e-7
    # the reduction order is fixed: a second pass gives the same bits
    loss2, g2 = CM.loss_grad(be, X, y, p)
    assert loss2 == loss and np.array_equal(g, g2)


def test_predict_matches_the_oracle(be):
    p, X, _ = _data(500, 9)
    got = CM.predict(be, X, p)
    assert np.allclose(got, OM.forward(p.astype(np.float64), X)[0], rtol=1e-5, atol=1e-5)
    assert np.allclose(CM.predict_host(p, X), got, rtol=1e-5, atol=1e-5)


def test_training_reduces_the_loss(be):
    p, X, y = _data(1000, 4)
    l0, _ = OM.loss_grad(p.astype(np.float64), X, y)
    params, loss = CM.train(be, X, y, steps=1500, lr=3e-3, params=p)
    assert loss < l0 / 5
    assert loss == pytest.approx(OM.loss_grad(params.astype(np.float64), X, y)[0], rel=1e-3)


@pytest.mark.skipif(not os.path.exists(CM.DATASET), reason="no committed pass timings")
def test_model_trained_here_beats_the_probe_on_heldout_shapes(be):
    data = CM.load_dataset()
    train, test = CM.split(data["records"])
    X, y = CM.design(train)
    params, loss = CM.train(be, X, y)
    ev = CM.evaluate(test, params, data["probe"])
    assert ev["shapes"] >= 50 and loss < 0.05
    assert ev["ms"]["model"] <= ev["ms"]["probe"] * 1.0005
    assert ev["mean_regret"]["model"] <= ev["mean_regret"]["probe"]


@pytest.mark.skipif(not os.path.exists(CM.MODEL), reason="no committed model")
def test_context_with_the_model_chooses_widths_without_probing():
    from lambda_vm_b200 import math_cuda as mc
    from lambda_vm_b200.device import Backend
    import oracle as O
    params, _ = CM.load_model()
    rng = np.random.default_rng(8)
    n, m = 1 << 16, 40
    t = rng.integers(0, 2**64, size=(n, m), dtype=np.uint64)
    w = O.coset_weights(n, 3)
    fresh = Backend(0)
    try:
        CM.install(fresh, params)
        before = fresh.launches()
        got = mc.coset_lde_batch_base(t, 2, w, fresh)
        # the two-level root table and the four passes: no probe launches
        assert fresh.launches() - before == 5
        assert (got == O.canon_array(O.coset_lde_row_major(t, 2, w))).all()
    finally:
        fresh.close()
