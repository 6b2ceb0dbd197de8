"""The learned result-count model: the device forward pass and gradient
against the CPU restatement (oracle/model_oracle.py), and what the trained
model gains over the sampled estimator on the 6-D workload."""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin, synth
from oracle import model_oracle as MO

pytestmark = pytest.mark.gpu


def test_forward_and_gradient_match_cpu():
    rng = np.random.default_rng(5)
    w = (rng.standard_normal(MO.NW) * 0.3).astype(np.float32)
    X = rng.uniform(0, 1, size=(300, MO.F)).astype(np.float32)   # 3 minibatches, the last one partial
    y = rng.uniform(0, 6, size=300).astype(np.float32)
    with SelfJoin(0) as sj:
        sj.model_weights(w)
        out = sj.model_predict(X)
        loss, grad = sj.model_loss_grad(X, y)
    ref_out = MO.forward(w, X)
    ref_loss, ref_grad = MO.loss_grad(w, X, y)
    np.testing.assert_allclose(out, ref_out, rtol=1e-4, atol=1e-4)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    np.testing.assert_allclose(grad, ref_grad, rtol=2e-3, atol=2e-5 * np.abs(ref_grad).max())


def test_training_is_deterministic_and_fits():
    pts = synth.generate("c3_gmm6d", 400_000)
    w = synth.WORKLOADS["c3_gmm6d"]
    cfg = JoinConfig(indexed_dims=6, stamp=True)
    weights, fits = [], []
    for _ in range(2):
        with SelfJoin(0) as sj:
            sj.run(pts, w.eps, cfg)
            X, y = sj.model_features()
            l0 = float(np.mean((sj.model_predict(X) - y) ** 2))
            sj.model_train(300)
            weights.append(sj.model_weights())
            l1 = float(np.mean((sj.model_predict(X) - y) ** 2))
            fits.append((l0, l1))
    assert np.array_equal(weights[0], weights[1])
    l0, l1 = fits[0]
    assert l1 < 0.25 * l0


def test_learned_estimate_gain_6d():
    """Train on the 6-D workload at half size, then join the full workload
    with the learned estimator: the same pair set, an estimate within the
    buffer margin (no re-run), and a cheaper estimate than the sampling pass."""
    w = synth.WORKLOADS["c3_gmm6d"]
    cfg = JoinConfig(indexed_dims=6, stamp=True)
    with SelfJoin(0) as sj:
        sj.run(synth.generate("c3_gmm6d", 2_500_000), w.eps, cfg)
        sj.model_train(400)
        full = synth.generate("c3_gmm6d")
        # each estimator's second full-size join is compared (the first one
        # allocates the buffers it needs)
        sj.run(full, w.eps, cfg)
        s_samp = sj.run(full, w.eps, cfg)
        c0, t0 = sj.counts(), sj.table()
        lcfg = JoinConfig(indexed_dims=6, stamp=True, learned=True)
        sj.run(full, w.eps, lcfg)
        s_learn = sj.run(full, w.eps, lcfg)
        c1, t1 = sj.counts(), sj.table()
    assert np.array_equal(c0, c1) and np.array_equal(t0, t1)
    R = s_learn["total_pairs"]
    err_l = abs(s_learn["estimate"] - R) / R
    err_s = abs(s_samp["estimate"] - R) / R
    print(f"\n6-D {R} pairs: sampled estimate {s_samp['estimate']} ({err_s:.3%}, "
          f"{s_samp['dev_ms_estimate']:.3f} ms), learned {s_learn['estimate']} ({err_l:.3%}, "
          f"{s_learn['dev_ms_estimate']:.3f} ms)")
    assert s_learn["reruns"] == 0
    assert err_l < 0.2
    assert s_learn["dev_ms_estimate"] < s_samp["dev_ms_estimate"]
