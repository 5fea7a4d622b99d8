"""The surrogate's hand-written training kernels and tensor-core inference,
against the FP64 CPU restatement in oracle/mlp_oracle.py."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trainer(cuda_ok):
    from argot_b200 import surrogate as S
    return S.Trainer("cuda", nT=32, seed=3)


def _tables():
    from argot_b200.pipeline import tables
    nu, cs = tables()
    cs = cs.astype(np.float64)
    nuf = nu.astype(np.float32).astype(np.float64)
    thr = np.array([1.0, 1.8125, 4.0])
    w6 = np.concatenate([cs, cs * np.maximum(nuf[:, None] - thr[None, :], 0)], 1)
    sig0 = np.array([cs[0, 0], cs[44, 1], cs[103, 2]])
    return cs, sig0, w6


def test_samples_match_exact_quadrature(trainer):
    X, Y = trainer.samples(4000, seed=11)
    X, Y = X.cpu().numpy(), Y.cpu().numpy()
    cs, sig0, w6 = _tables()
    want = MO.exact_targets(X, trainer.spec_np, trainer.i0_np, cs, sig0, w6)
    # float32 storage of q and of the inputs
    assert np.allclose(Y, want, rtol=2e-5, atol=2e-5)
    assert X[:, :3].min() >= -6 and X[:, :3].max() <= 3
    # Jensen: the thin limit bounds y from below, so q <= 0
    assert Y.max() <= 1e-6 and Y.min() > -12


def test_gradient_matches_fp64_oracle(trainer):
    import torch
    X, Y = trainer.samples(2048, seed=5)
    g, loss = trainer.gradient(X, Y)
    p = trainer.params.cpu().numpy()
    want_loss, want = MO.loss_and_grad(p, X.cpu().numpy(), Y.cpu().numpy())
    got = g.cpu().numpy().astype(np.float64)
    assert abs(loss / want_loss - 1) < 1e-4
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel < 2e-3, rel
    for lo, hi in ((MO.OFF_W1, MO.OFF_B1), (MO.OFF_W2, MO.OFF_B2), (MO.OFF_W4, MO.OFF_B4)):
        r = np.linalg.norm(got[lo:hi] - want[lo:hi]) / np.linalg.norm(want[lo:hi])
        assert r < 5e-3, (lo, r)
    # and the oracle's gradient is the derivative of its loss
    rng = np.random.default_rng(0)
    d = rng.standard_normal(p.size) * 1e-3
    lp, _ = MO.loss_and_grad(p + d, X.cpu().numpy()[:256], Y.cpu().numpy()[:256])
    lm, _ = MO.loss_and_grad(p - d, X.cpu().numpy()[:256], Y.cpu().numpy()[:256])
    _, g256 = MO.loss_and_grad(p, X.cpu().numpy()[:256], Y.cpu().numpy()[:256])
    fd = (lp - lm) / 2
    # BF16 rounding makes the loss piecewise constant in the weights; the
    # straight-through gradient predicts the smooth trend
    assert abs(fd - g256 @ d) < 0.2 * abs(g256 @ d) + 1e-9


def test_training_reduces_loss(trainer):
    X, Y = trainer.samples(1_000_000, seed=7)
    _, loss0 = trainer.gradient(X[:8192].contiguous(), Y[:8192].contiguous())
    hist = trainer.train(X, Y, epochs=4, batch=8192, lr=3e-3)
    assert hist[-1] < 0.1 * loss0, (loss0, hist)
    assert hist[-1] < hist[0]


def test_tensor_core_inference_matches_training_forward(trainer):
    from argot_b200 import surrogate as S
    X, _ = trainer.samples(3000, seed=9)
    p = trainer.params.cpu().numpy()
    sur = S.Surrogate(p, np.ones((6, S.ENV_BINS), np.float32), tol=1.0)
    t_tc = sur.eval(X).cpu().numpy()
    t_ref = trainer.predict(X).cpu().numpy()
    o, _ = MO.forward(p, X.cpu().numpy())
    t_orc = o * MO.OUT_SCALE + MO.OUT_SHIFT
    # same weights and rounding; the tensor-core path uses the hardware tanh
    # in SiLU and a different summation order
    assert np.max(np.abs(t_ref - t_orc)) < 5e-3
    assert np.max(np.abs(t_tc - t_orc)) < 2e-2
    assert np.mean(np.abs(t_tc - t_orc)) < 2e-3
