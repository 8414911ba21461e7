"""The surrogate network's tcgen05 kernels against PyTorch and the NumPy FP32 restatement
(oracle/mlp_ref.py): the raw tensor-core product (TMA-staged BF16 tiles, FP32 accumulators in
tensor memory) at several shapes, split-K and ragged row counts; the forward pass; the loss
gradients of one training step (read back from the Adam first moment); and three Adam steps.

Tolerances: the product is FP32 accumulation of exact BF16 products, so it matches a double
product of the same BF16 values to 1e-5 relative to the sum of |terms|; the network's values
match the restatement (same BF16 rounding points, FP32 vs double accumulation) to 2e-3
relative, gradients to 1e-2 of their largest magnitude (a gradient feeds through BF16-rounded
intermediates, where one rounding flip moves a term by 2^-8)."""

import numpy as np
import pytest
import torch

from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _bf(a):
    return torch.from_numpy(mlp_ref.bf16(np.asarray(a, np.float32))).cuda().to(torch.bfloat16)


@pytest.mark.parametrize("m,n,k,ks,acc", [(128, 128, 64, 1, False), (256, 256, 1280, 1, False),
                                          (200, 128, 128, 1, False), (128, 1280, 2048, 8, True),
                                          (384, 128, 1280, 4, True)])
def test_umma_gemm_matches_double_product(m, n, k, ks, acc):
    from epsr_python_translation_b200.surrogate import umma_gemm
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((n, k)).astype(np.float32)
    at, bt = _bf(a), _bf(b)
    out = umma_gemm(at, bt, kslices=ks, accumulate=acc)
    torch.cuda.synchronize()
    a64 = at.float().cpu().numpy().astype(np.float64)
    b64 = bt.float().cpu().numpy().astype(np.float64)
    ref = a64 @ b64.T
    scale = np.abs(a64) @ np.abs(b64).T
    err = np.abs(out.cpu().numpy() - ref)
    assert np.all(err <= 1e-5 * scale + 1e-6), float(np.max(err / (scale + 1e-30)))


def _features(rows, seed):
    rng = np.random.default_rng(seed)
    x = np.abs(rng.standard_normal((rows, mlp_ref.IN))).astype(np.float32) * 0.5
    x[rng.random(x.shape) < 0.7] = 0.0      # sparse like radial histograms
    return mlp_ref.bf16(x)


def test_forward_matches_restatement():
    from epsr_python_translation_b200.surrogate import SurrogateNet
    p = mlp_ref.init_params(1)
    p["b1"] = (np.random.default_rng(2).standard_normal(128) * 0.1).astype(np.float32)
    p["b3"] = np.array([0.3], np.float32)
    net = SurrogateNet(params=p)
    x = _features(300, 3)
    y = net.forward(_bf(x)).cpu().numpy()
    net.check_status()
    yr, _ = mlp_ref.forward(p, x)
    assert np.allclose(y, yr, rtol=2e-3, atol=2e-3 * np.max(np.abs(yr))), float(np.max(np.abs(y - yr)))


def test_training_gradients_match_restatement():
    from epsr_python_translation_b200.surrogate import SurrogateNet
    p = mlp_ref.init_params(4)
    net = SurrogateNet(params={k: v.copy() for k, v in p.items()})
    R = 512
    x = _features(R, 5)
    # pairs (2q, 2q+1): the same move's features in both orders
    x[1::2] = np.concatenate([x[0::2, 640:], x[0::2, :640]], axis=1)
    tgt = np.random.default_rng(6).standard_normal(R // 2).astype(np.float32)
    xt = _bf(x)
    xtt = xt.t().contiguous()
    tg = torch.from_numpy(tgt).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.train_step(xt, xtt, 0, R, tg, lr=1e-12, loss=loss)
    torch.cuda.synchronize()
    net.check_status()
    lref, gref = mlp_ref.grads(p, x, tgt)
    assert abs(float(loss.item()) - lref) <= 2e-3 * lref
    m1 = net.m1.cpu().numpy() / 0.1          # after one step the first moment is 0.1 x gradient
    offs = {"w1": 0, "b1": 128 * 1280, "w2": 128 * 1280 + 128, "b2": 128 * 1280 + 128 + 128 * 128,
            "w3": 128 * 1280 + 2 * 128 + 128 * 128, "b3": 128 * 1280 + 3 * 128 + 128 * 128}
    for k, o in offs.items():
        g = gref[k].reshape(-1)
        mine = m1[o:o + g.size]
        tol = 1e-2 * np.max(np.abs(g)) + 1e-9
        assert np.max(np.abs(mine - g)) <= tol, (k, float(np.max(np.abs(mine - g))), tol)


def test_adam_steps_follow_restatement_and_reduce_loss():
    from epsr_python_translation_b200.surrogate import SurrogateNet
    p = mlp_ref.init_params(7)
    net = SurrogateNet(params={k: v.copy() for k, v in p.items()})
    R = 256
    x = _features(R, 8)
    x[1::2] = np.concatenate([x[0::2, 640:], x[0::2, :640]], axis=1)
    # a learnable target: a fixed linear function of the feature difference
    wt = np.random.default_rng(9).standard_normal(640).astype(np.float32) * 0.05
    tgt = ((x[0::2, 640:] - x[0::2, :640]) @ wt).astype(np.float32)
    xt = _bf(x)
    xtt = xt.t().contiguous()
    tg = torch.from_numpy(tgt).cuda()
    m = {k: np.zeros_like(v, dtype=np.float64) for k, v in p.items()}
    v = {k: np.zeros_like(v2, dtype=np.float64) for k, v2 in p.items()}
    losses = []
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    for step in range(1, 4):
        net.train_step(xt, xtt, 0, R, tg, lr=1e-3, loss=loss)
        lref, g = mlp_ref.grads(p, x, tgt)
        mlp_ref.adam(p, g, m, v, step, 1e-3)
        losses.append(float(loss.item()))
        assert abs(losses[-1] - lref) <= 5e-3 * lref + 1e-6
    # Adam normalises each step by the gradient's own magnitude, so a parameter whose gradient
    # is near zero can take a full step of either sign on rounding alone: nearly all
    # parameters agree closely, every one within the three steps' reach
    got = net.params()
    for k in p:
        d = np.abs(got[k] - p[k])
        assert np.mean(d <= 2e-4) >= 0.99, (k, float(np.mean(d <= 2e-4)))
        assert np.max(d) <= 6.1e-3, (k, float(np.max(d)))
    for _ in range(60):
        net.train_step(xt, xtt, 0, R, tg, lr=1e-3, loss=loss)
    assert float(loss.item()) < 0.5 * losses[0]
