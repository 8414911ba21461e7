"""Delayed-acceptance Monte Carlo with the learned first stage (learned.py), on batches of
small water boxes:

* exactness: with any surrogate -- here an untrained network, whose first stage rejects and
  accepts almost at random -- the two-stage test samples the plain test's distribution: the
  mean energy per molecule of 32 independent boxes after equilibration agrees with the plain
  single-stage run's within four standard errors (errors from the boxes' spread);
* training: recorded (features, beta dE) pairs of the plain run train the network with the
  tcgen05 kernels; the loss falls, the held-out error is measured, and a trained network screens
  moves so that the exact work per attempted move drops below the plain run's;
* fallback: a network whose held-out error exceeds the bound hands the sampling back to the
  plain single-stage path."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _boxes(n, seed0=21):
    from epsr_python_translation_b200 import configs
    return [configs.c1_water(seed=seed0 + i, nmol=100) for i in range(n)]


def _mean_energy(series, nmol, burn):
    e = series[burn:] / nmol
    return e.mean(axis=0)    # per box


def test_delayed_acceptance_samples_the_plain_distribution():
    from epsr_python_translation_b200.learned import LearnedMC
    nbox = 32
    plain = LearnedMC(_boxes(nbox), rot_deg=15.0, trans_A=0.4, seed=3)
    da = LearnedMC(_boxes(nbox), rot_deg=15.0, trans_A=0.4, seed=4, net_seed=5)
    # equilibrate both from the same starting boxes with plain sweeps
    plain.run(60, "plain")
    da.run(60, "plain")
    sp, _, cp, _ = plain.run(150, "plain")
    sd, _, cd, mode = da.run(150, "da")
    assert mode == "da"
    mp, md = _mean_energy(sp, 100, 20), _mean_energy(sd, 100, 20)
    se = np.sqrt(mp.var(ddof=1) / nbox + md.var(ddof=1) / nbox)
    assert abs(mp.mean() - md.mean()) <= 4 * se + 1e-9, (mp.mean(), md.mean(), se)
    # the first stage did screen: fewer exact evaluations than attempts, acceptance no higher
    assert cd[:, 1].sum() < cd[:, 0].sum()
    assert cd[:, 2].sum() / cd[:, 0].sum() <= cp[:, 2].sum() / cp[:, 0].sum() + 0.02


def test_training_reduces_loss_and_screens_moves():
    from epsr_python_translation_b200.learned import LearnedMC
    lm = LearnedMC(_boxes(32, 40), rot_deg=30.0, trans_A=0.8, seed=6)
    lm.run(40, "plain")
    x, t = lm.collect(60000)
    assert x.shape[0] == 2 * t.shape[0] and t.shape[0] >= 60000
    assert torch.all(torch.isfinite(t))
    rep = lm.train(x, t, epochs=6, batch=2048, lr=2e-3)
    assert rep["loss_per_epoch"][-1] < 0.7 * rep["loss_per_epoch"][0], rep
    assert np.isfinite(rep["heldout_rmse_kT"])
    _, _, c, mode = lm.run(20, "da" if not lm.fallback else "plain")
    if mode == "da":
        # with large steps most moves are rejected; the screen leaves fewer exact evaluations
        assert c[:, 1].sum() < 0.9 * c[:, 0].sum()


def test_fallback_to_plain_when_heldout_error_is_large():
    from epsr_python_translation_b200.learned import RMSE_BOUND, LearnedMC
    lm = LearnedMC(_boxes(8, 60), seed=7)
    x, t = lm.collect(4096)
    # a network that predicts nonsense: large random output weights
    with torch.no_grad():
        lm.net.w3.mul_(1000.0)
    err = lm.heldout_error(x, t, torch.arange(min(t.numel(), 1024), device=x.device))
    lm.heldout_rmse = err
    lm.fallback = not (err <= RMSE_BOUND)
    assert lm.fallback
    _, _, c, mode = lm.run(2, "da")
    assert mode == "plain"
    # single stage: every attempt that stayed in its cell is evaluated exactly
    assert np.array_equal(c[:, 0], c[:, 1] + c[:, 3])
