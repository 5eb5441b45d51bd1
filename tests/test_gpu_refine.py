"""Template refinement (cdtw_refine_templates) through the C ABI: top-k matches
per template, then Adam steps on the templates, all steps in one graph; and
the refinement that searches the matches again at every step inside the
graph (cdtw_refine_templates_search).

* steps = 0: the reported losses are the mean z-normalised cDTW of each
  template over its matches, equal to the FP64 oracle's to 1e-4.
* one step: Adam's first update is -lr * g / (|g| + eps), i.e. -lr * sign(g)
  where |g| >> eps; its sign must match the FP64 oracle gradient on the
  elements where that gradient is not tiny.
* many steps on templates of several lengths (several groups and graph
  branches): the loss falls, and the final loss row equals the FP64 recheck
  of the refined templates against the same windows to 1e-4."""
import numpy as np
import pytest
import torch

import oracle
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from cudadtw_b200 import Handle
    h = Handle(0)
    x = synth.ecg_like(1 << 16, seed=11)
    dx = torch.from_numpy(x).cuda()
    rng = np.random.default_rng(3)
    temps, bands, locs = [], [], []
    for i, m in enumerate((64, 80, 96, 128, 64, 80)):
        q, _ = synth.cut_query(x, m, seed=50 + i, noise=0.2)
        q = q + rng.normal(0, 0.1, m).astype(np.float32)
        w = synth.band_from_percent(m, 10)
        avg, std = h.avg_std(dx, m)
        h.set_query(q, w)
        l, _ = h.topk(dx, avg, std, 20)
        assert l.size == 20
        temps.append(q.astype(np.float32))
        bands.append(w)
        locs.append(l)
    yield h, x, dx, temps, bands, np.stack(locs)
    h.close()


def fp64_loss_and_grad(x, temps, bands, locs):
    out_l, out_g = [], []
    for t, (q, w) in enumerate(zip(temps, bands)):
        m = q.size
        win = np.stack([x[s:s + m] for s in locs[t]]).astype(np.float32)
        qq = np.repeat(q[None, :], len(locs[t]), axis=0)
        D, dq, _, _ = oracle.pair_fwdbwd(qq, win, w, znorm=True)
        out_l.append(D.mean())
        out_g.append(dq.mean(axis=0))
    return np.array(out_l), out_g


def test_zero_steps_loss_matches_fp64(setup):
    h, x, dx, temps, bands, locs = setup
    new, losses = h.refine_templates(dx, temps, bands, locs, steps=0)
    ref, _ = fp64_loss_and_grad(x, temps, bands, locs)
    np.testing.assert_allclose(losses[0], ref, rtol=1e-4)
    for a, b in zip(new, temps):
        np.testing.assert_array_equal(a, b)


def test_first_step_follows_gradient_sign(setup):
    h, x, dx, temps, bands, locs = setup
    lr = 1e-2
    new, _ = h.refine_templates(dx, temps, bands, locs, steps=1, lr=lr)
    _, grads = fp64_loss_and_grad(x, temps, bands, locs)
    agree = total = 0
    for a, b, g in zip(new, temps, grads):
        step = a.astype(np.float64) - b
        big = np.abs(g) > 1e-2 * np.abs(g).max()
        assert np.all(np.abs(step) <= lr * 1.001)
        agree += np.sum(np.sign(step[big]) == -np.sign(g[big]))
        total += big.sum()
    assert agree >= 0.95 * total, (agree, total)


def test_many_steps_reduce_loss_fp64_recheck(setup):
    h, x, dx, temps, bands, locs = setup
    new, losses = h.refine_templates(dx, temps, bands, locs, steps=30, lr=1e-2)
    assert losses.shape == (31, len(temps))
    assert np.all(losses[-1] < losses[0])
    ref, _ = fp64_loss_and_grad(x, new, bands, locs)
    np.testing.assert_allclose(losses[-1], ref, rtol=1e-4)


def test_refine_rejects_bad_windows(setup):
    from cudadtw_b200 import CudaDTWError
    h, x, dx, temps, bands, locs = setup
    bad = locs.copy()
    bad[0, 0] = x.size  # past the end
    with pytest.raises(CudaDTWError):
        h.refine_templates(dx, temps, bands, bad, steps=1)


def test_search_refine_zero_steps_matches_topk_and_fp64(setup):
    """steps = 0: the matches are the top-k of each template, the loss the
    FP64 oracle's mean distance to them."""
    h, x, dx, temps, bands, locs = setup
    new, losses, got = h.refine_templates_search(dx, temps, bands, 20, steps=0)
    for t, (q, w) in enumerate(zip(temps, bands)):
        avg, std = h.avg_std(dx, q.size)
        h.set_query(q, w)
        want, _ = h.topk(dx, avg, std, 20)
        np.testing.assert_array_equal(got[t], want)
    ref, _ = fp64_loss_and_grad(x, temps, bands, got)
    np.testing.assert_allclose(losses[0], ref, rtol=1e-4)
    for a, b in zip(new, temps):
        np.testing.assert_array_equal(a, b)


def test_search_refine_first_step_equals_fixed_match_refine(setup):
    """The first step searches the same matches as cdtw_topk and runs the same
    kernels on them: one step gives bit-identical templates and losses to
    the fixed-match refinement given those matches."""
    h, x, dx, temps, bands, locs = setup
    a, la, _ = h.refine_templates_search(dx, temps, bands, 20, steps=1, lr=1e-2)
    b, lb = h.refine_templates(dx, temps, bands, locs, steps=1, lr=1e-2)
    np.testing.assert_array_equal(la[0], lb[0])
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)


def test_search_refine_many_steps(setup):
    """30 steps with fresh matches at every step: the last step's matches are
    the top-k of the refined templates (host top-k search), the last loss row
    equals the FP64 recheck against them, and the mean loss falls."""
    h, x, dx, temps, bands, locs = setup
    new, losses, got = h.refine_templates_search(dx, temps, bands, 20, steps=30, lr=1e-2)
    assert losses.shape == (31, len(temps))
    for t, (q, w) in enumerate(zip(new, bands)):
        avg, std = h.avg_std(dx, q.size)
        h.set_query(q, w)
        want, _ = h.topk(dx, avg, std, 20)
        np.testing.assert_array_equal(got[t], want)
    ref, _ = fp64_loss_and_grad(x, new, bands, got)
    np.testing.assert_allclose(losses[-1], ref, rtol=1e-4)
    assert losses[-1].mean() < losses[0].mean()


def test_search_refine_rejects_short_subject(setup):
    from cudadtw_b200 import CudaDTWError
    h, x, dx, temps, bands, locs = setup
    with pytest.raises(CudaDTWError):
        # 2^16 samples hold 512 segments of 2 x 64 windows: fewer than 2k
        h.refine_templates_search(dx, temps[:1], bands[:1], 300, steps=1)
