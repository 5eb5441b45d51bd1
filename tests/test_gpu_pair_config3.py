"""The differentiated-cDTW workload at full size: 4096 (query, window) pairs of
length 256, both z-normalised random walks with N(0,1) increments, band 10 %
(W = 25), forward distance and gradients with respect to both series.

* FP64 central finite differences (h = 1e-6, on the exact FP64 widening of
  the float32 inputs) on 64 sampled pairs at non-tie points (the optimal
  path does not change within the step).
* An FP64 CPU backtracking gradient on all 4096 pairs.  Smooth random walks
  leave near-ties along almost every path (relative predecessor gaps around
  1e-7), so a float DP may follow another optimal path: along the path the
  device recorded, every pair's path must be a valid band path whose FP64
  cost equals the FP64 optimum (1e-5 relative), and the device gradient must
  equal the FP64 gradient along it (1e-4 of the gradient's scale)."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

N_PAIRS, L, W = 4096, 256, 25


@pytest.fixture(scope="module")
def config3():
    from cudadtw_b200 import Handle
    rng = np.random.default_rng(3)
    q = np.cumsum(rng.standard_normal((N_PAIRS, L)), axis=1).astype(np.float32)
    s = np.cumsum(rng.standard_normal((N_PAIRS, L)), axis=1).astype(np.float32)
    with Handle(0) as h:
        dq, ds = torch.from_numpy(q).cuda(), torch.from_numpy(s).cuda()
        path = torch.empty(h.pair_path_bytes(N_PAIRS, L), dtype=torch.uint8, device="cuda")
        D = h.pair_fwd(dq, ds, W, path=path)
        gq, gs = h.pair_bwd(dq, ds, path)
        torch.cuda.synchronize()
        raw = path.cpu().numpy()
    n = N_PAIRS
    rows = raw[32 * n:32 * n + 4 * n * L].view(np.uint32).reshape(n, L)
    cols = raw[32 * n + 4 * n * L:32 * n + 8 * n * L].view(np.uint32).reshape(n, L)
    return q, s, D.cpu().numpy(), gq.cpu().numpy(), gs.cpu().numpy(), rows, cols


def test_config3_gradient_central_differences(config3):
    """At each checked coordinate the FP64 backtracking gradients at x + h and
    x - h must agree (no near-tie of the optimal path is crossed within the
    step; otherwise the coordinate is skipped as a tie point).  There the
    central difference must equal the FP64 backtracking gradient (1e-5), and,
    for pairs whose device path is the FP64 path, the device gradient
    (1e-4 of the pair's gradient scale)."""
    q, s, D, gq, gs, _, _ = config3
    rng = np.random.default_rng(33)
    picks = rng.choice(N_PAIRS, 64, replace=False)
    q64, s64 = q[picks].astype(np.float64), s[picks].astype(np.float64)
    _, gq64, gs64, _ = oracle.pair_fwdbwd64(q64, s64, W)
    h = 1e-6
    smooth = tested = gpu_checked = 0
    for r, p in enumerate(picks):
        sc = max(np.abs(gq64[r]).max(), np.abs(gs64[r]).max())
        same = (np.abs(gq[p] - gq64[r]).max() <= 1e-4 * sc and
                np.abs(gs[p] - gs64[r]).max() <= 1e-4 * sc)
        for t in rng.choice(L, 4, replace=False):
            for side in (0, 1):
                tested += 1
                a, b = q64[r:r + 1].copy(), s64[r:r + 1].copy()
                x = a if side == 0 else b
                x[0, t] += h
                dp, gqp, gsp, _ = oracle.pair_fwdbwd64(a, b, W)
                x[0, t] -= 2 * h
                dm, gqm, gsm, _ = oracle.pair_fwdbwd64(a, b, W)
                if np.abs(gqp - gqm).max() > 1e-6 * sc or np.abs(gsp - gsm).max() > 1e-6 * sc:
                    continue  # a near-tie of the path lies within the step
                smooth += 1
                fd = (dp[0] - dm[0]) / (2 * h)
                g64 = (gq64 if side == 0 else gs64)[r, t]
                assert abs(fd - g64) <= 1e-5 * (1 + abs(g64)), (p, t, side, fd, g64)
                if same:
                    g = (gq if side == 0 else gs)[p, t]
                    assert abs(g - fd) <= 1e-4 * sc + 1e-5, (p, t, side, g, fd)
                    gpu_checked += 1
    assert smooth >= 0.75 * tested
    assert gpu_checked >= 0.25 * tested


def test_config3_fp64_backtracking_all_pairs(config3):
    """Every pair: the device path is a valid band path whose FP64 cost is
    the FP64 optimum, and the device gradient is the FP64 gradient along it."""
    q, s, D, gq, gs, rows, cols = config3
    Do, gqo, gso, _ = oracle.pair_fwdbwd(q, s, W, euclid=True, znorm=True)
    np.testing.assert_allclose(D, Do, rtol=1e-4, atol=1e-5)
    cost, gqp, gsp, valid = oracle.pair_path_grad(q, s, W, rows, cols, True, True)
    assert valid.all()
    np.testing.assert_allclose(cost, Do, rtol=1e-5, atol=1e-6)
    sc = np.maximum(np.abs(gqp).max(axis=1), np.abs(gsp).max(axis=1))[:, None]
    assert np.all(np.abs(gq - gqp) <= 1e-4 * sc)
    assert np.all(np.abs(gs - gsp) <= 1e-4 * sc)
    # and on almost every pair the device path is the oracle's own FP64 path
    # (about 99 % by the oracle's float replay of the device arithmetic)
    sco = np.maximum(np.abs(gqo).max(axis=1), np.abs(gso).max(axis=1))
    same = ((np.abs(gq - gqo).max(axis=1) <= 1e-4 * sco) &
            (np.abs(gs - gso).max(axis=1) <= 1e-4 * sco))
    assert same.mean() >= 0.95
