"""GPU parity of the differentiable pairwise cDTW (cdtw_pair_fwd /
cdtw_pair_bwd) through the C ABI.

* Pre-normalised inputs without device z-normalisation: the device DP is
  replayed exactly by the oracle's float mode (one fused multiply-add per
  cell, same tie rule), so D is bit-identical and the gradients agree to
  float rounding of their short sums.
* Raw random walks with z-normalisation against the FP64 oracle: D within
  1e-4 relative of the FP64 optimum.  Smooth series leave near-ties along
  the path (relative predecessor gaps of 1e-7 are common), so a float DP may
  take another optimal path; the recorded device path is read back and must
  be a valid band path whose FP64 cost equals the FP64 optimum to 1e-5, and
  the device gradient must equal the FP64 gradient along that path to 1e-4
  of the gradient scale.
* The full 4096-pair workload (L = 256, W = 25) through size-independent
  properties: shift/scale invariance of the z-normalised gradient and
  agreement with the oracle on a sample."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _walks(rng, n, L):
    return np.cumsum(rng.standard_normal((n, L)), axis=1).astype(np.float32)


def _runs(path, n, L):
    raw = path.cpu().numpy()
    rows = raw[32 * n:32 * n + 4 * n * L].view(np.uint32).reshape(n, L)
    cols = raw[32 * n + 4 * n * L:32 * n + 8 * n * L].view(np.uint32).reshape(n, L)
    return rows, cols


def _check_fp64(q, s, W, euclid, D, gq, gs, rows, cols, dD=None):
    Do = oracle.pair_fwdbwd(q, s, W, euclid=euclid, znorm=True, dD=dD)[0]
    cost, gqp, gsp, valid = oracle.pair_path_grad(q, s, W, rows, cols, euclid, True, dD)
    assert valid.all()
    np.testing.assert_allclose(D, Do, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(cost, Do, rtol=1e-5, atol=1e-6)
    sc = np.maximum(np.abs(gqp).max(axis=1), np.abs(gsp).max(axis=1))[:, None]
    assert np.all(np.abs(gq - gqp) <= 1e-4 * sc)
    assert np.all(np.abs(gs - gsp) <= 1e-4 * sc)


def _run(h, q, s, W, euclid=True, znorm=True, dD=None, want_path=False):
    dq_ = torch.from_numpy(q).cuda()
    ds_ = torch.from_numpy(s).cuda()
    n, L = q.shape
    path = torch.empty(h.pair_path_bytes(n, L), dtype=torch.uint8, device="cuda")
    metric = 0 if euclid else 1
    D = h.pair_fwd(dq_, ds_, W, metric=metric, znorm=znorm, path=path)
    up = None if dD is None else torch.from_numpy(np.asarray(dD, np.float32)).cuda()
    gq, gs = h.pair_bwd(dq_, ds_, path, dD=up, metric=metric, znorm=znorm)
    torch.cuda.synchronize()
    out = (D.cpu().numpy(), gq.cpu().numpy(), gs.cpu().numpy())
    return out + _runs(path, n, L) if want_path else out


SHAPES = [(1, 0), (2, 1), (16, 0), (16, 15), (33, 12), (64, 9), (100, 99), (128, 12),
          (256, 25), (300, 70), (513, 130), (1024, 204), (2048, 409), (1100, 511)]


@pytest.mark.parametrize("L,W", SHAPES)
@pytest.mark.parametrize("euclid", [True, False])
def test_pair_exact_float_replay(handle, L, W, euclid):
    rng = np.random.default_rng(L * 7 + W)
    n = 9 if L <= 1024 else 3
    zq = rng.standard_normal((n, L)).astype(np.float32)
    zs = rng.standard_normal((n, L)).astype(np.float32)
    D, gq, gs = _run(handle, zq, zs, W, euclid, znorm=False)
    Do, gqo, gso, _ = oracle.pair_fwdbwd(zq, zs, W, euclid=euclid, znorm=False, f32=True)
    np.testing.assert_array_equal(D, Do.astype(np.float32))
    np.testing.assert_allclose(gq, gqo, rtol=1e-6, atol=1e-5)
    np.testing.assert_allclose(gs, gso, rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("L,W,n", [(256, 25, 512), (128, 12, 256), (2048, 409, 8)])
@pytest.mark.parametrize("euclid", [True, False])
def test_pair_znorm_against_fp64(handle, L, W, n, euclid):
    rng = np.random.default_rng(L + W + n)
    q, s = _walks(rng, n, L), _walks(rng, n, L)
    dD = rng.uniform(0.5, 2.0, n).astype(np.float32)
    D, gq, gs, rows, cols = _run(handle, q, s, W, euclid, znorm=True, dD=dD, want_path=True)
    _check_fp64(q, s, W, euclid, D, gq, gs, rows, cols, dD)


def test_pair_full_workload_properties(handle):
    """4096 pairs of length 256, W = 25 (10%)."""
    rng = np.random.default_rng(2024)
    n, L, W = 4096, 256, 25
    q, s = _walks(rng, n, L), _walks(rng, n, L)
    D, gq, gs, rows, cols = _run(handle, q, s, W, want_path=True)
    assert np.all(np.isfinite(D)) and np.all(D >= 0)
    # shift / scale invariance of the z-normalised distance
    for g, x in ((gq, q), (gs, s)):
        sc = np.abs(g).max(axis=1) * L
        assert np.all(np.abs(g.sum(axis=1)) <= 1e-5 * sc)
        xc = x - x.mean(axis=1, keepdims=True)
        assert np.all(np.abs((g * xc).sum(axis=1)) <= 1e-4 * sc * np.abs(xc).max(axis=1))
    idx = np.sort(rng.choice(n, 256, replace=False))
    _check_fp64(q[idx], s[idx], W, True, D[idx], gq[idx], gs[idx], rows[idx], cols[idx])


@pytest.mark.parametrize("L,W,n", [(300, 70, 40), (513, 130, 24), (1024, 204, 16),
                                   (2048, 409, 8), (1100, 511, 6), (700, 9, 33)])
@pytest.mark.parametrize("euclid", [True, False])
def test_pair_recompute_equals_stored_directions(handle, L, W, n, euclid):
    """The checkpointed mode recomputes each segment of anti-diagonals from
    its checkpoint with the forward's own arithmetic, so its path record is
    byte-identical to the stored-direction mode's, and so are D and the
    gradients; checked against FP64 as well."""
    rng = np.random.default_rng(L + 3 * W)
    q, s = _walks(rng, n, L), _walks(rng, n, L)
    dq_, ds_ = torch.from_numpy(q).cuda(), torch.from_numpy(s).cuda()
    metric = 0 if euclid else 1
    out = {}
    for mode in ("store", "recompute"):
        path = torch.empty(handle.pair_path_bytes(n, L), dtype=torch.uint8, device="cuda")
        D = handle.pair_fwd(dq_, ds_, W, metric=metric, path=path, mode=mode)
        assert handle.pair_last_mode() == mode
        gq, gs = handle.pair_bwd(dq_, ds_, path, metric=metric)
        out[mode] = (D.cpu().numpy(), path.cpu().numpy(), gq.cpu().numpy(), gs.cpu().numpy())
    for a, b in zip(out["store"], out["recompute"]):
        np.testing.assert_array_equal(a, b)
    assert (handle.pair_workspace_bytes(n, L, W, mode="recompute") <
            handle.pair_workspace_bytes(n, L, W, mode="store"))
    D, raw, gq, gs = out["recompute"]
    rows = raw[32 * n:32 * n + 4 * n * L].view(np.uint32).reshape(n, L)
    cols = raw[32 * n + 4 * n * L:32 * n + 8 * n * L].view(np.uint32).reshape(n, L)
    _check_fp64(q, s, W, euclid, D, gq, gs, rows, cols)


def test_pair_forward_only_and_one_sided_backward(handle):
    rng = np.random.default_rng(5)
    n, L, W = 33, 200, 20
    q, s = _walks(rng, n, L), _walks(rng, n, L)
    dq_, ds_ = torch.from_numpy(q).cuda(), torch.from_numpy(s).cuda()
    D0 = handle.pair_fwd(dq_, ds_, W).cpu().numpy()  # no path record
    D, gq, gs = _run(handle, q, s, W)
    np.testing.assert_array_equal(D0, D)
    path = torch.empty(handle.pair_path_bytes(n, L), dtype=torch.uint8, device="cuda")
    handle.pair_fwd(dq_, ds_, W, path=path)
    only_q, none_s = handle.pair_bwd(dq_, ds_, path, need_s=False)
    assert none_s is None
    np.testing.assert_array_equal(only_q.cpu().numpy(), gq)


def test_pair_errors(handle):
    from cudadtw_b200 import CudaDTWError
    q = torch.zeros((2, 1100), device="cuda")
    with pytest.raises(CudaDTWError) as e:
        handle.pair_fwd(q, q, 600)
    assert e.value.status == 5  # CDTW_EUNSUPPORTED
    big = torch.zeros((1, 8193), device="cuda")
    with pytest.raises(CudaDTWError):
        handle.pair_fwd(big, big, 10)
    with pytest.raises(CudaDTWError):
        handle._check(handle._lib.cdtw_pair_fwd(handle._h, q.data_ptr(), q.data_ptr(), 2, 1100,
                                                10, 0, 8, q.data_ptr(), None))
    with pytest.raises(CudaDTWError):  # the two path modes exclude each other
        handle._check(handle._lib.cdtw_pair_fwd(handle._h, q.data_ptr(), q.data_ptr(), 2, 1100,
                                                10, 0, 6, q.data_ptr(), q.data_ptr()))
