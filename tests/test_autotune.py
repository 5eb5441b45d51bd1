"""Autotuner logic without a GPU: bucket keys, the candidate shapes the C ABI
accepts, selection of the fastest candidate, the per-query shape arrays and the
JSON cache."""
import numpy as np

from cudadtw_b200 import autotune as at


def test_bucket_keys():
    assert at.bucket(64, 0) == "M64_W0"
    assert at.bucket(65, 1) == "M128_W8"
    assert at.bucket(1024, 204) == "M1024_W208"
    assert at.bucket(11, 3) == "M64_W8"


def test_candidates_respect_kernel_limits():
    # register band only up to W = 96; strips of R rows need W >= R - 1
    assert (0, 1024) in at.batched_candidates(96)
    assert all(r != 0 for r, _ in at.batched_candidates(97))
    assert all(r <= 8 for r, _ in at.batched_candidates(7))
    assert at.variant_candidates(10) == ["register"]
    assert at.variant_candidates(40) == ["register", "strip16", "strip32", "lane"]
    assert at.variant_candidates(200) == ["strip16", "strip32", "lane"]
    assert at.variant_candidates(800) == ["strip16", "strip32"]
    assert at.variant_candidates(384) == ["strip16", "strip32"]  # no lane shape fits
    assert at.lane_shape(204) == (16, 26) and at.lane_shape(409) == (32, 26)


def test_tune_picks_fastest_and_maps_queries(tmp_path):
    rng = np.random.default_rng(0)
    qs = [np.zeros(m, np.float32) for m in (100, 120, 500, 900)]
    ws = [10, 12, 100, 180]

    def measure(idx, rows, tiles):  # fake: strips of 4 rows with 2048-wide tiles win
        return 1.0 + abs(rows - 4) + abs(tiles - 2048) / 1024 + 1e-3 * rng.random()

    table = at.tune_batched(qs, ws, measure)
    assert set(table) == {at.bucket(len(q), w) for q, w in zip(qs, ws)}
    for e in table.values():
        assert (e["rows"], e["tiles"]) == (4, 2048)
    rows, tiles = at.shapes_for(qs, ws, table)
    assert list(rows) == [4] * 4 and list(tiles) == [2048] * 4
    assert at.shapes_for(qs, ws, {}) == (None, None)

    path = str(tmp_path / "cache.json")
    at.save("B200-test", {"batched": table}, path)
    at.save("other", {"batched": {}}, path)
    assert at.load("B200-test", path)["batched"] == table
    assert at.load("missing", path) == {}


def test_tune_variants_fake():
    v = at.tune_variants([10, 50, 200], lambda w, var: {"register": 3, "strip16": 2,
                                                          "strip32": 1, "lane": 1.5}[var]
                         if w > 40 else 1)
    assert v == {"10": "register", "50": "strip32", "200": "strip32"}
    v = at.tune_variants([200], lambda w, var: {"strip16": 2, "strip32": 3, "lane": 1}[var])
    assert v == {"200": "lane"}
