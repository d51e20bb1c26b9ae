"""CPU tests of the grouped GEMM's host-side scheduling (no GPU)."""
import math

import pytest

import sgemm_b200 as sg


def test_bucket_classes():
    assert sg.grouped_bucket(64, 64, 64) == 0
    assert sg.grouped_bucket(64, 64, 4096) == 2
    assert sg.grouped_bucket(512, 512, 1000) == 4
    assert sg.grouped_bucket(4096, 4096, 4096) == 8
    assert sg.grouped_bucket(1024, 512, 100) == 3
    assert sg.grouped_bucket(2048, 512, 100) == 6


TILES = {"tall": (128, 64, 1.0), "wide": (64, 128, 0.994), "skinny": (32, 128, 0.75)}


def _tile_for(m, n, bucket_tile="tall"):
    """The library's per-problem rule: the bucket's tile unless another tile's
    zero-padded area per unit efficiency is at least 2% smaller."""
    def cost(t):
        bm, bn, eff = TILES[t]
        return math.ceil(m / bm) * bm * math.ceil(n / bn) * bn / eff
    best = bucket_tile
    for t in TILES:
        if cost(t) < 0.98 * cost(bucket_tile) and cost(t) < cost(best):
            best = t
    return best


def _area(rows, n, t):
    bm, bn, eff = TILES[t]
    return math.ceil(rows / bm) * bm * math.ceil(n / bn) * bn / eff


def _tiles_for(m, n, bucket_tile="tall"):
    """Tile count of a split-1 problem under the library's rule: the single
    tile above, or -- when it pads at least 2% less -- the whole tiles of a
    taller shape over the first rows plus a strip of a shorter shape over the
    rest."""
    if m == 0 or n == 0:
        return 0, None
    best = _tile_for(m, n, bucket_tile)
    best_area = _area(m, n, best)
    bm, bn, _ = TILES[best]
    count, mixed = math.ceil(m / bm) * math.ceil(n / bn), None
    for t in ("tall", "wide"):
        for u in ("wide", "skinny"):
            if TILES[u][0] >= TILES[t][0]:
                continue
            bulk = m // TILES[t][0] * TILES[t][0]
            if bulk in (0, m):
                continue
            a = _area(bulk, n, t) + _area(m - bulk, n, u)
            if a < 0.98 * best_area:
                best_area = a
                mixed = (t, u)
                count = (bulk // TILES[t][0]) * math.ceil(n / TILES[t][1]) + \
                    math.ceil((m - bulk) / TILES[u][0]) * math.ceil(n / TILES[u][1])
    return count, mixed


def test_schedule_default_counts():
    shapes = [(64, 64, 64), (300, 520, 1001), (4096, 4096, 64), (1, 1, 1), (129, 257, 0),
              (136, 4096, 4096), (200, 4096, 4096), (16, 4096, 4096)]
    probs = sg.host_problems(shapes)
    s = sg.grouped_schedule(probs)
    tiles = sum(_tiles_for(m, n)[0] for m, n, _ in shapes)
    assert s["tiles"] == tiles
    assert s["work_items"] == tiles  # no split-K by default: results equal the plain path
    assert s["workspace_bytes"] == 0
    # the rule moves some of these off the default tile
    assert [_tile_for(m, n) for m, n, _ in shapes[:5]] == ["tall", "wide", "tall", "skinny",
                                                           "wide"]
    # tall-skinny serving requests: 136 rows as one 128-row tile plus a strip
    # of 32-row tiles instead of two 64-row tiles
    assert _tiles_for(136, 4096)[1] == ("tall", "skinny")
    assert _tiles_for(16, 4096)[1] is None


def test_schedule_ignores_table_for_other_device(tmp_path):
    p = tmp_path / "t.json"
    p.write_text('{\n "device": "Some Other GPU",\n "sm_count": 7,\n "stages": 3,\n'
                 ' "buckets": [\n  {"mn": 0, "k": 2, "tile": 1, "split": 4}\n ]\n}\n')
    probs = sg.host_problems([(64, 64, 4096)])
    assert sg.grouped_schedule(probs, str(p))["work_items"] == 1


def test_schedule_rejects_bad_problem():
    probs = sg.host_problems([(64, 64, 64)])
    probs[0].ldc = 3
    with pytest.raises(sg.SgemmError) as e:
        sg.grouped_schedule(probs)
    assert e.value.status == sg.ERR_INVALID_ARG


def test_schedule_uses_skinny_tile_for_short_problems():
    # problems a few rows tall run on 32 x 128 tiles instead of padding
    # 128-row tiles; up to 64 rows the 64 x 128 tile is cheaper
    shapes = [(16, 4096, 4096), (1, 1000, 300), (33, 4100, 64), (48, 640, 2048)]
    assert [_tile_for(m, n) for m, n, _ in shapes] == ["skinny", "skinny", "wide", "wide"]
    s = sg.grouped_schedule(sg.host_problems(shapes))
    want = 0
    for m, n, _ in shapes:
        bm, bn, _ = TILES[_tile_for(m, n)]
        want += math.ceil(m / bm) * math.ceil(n / bn)
    assert s["tiles"] == want
    # square problems keep the 128 x 64 tile
    s = sg.grouped_schedule(sg.host_problems([(256, 256, 256)]))
    assert s["tiles"] == math.ceil(256 / 128) * math.ceil(256 / 64)
