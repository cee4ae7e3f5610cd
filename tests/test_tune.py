"""Tile-shape variants and the autotuner's table (host side, no GPU): the
selection rule, the table format, and the library's table loader and
per-class variant setting (pa_set_tile_variant, pa_load_tile_table,
pa_tile_shape)."""

import pytest

from pysisyphus_addons import _native as nat
from pysisyphus_addons import tune


@pytest.fixture(autouse=True)
def default_variants():
    saved = {(a, b): nat.get_tile_variant(a, b) for a in range(2 * nat.LMAX + 1) for b in range(nat.LAUXMAX + 1)}
    yield
    for (a, b), v in saved.items():
        nat.set_tile_variant(a, b, v)


def test_choose_mean_ratio_and_margin():
    times = {
        "small": {0: {(4, 3): 1.0, (4, 2): 1.0, (3, 5): 2.0}, 1: {(4, 3): 0.80, (4, 2): 1.30, (3, 5): 1.98},
                  2: {(4, 3): 0.90, (4, 2): 1.50, (3, 5): 1.70}},
        "large": {0: {(4, 3): 100.0, (4, 2): 50.0, (3, 5): 10.0}, 1: {(4, 3): 90.0, (4, 2): 70.0, (3, 5): 10.0},
                  2: {(4, 3): 99.0, (4, 2): 80.0, (3, 5): 9.0}},
    }
    table, mean = tune.choose(times, margin=0.03)
    assert mean[(4, 3)][1] == pytest.approx((0.8 + 0.9) / 2)
    assert table[(4, 3)] == 1  # 0.85 < 0.97
    assert table[(4, 2)] == 0  # every alternative slower
    assert table[(3, 5)] == 2  # (0.85 + 0.9) / 2
    # a gain inside the margin keeps variant 0
    table, _ = tune.choose({"w": {0: {(1, 1): 1.0}, 1: {(1, 1): 0.98}}}, margin=0.03)
    assert table[(1, 1)] == 0


def test_choose_rejects_a_loss_on_one_workload_and_duplicate_shapes():
    times = {"a": {0: {(4, 3): 1.0}, 1: {(4, 3): 0.70}, 2: {(4, 3): 0.5}},
             "b": {0: {(4, 3): 1.0}, 1: {(4, 3): 1.05}, 2: {(4, 3): 0.9}}}
    # variant 1: mean 0.875 but 5 % slower on b; variant 2 wins on both
    table, _ = tune.choose(times, margin=0.03)
    assert table[(4, 3)] == 2
    # variant 2 has variant 0's shape: the same kernel, so its gain is noise
    table, mean = tune.choose(times, margin=0.03, shapes={(4, 3): {0: "s0", 1: "s1", 2: "s0"}})
    assert table[(4, 3)] == 0 and 2 not in mean[(4, 3)]


def test_choose_ignores_classes_without_a_baseline():
    table, mean = tune.choose({"w": {0: {(2, 2): 1.0}, 1: {(2, 2): 0.5, (3, 3): 0.1}}})
    assert table == {(2, 2): 1} and (3, 3) not in mean


def test_table_format_round_trip(tmp_path):
    table = {(4, 3): 1, (3, 5): 2, (0, 0): 0}
    text = tune.format_table(table, {(4, 3): {0: 1.0, 1: 0.85}}, header=["device: test"])
    assert tune.parse_table(text) == {(4, 3): 1, (3, 5): 2}
    p = tmp_path / "tiles.txt"
    p.write_text(text)
    assert nat.load_tile_table(p) == 2
    assert nat.get_tile_variant(4, 3) == 1 and nat.get_tile_variant(3, 5) == 2 and nat.get_tile_variant(0, 0) == 0


def test_table_errors_leave_the_selection(tmp_path):
    nat.set_tile_variant(4, 3, 1)
    for bad in ["4 3\n", "4 3 1 7\n", "9 0 1\n", "4 6 1\n", f"4 3 {nat.TILE_VARIANTS}\n", "4 x 1\n"]:
        p = tmp_path / "bad.txt"
        p.write_text("2 2 1\n" + bad)
        with pytest.raises(RuntimeError):
            nat.load_tile_table(p)
        assert nat.get_tile_variant(4, 3) == 1 and nat.get_tile_variant(2, 2) == 0
    with pytest.raises(RuntimeError):
        nat.load_tile_table(tmp_path / "missing.txt")


def test_set_tile_variant_range():
    for args in [(-1, 0, 0), (2 * nat.LMAX + 1, 0, 0), (0, nat.LAUXMAX + 1, 0), (0, 0, -1), (0, 0, nat.TILE_VARIANTS)]:
        with pytest.raises(RuntimeError):
            nat.set_tile_variant(*args)


def test_tile_shapes():
    """Variant 0 is the largest tile for two blocks per SM; variant 1 keeps at
    least half of it and never fewer busy lanes; variant 2 sizes team classes
    (L > 5) for three blocks per SM where one shell fits in 72 KB."""
    for lab in range(2 * nat.LMAX + 1):
        for lc in range(nat.LAUXMAX + 1):
            s0, s1, s2 = (nat.tile_shape(lab, lc, v) for v in range(3))
            assert s0["blocks_per_sm"] == 2 and s0["smem"] <= 110 * 1024 + 8192
            assert 2 * s1["tc"] >= s0["tc"] and s1["tc"] <= s0["tc"]
            busy = lambda s: min(s["tc"] * s["ub"] * s["lanes"], 256)
            assert busy(s1) >= busy(s0)
            if s2["blocks_per_sm"] == 3:
                assert lab + lc > 5 and s2["smem"] <= 72 * 1024 + 8192
            else:
                assert s2 == s0 or lab + lc <= 5
    assert nat.tile_shape(4, 3, 1)["tc"] == 16 and nat.tile_shape(4, 3, 1)["lanes"] == 16


def test_committed_table_parses():
    if tune.DEFAULT_TABLE.exists():
        table = tune.parse_table(tune.DEFAULT_TABLE.read_text())
        assert all(0 <= v < nat.TILE_VARIANTS for v in table.values())
        assert all(0 <= a <= 2 * nat.LMAX and 0 <= b <= nat.LAUXMAX for a, b in table)
