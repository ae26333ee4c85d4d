"""Autotuner search and cache (host logic; the GPU timing itself is exercised
by the bench's tiled leg)."""
import json

import pytest

from terawarp_b200 import autotune


def test_tune_picks_the_fastest_candidate_best_of_repeats():
    calls = []
    times = {((512, 512, 512), 2): [0.30, 0.20], ((1024, 1024, 256), 3): [0.25, 0.26], ((256, 256, 256), 4): [0.5, 0.4]}

    def run(tile, depth):
        k = (tile, depth)
        calls.append(k)
        return times[k][sum(1 for c in calls if c == k) - 1]

    tile, depth, table = autotune.tune(run, list(times), repeats=2)
    assert (tile, depth) == ((512, 512, 512), 2)  # best-of-2: 0.20 beats 0.25
    assert [t[2] for t in table] == [0.20, 0.25, 0.4]
    assert len(calls) == 6


def test_tune_rejects_an_empty_candidate_list():
    with pytest.raises(ValueError):
        autotune.tune(lambda t, d: 1.0, [])


def test_cache_key_buckets_landmark_counts():
    k1 = autotune.cache_key("tps", (512, 2048, 2048), "u16", 16, 1500, "B200")
    k2 = autotune.cache_key("tps", (512, 2048, 2048), "u16", 16, 2000, "B200")
    k3 = autotune.cache_key("tps", (512, 2048, 2048), "u16", 16, 2049, "B200")
    assert k1 == k2 != k3
    assert k1 == "tps:2048x2048x512:u16:g16:n2048:B200"


def test_cache_round_trip(tmp_path):
    p = tmp_path / "sub" / "autotune.json"
    assert autotune.load_cache(p) == {}
    table = [((512, 512, 512), 2, 0.2), ((1024, 1024, 256), 3, 0.25)]
    autotune.store_cache(p, "k", (512, 512, 512), 2, table)
    autotune.store_cache(p, "k2", (1024, 1024, 256), 3, table)
    data = json.loads(p.read_text())
    assert data["k"]["tile"] == [512, 512, 512] and data["k"]["depth"] == 2
    assert data["k2"]["table"][1] == [[1024, 1024, 256], 3, 0.25]


def test_tune_tiled_tps_returns_a_cached_choice_without_running(tmp_path):
    import numpy as np
    src = np.zeros((64, 128, 256), np.uint16)
    tar = np.zeros((100, 3), np.float32)
    key = autotune.cache_key("tps", src.shape, "u16", 16, 100, "B200")
    path = tmp_path / "a.json"
    autotune.store_cache(path, key, (256, 128, 64), 3, [((256, 128, 64), 3, 0.01)])
    tile, depth, table = autotune.tune_tiled_tps(None, tar, tar, 1.0, 16, src, cache_path=path, device_name="B200")
    assert (tile, depth) == ((256, 128, 64), 3)
    assert table == [((256, 128, 64), 3, 0.01)]
