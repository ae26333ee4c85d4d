"""The tiled autotuner's cache (tw_tune_tiled_tps consulted without a
context: CPU only).  Choices are keyed by volume dims, dtype, grid spacing,
the landmark count rounded up to a power of two, and the device name; the
last line of a key in the cache file wins."""
import numpy as np

from terawarp_b200 import autotune


def write_cache(path, lines):
    path.write_text("".join(l + "\n" for l in lines))


def test_cached_choice_from_the_file(tmp_path):
    p = tmp_path / "tune.txt"
    write_cache(p, ["tps:256x128x64:u16:g16:n128: 256 128 64 3 0.01",
                    "tps:256x128x64:u8:g16:n128: 128 128 64 2 0.02"])
    assert autotune.cached_choice((64, 128, 256), np.uint16, 16, 100, p) == ((256, 128, 64), 3)
    assert autotune.cached_choice((64, 128, 256), np.uint8, 16, 100, p) == ((128, 128, 64), 2)


def test_landmark_counts_share_a_power_of_two_bucket(tmp_path):
    p = tmp_path / "tune.txt"
    write_cache(p, ["tps:2048x2048x512:u16:g16:n2048: 1024 1024 256 3 0.5"])
    assert autotune.cached_choice((512, 2048, 2048), np.uint16, 16, 1500, p) == ((1024, 1024, 256), 3)
    assert autotune.cached_choice((512, 2048, 2048), np.uint16, 16, 2048, p) == ((1024, 1024, 256), 3)
    assert autotune.cached_choice((512, 2048, 2048), np.uint16, 16, 2049, p) is None
    assert autotune.cached_choice((512, 2048, 2048), np.uint16, 8, 2000, p) is None


def test_last_line_of_a_key_wins_and_misses_report_none(tmp_path):
    p = tmp_path / "tune.txt"
    write_cache(p, ["tps:64x64x64:u16:g8:n16: 64 64 64 2 0.3",
                    "tps:64x64x64:u16:g8:n16: 64 64 32 4 0.2"])
    assert autotune.cached_choice((64, 64, 64), np.uint16, 8, 16, p) == ((64, 64, 32), 4)
    assert autotune.cached_choice((64, 64, 65), np.uint16, 8, 16, p) is None
    # a choice once made is remembered by the process, file or not
    assert autotune.cached_choice((64, 64, 64), np.uint16, 8, 16, tmp_path / "absent.txt") == ((64, 64, 32), 4)
    assert autotune.cached_choice((96, 64, 64), np.uint16, 8, 16, tmp_path / "absent.txt") is None
