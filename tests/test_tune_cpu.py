"""The autotuner's table and cache file (host logic only, no device work): entries keyed by
device name and grid, a save/load round trip, malformed lines skipped, bad keys refused."""

from __future__ import annotations

import pytest

from omb200 import ops


def test_tune_table_round_trip(tmp_path):
    ops.tune_clear()
    ops.tune_set("NVIDIA B200", 256, 256, 4, 5, 3)
    ops.tune_set("NVIDIA B200", 128, 192, 0, 1)
    ops.tune_set("Other GPU", 256, 256, 1, 2, 1)
    assert ops.tune_get("NVIDIA B200", 256, 256) == (4, 5, 3)
    assert ops.tune_get("Other GPU", 256, 256) == (1, 2, 1)
    p = tmp_path / "sub" / "tiles.txt"
    ops.tune_save(str(p))
    lines = p.read_text().splitlines()
    assert len(lines) == 3 and all(line.count("|") == 6 for line in lines)
    ops.tune_clear()
    with pytest.raises(ops._lib.OmbError):
        ops.tune_get("NVIDIA B200", 256, 256)
    # a malformed line and out-of-range variants are skipped; a line without a wave field
    # (an older cache) reads as wave 0
    p.write_text(p.read_text() + "garbage line\nNVIDIA B200|64|64|7|0|0.1\nNVIDIA B200|32|32|1|1|0.1|9\n"
                 "NVIDIA B200|96|96|2|2|0.5\n")
    assert ops.tune_load(str(p)) == 4
    assert ops.tune_get("NVIDIA B200", 128, 192) == (0, 1, 0)
    assert ops.tune_get("NVIDIA B200", 96, 96) == (2, 2, 0)
    with pytest.raises(ops._lib.OmbError):
        ops.tune_get("NVIDIA B200", 64, 64)
    ops.tune_clear()


def test_tune_rejects_bad_entries():
    with pytest.raises(ops._lib.OmbError):
        ops.tune_set("NVIDIA B200", 256, 256, 7, 0)
    with pytest.raises(ops._lib.OmbError):
        ops.tune_set("NVIDIA B200", 256, 256, 1, 6)
    with pytest.raises(ops._lib.OmbError):
        ops.tune_set("", 256, 256, 1, 1)
    with pytest.raises(ops._lib.OmbError):
        ops.tune_set("NVIDIA B200", 256, 256, 1, 1, 4)
