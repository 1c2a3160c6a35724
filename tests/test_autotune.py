"""Tuning table plumbing of the autotuner (no device needed): keys, the
JSON round trip, and that set_tuning rejects out-of-range fields."""
import json

import pytest

import fknn
from fknn import autotune


def test_table_round_trip(tmp_path):
    path = str(tmp_path / "t.json")
    key = autotune.table_key("NVIDIA B200", 1_000_000, fknn.MODE_BF16_RERANK)
    assert key == "NVIDIA B200|n=1e6|mode=1"
    assert autotune.table_key("NVIDIA B200", 9_000_000, 1) == "NVIDIA B200|n=1e7|mode=1"
    entry = {"tuning": {"list_slack": 256, "items_per_sm": 3, "min_chunk_blocks": 8, "bound_refresh": 0,
                        "pilot_stride": 16}, "kprime": 200, "ms": 31.5, "recall": 0.999}
    autotune.save_entry(key, entry, path)
    autotune.save_entry("other", {"kprime": 0}, path)
    t = autotune.load_table(path)
    assert t[key] == entry and "other" in t
    assert json.load(open(path))[key]["kprime"] == 200


def test_missing_table_is_empty(tmp_path):
    assert autotune.load_table(str(tmp_path / "none.json")) == {}


def test_tuning_struct_matches_header():
    names = [f for f, _ in fknn._lib.Tuning._fields_]
    assert names == ["list_slack", "items_per_sm", "min_chunk_blocks", "bound_refresh", "pilot_stride"]
