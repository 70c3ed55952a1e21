"""Autotuner bookkeeping on the CPU: the best candidate wins, the choice is
cached per key in the JSON file and read back without measuring again."""
import json
import os

import pytest


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("FASTLPR_B200_CACHE", str(tmp_path / "autotune.json"))
    from fastlpr_b200 import autotune
    calls = []

    def measure(c):
        calls.append(c)
        return {1024: 3.0, 2048: 1.5, 4096: 2.0}[c["spread_item_points"]]

    cands = [{"spread_item_points": v} for v in (1024, 2048, 4096)]
    rec = autotune.tune("k1", cands, measure)
    assert rec["best"] == {"spread_item_points": 2048}
    assert len(calls) == 3 and len(rec["trials"]) == 3
    saved = json.load(open(tmp_path / "autotune.json"))
    assert saved["k1"]["best"] == {"spread_item_points": 2048}
    # cached: no measurement the second time
    rec2 = autotune.tune("k1", cands, lambda c: pytest.fail("measured again"))
    assert rec2["best"] == rec["best"]
    # force re-measures
    rec3 = autotune.tune("k1", cands, lambda c: 1.0 if c["spread_item_points"] == 4096 else 2.0,
                         force=True)
    assert rec3["best"] == {"spread_item_points": 4096}


def test_unwritable_cache_still_tunes(tmp_path, monkeypatch):
    target = tmp_path / "ro" / "autotune.json"
    os.makedirs(tmp_path / "ro")
    os.chmod(tmp_path / "ro", 0o500)
    monkeypatch.setenv("FASTLPR_B200_CACHE", str(target))
    from fastlpr_b200 import autotune
    try:
        rec = autotune.tune("k", [{"a": 1}, {"a": 2}], lambda c: float(c["a"]))
        assert rec["best"] == {"a": 1}
    finally:
        os.chmod(tmp_path / "ro", 0o700)
