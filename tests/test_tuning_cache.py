"""The autotuner's JSON cache (host side, no GPU)."""
from igap4standard_b200 import tuning


def test_store_and_load_roundtrip(tmp_path):
    p = str(tmp_path / "sub" / "tune.json")
    assert tuning.load(p) == {}
    tuning.store(p, "k1", {"residual_tile": 4})
    tuning.store(p, "k2", {"order": 1})
    d = tuning.load(p)
    assert d["k1"] == {"residual_tile": 4} and d["k2"] == {"order": 1}


def test_corrupt_cache_is_ignored(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    assert tuning.load(str(p)) == {}
