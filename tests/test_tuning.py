"""The persisted autotuner cache (zxh_adae_b200/tuning.py), on the CPU."""
import json

import pytest

from zxh_adae_b200.tuning import KNOBS, TuneCache, batch_key


def test_batch_key_shape():
    k = batch_key([10, 22, 15], "complex64", "NVIDIA B200", 148)
    assert k == "complex64|n10-22|c4|NVIDIA B200|sm148"
    assert batch_key([12] * 512, "complex128", "G", 8) == "complex128|n12-12|c512|G|sm8"
    assert batch_key([12] * 300, "complex128", "G", 8) == batch_key([12] * 512, "complex128", "G", 8)
    with pytest.raises(ValueError):
        batch_key([], "complex64", "G", 1)


def test_cache_round_trip_and_bad_files(tmp_path):
    path = tmp_path / "sub" / "tune.json"
    c = TuneCache(path)
    assert c.get("x") is None  # no file yet
    s = {"grow_regs": 3, "adj_regs": 2, "task_items": 512, "task_elems": 524288, "threads": 128}
    c.put("x", s)
    c.put("y", {**s, "threads": 64})
    assert c.get("x") == s and c.get("y")["threads"] == 64
    assert not list(path.parent.glob("*.tmp"))  # the temporary file was renamed over the cache
    assert set(json.loads(path.read_text())) == {"x", "y"}
    path.write_text("{ not json")
    assert TuneCache(path).get("x") is None and TuneCache(path).load() == {}
    path.write_text(json.dumps({"x": {"grow_regs": 3}}))  # missing knobs: not used
    assert TuneCache(path).get("x") is None
    assert set(KNOBS) == set(s)
