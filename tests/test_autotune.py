"""The sweep autotuner's bucketing, feasibility and on-disk cache."""

import json

from momwire_b200 import autotune


def test_bucket_and_feasible():
    assert autotune.bucket(1) == 32 and autotune.bucket(33) == 64 and autotune.bucket(432) == 512
    assert autotune.feasible(400) == [8, 16, 32]
    assert autotune.feasible(1000) == [8, 16]
    assert autotune.feasible(5000) == []


def test_choose_times_once_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("MOMWIRE_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_cache", None)
    calls = []

    def fake(w):
        calls.append(w)
        return {8: 3.0, 16: 1.0, 32: 2.0}[w]

    assert autotune.choose(400, 2, "free", fake) == 16
    assert calls == [8, 16, 32]
    assert autotune.choose(450, 2, "free", fake) == 16  # same bucket: cached
    assert calls == [8, 16, 32]
    saved = json.loads((tmp_path / "tune.json").read_text())
    assert saved[autotune.key(400, 2, "free")]["width"] == 16
    monkeypatch.setattr(autotune, "_cache", None)  # a new process reads the file
    assert autotune.choose(500, 2, "free", lambda w: 1 / 0) == 16


def test_disabled_uses_default(monkeypatch):
    monkeypatch.setenv("MOMWIRE_B200_AUTOTUNE", "0")
    assert autotune.choose(400, 2, "free", lambda w: 1 / 0) == autotune.DEFAULT_WIDTH
