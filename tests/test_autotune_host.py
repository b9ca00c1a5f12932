"""The autotuner's JSON cache (KCFD_TUNE_CACHE) on the host: written atomically, read back,
and a corrupt file ignored. No device call."""


def test_tune_cache_round_trip(tmp_path, monkeypatch):
    from kcfd import autotune
    path = tmp_path / "tune.json"
    monkeypatch.setenv("KCFD_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "_CACHE", {"10:50:1:jacobi:0:1": {"lanes": 2, "block": 256, "ms": 0.5}})
    autotune._save()
    assert path.exists() and not list(tmp_path.glob("*.tmp"))
    monkeypatch.setattr(autotune, "_CACHE", {})
    autotune._load()
    assert autotune._CACHE == {"10:50:1:jacobi:0:1": {"lanes": 2, "block": 256, "ms": 0.5}}
    path.write_text("{not json")
    monkeypatch.setattr(autotune, "_CACHE", {})
    autotune._load()
    assert autotune._CACHE == {}
