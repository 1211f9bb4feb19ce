"""The sweep autotuner's cache (CPU): size classes, the fallback rule,
recording the fastest lane count and reading it back per device and class."""

import json


def test_size_class_and_default():
    from sieb200 import autotune
    assert autotune.size_class([4000, 5000]) == 8192
    assert autotune.size_class([8192]) == 8192
    assert autotune.size_class([8193]) == 16384
    assert autotune.default_concurrency([4000]) == 4
    assert autotune.default_concurrency([12000]) == 3
    assert autotune.default_concurrency([24000]) == 2


def test_record_and_lookup(tmp_path, monkeypatch):
    from sieb200 import autotune
    monkeypatch.setattr(autotune, "device_name", lambda ctx=None: "TestGPU")
    path = tmp_path / "tune.json"
    assert autotune.sweep_concurrency([5000], path=path) == autotune.default_concurrency([5000])
    best = autotune.record([5000, 7000], {1: 3.0, 2: 1.7, 3: 1.9, 4: 2.2}, path=path)
    assert best == 2
    assert autotune.sweep_concurrency([6000], path=path) == 2  # same class (8192)
    assert autotune.sweep_concurrency([9000], path=path) == autotune.default_concurrency([9000])
    data = json.loads(path.read_text())
    assert data["TestGPU|sweep|8192"]["concurrency"] == 2
    # a second class is added without losing the first
    autotune.record([20000], {1: 5.0, 2: 4.0}, path=path)
    assert autotune.sweep_concurrency([5000], path=path) == 2
    assert autotune.sweep_concurrency([20000], path=path) == 2
    # another device does not see these entries
    monkeypatch.setattr(autotune, "device_name", lambda ctx=None: "OtherGPU")
    assert autotune.sweep_concurrency([5000], path=path) == autotune.default_concurrency([5000])
