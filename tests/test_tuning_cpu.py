"""The GEMM autotuner's selection and its on-disk cache, with a fake timer (no GPU).

A candidate that misses the tolerance against the plain FP64 result is never chosen, the fastest
accepted one is, the record lands in the cache file under the structure key, and a second process
that opens the same file finds the record without measuring anything."""
import json
import os
import subprocess
import sys

import pytest

from tensorkit_b200 import tuning as T

BLOCKS = [(384, 256, 256, 0, 0, 0, 384, 256, 384, 0, 0), (576, 384, 384, 98304, 65536, 98304, 576, 384, 576, 0, 0)]


def test_structure_key_depends_on_shapes_ops_dtype_device():
    k = T.structure_key(BLOCKS, 0, "B200", 200)
    assert k == T.structure_key(BLOCKS, 0, "B200", 200)
    other = [tuple(b) for b in BLOCKS]
    other[1] = other[1][:9] + (1, 0)
    assert k != T.structure_key(other, 0, "B200", 200)  # an op differs
    assert k != T.structure_key(BLOCKS, 1, "B200", 200)
    assert k != T.structure_key(BLOCKS, 0, "H100", 200)
    assert k != T.structure_key(BLOCKS, 0, "B200", 100)
    # offsets and leading dimensions do not change the key (only shapes and ops do)
    shifted = [b[:3] + (b[3] + 8, b[4], b[5], b[6] + 2, b[7], b[8]) + b[9:] for b in BLOCKS]
    assert k == T.structure_key(shifted, 0, "B200", 200)


def test_select_rejects_inaccurate_and_keeps_fastest():
    us = {("plain", 8, 4): 30.0, ("plain", 1, 4): 40.0, ("split", 8, 4): 20.0, ("split", 1, 4): 10.0}
    err = {("split", 8, 4): 3e-13, ("split", 1, 4): 5e-12}  # the fastest misses 1e-12

    def measure(c):
        return us[c], (None if c[0] == "plain" and c == ("plain", 8, 4) else err.get(c, 1e-16))

    best, rec = T.select(list(us), measure)
    assert best == ("split", 8, 4)
    assert rec["timings"]["split/1/4"]["accepted"] is False
    assert rec["choice"] == ["split", 8, 4]


def test_select_raises_when_nothing_is_accurate():
    with pytest.raises(RuntimeError):
        T.select([("split", 8, 4)], lambda c: (1.0, 1.0))


def test_cache_round_trip_and_second_process(tmp_path):
    path = tmp_path / "tune.json"
    cache = T.TuneCache(str(path))
    key = T.structure_key(BLOCKS, 0, "B200", 200)
    calls = []

    def measure(c):
        calls.append(c)
        return (5.0 if c == ("split", 4, 8) else 9.0), (None if len(calls) == 1 else 1e-14)

    assert cache.get(key) is None
    best, rec = T.select(T.CANDIDATES, measure)
    cache.put(key, rec)
    assert len(calls) == len(T.CANDIDATES) and best == ("split", 4, 8)
    assert json.load(open(path))[key]["choice"] == ["split", 4, 8]
    # a second process reads the choice without measuring
    code = (
        "import sys; sys.path.insert(0, %r); from tensorkit_b200 import tuning as T; "
        "c = T.TuneCache(%r); r = c.get(%r); print(r['choice'])"
        % (os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tensorkit.jl_b200"),
           str(path), key))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    assert out.strip() == "['split', 4, 8]"
    # a second structure is added without losing the first
    key2 = T.structure_key(BLOCKS[:1], 0, "B200", 200)
    T.TuneCache(str(path)).put(key2, {"choice": ["plain", 8, 4], "timings": {}})
    data = json.load(open(path))
    assert set(data) == {key, key2}


def test_default_cache_path_from_environment(tmp_path, monkeypatch):
    monkeypatch.setenv("TKB_TUNE_CACHE", str(tmp_path / "x.json"))
    assert T.default_cache().path == str(tmp_path / "x.json")
