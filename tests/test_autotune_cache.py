"""The autotuner's on-disk cache (no device needed): the key of a batch, and a
round trip through the cache file named by NPPB_AUTOTUNE_CACHE."""
import ctypes

import numpy as np

from numpp_b200 import _lib


def _key(L, n, k, flags):
    n = np.ascontiguousarray(n, np.int32)
    k = np.ascontiguousarray(k, np.int32)
    buf = ctypes.create_string_buffer(4096)
    assert L.nppb_autotune_key(len(n), n.ctypes.data, k.ctypes.data, flags, buf, 4096) == 0, _lib.last_error()
    return buf.value


def _get(L, key):
    c, ms, found = ctypes.c_int32(), ctypes.c_float(), ctypes.c_int32()
    assert L.nppb_autotune_cache_get(key, ctypes.byref(c), ctypes.byref(ms), ctypes.byref(found)) == 0
    return (c.value, ms.value) if found.value else None


def test_key_names_device_flags_and_class_histogram():
    L = _lib.load()
    a = _key(L, [8, 30, 100, 101, 500], [1, 8, 1, 1, 32], 7)
    # the same histogram over (order class, rhs class) in another order: same key
    assert _key(L, [101, 500, 8, 100, 30], [1, 32, 1, 1, 8], 7) == a
    # orders within the same class, counts within the same power of two: same key
    assert _key(L, [7, 29, 65, 120, 400], [1, 5, 1, 1, 20], 7) == a
    # other flags, another class, or a count past the next power of two: another key
    assert _key(L, [8, 30, 100, 101, 500], [1, 8, 1, 1, 32], 3) != a
    assert _key(L, [8, 30, 100, 101, 600], [1, 8, 1, 1, 32], 7) != a
    assert _key(L, [8, 30, 100, 101, 102, 103, 500], [1, 8, 1, 1, 1, 1, 32], 7) != a
    assert b"|f7" in a and a.count(b"|n") == 4


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "nested" / "autotune.txt"
    monkeypatch.setenv("NPPB_AUTOTUNE_CACHE", str(path))
    L = _lib.load()
    key = _key(L, [300] * 64, [1] * 64, 3)
    assert _get(L, key) is None
    assert L.nppb_autotune_cache_put(key, -3, 12.5) == 0, _lib.last_error()
    assert _get(L, key) == (-3, 12.5)
    assert L.nppb_autotune_cache_put(key, 2, 11.0) == 0
    assert _get(L, key) == (2, 11.0)  # the last line of a key wins
    other = _key(L, [30] * 64, [1] * 64, 3)
    assert _get(L, other) is None
    lines = path.read_text().splitlines()
    assert len(lines) == 2 and all(l.split("\t")[0] == key.decode() for l in lines)


def test_cache_disabled_by_empty_path(monkeypatch):
    monkeypatch.setenv("NPPB_AUTOTUNE_CACHE", "")
    L = _lib.load()
    key = _key(L, [64], [1], 3)
    assert L.nppb_autotune_cache_put(key, 1, 1.0) != 0
    assert _get(L, key) is None
