"""Autotuner host logic (CPU): candidate choice, the cache file, the native
threshold setter.  The timed paths are covered in test_tune_gpu.py."""
import json

import numpy as np
import pytest

from ccsd_gpu_b200 import _native, tune


def test_pick_takes_the_fastest_and_breaks_ties_by_order():
    ran = []
    fake = {1: 5.0, 2: 3.0, 4: 3.0, 8: 9.0}
    timer = lambda fn: (fn(), fake[ran[-1]] * 3)[1]     # noqa: E731
    best, times = tune.pick([1, 2, 4, 8], ran.append, reps=3, timer=timer)
    assert best == 2 and times[4] == 3.0
    assert ran.count(8) == 4          # one untimed run and three timed runs per candidate


def test_cache_file_round_trip(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    monkeypatch.setenv("CCSD_B200_TUNE_CACHE", str(p))
    monkeypatch.setattr(tune, "_cache", None)
    monkeypatch.setattr(tune, "_have_gemm", False)
    tune._store("gemm:tf32x3:128:256:4096", 4)
    tune._store("eri:1:l2:p6:d0.6", 250)
    assert json.loads(p.read_text()) == {"eri:1:l2:p6:d0.6": 250, "gemm:tf32x3:128:256:4096": 4}
    monkeypatch.setattr(tune, "_cache", None)
    monkeypatch.setattr(tune, "_have_gemm", False)
    assert tune.cache()["eri:1:l2:p6:d0.6"] == 250
    assert tune.gemm_tuning_active()
    # a held split is used without timing, capped by the shape's chunk count
    assert tune.gemm_split(128, 256, 4096, "tf32x3", 1, 2, run=None) == 2


def test_eri_key_and_basis_dshare():
    bas = np.array([[0, 0, 3, 1, 0, 0, 0, 0], [0, 1, 2, 1, 0, 0, 0, 0], [0, 2, 1, 1, 0, 0, 0, 0],
                    [0, 0, 6, 1, 0, 0, 0, 0]])
    d = tune.basis_dshare(bas)
    assert abs(d - (1 - 0.75 ** 4)) < 1e-15
    assert tune.eri_key(bas, 1, d) == "eri:1:l2:p6:d0.7"


def test_native_heavy_threshold_setter():
    old = tune.get_heavy_nf(1)
    try:
        tune.set_heavy_nf(1, 321)
        assert tune.get_heavy_nf(1) == 321
        assert tune.get_heavy_nf(2) == -1
        with pytest.raises(_native.NativeError):
            tune.set_heavy_nf(1, 0)
        with pytest.raises(_native.NativeError):
            tune.set_heavy_nf(2, 100)
    finally:
        tune.set_heavy_nf(1, old)


def test_native_path_table_round_trip():
    old = [tune.get_paths(d) for d in (0, 1)]
    try:
        t = [(c * 7) % 3 for c in range(81)]
        tune.set_paths(1, t)
        assert tune.get_paths(1) == t
        assert tune.get_paths(0) == old[0]          # per derivative order
        with pytest.raises(_native.NativeError):
            tune.set_paths(1, [3] + [0] * 80)
        with pytest.raises(_native.NativeError):
            tune.set_paths(2, [0] * 81)
        assert tune.get_paths(1) == t               # a refused table changes nothing
    finally:
        for d in (0, 1):
            tune.set_paths(d, old[d])


def test_path_tuner_uses_a_held_table_without_timing(monkeypatch):
    bas = np.array([[0, 0, 3, 1, 0, 0, 0, 0], [0, 2, 2, 1, 0, 0, 0, 0]])
    monkeypatch.setattr(tune, "_cache", {})
    key = tune.eri_key(bas, 1, 0.5) + ":paths"
    held = "".join(str(c % 3) for c in range(81))
    tune.cache()[key] = held
    old = tune.get_paths(1)
    try:
        got = tune.tune_eri_paths(None, bas, None, 1, 0.5)      # no device work on this path
        assert "".join(map(str, got)) == held and tune.get_paths(1) == got
    finally:
        tune.set_paths(1, old)
