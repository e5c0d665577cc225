"""Host side of the autotuner (master_b200/autotune.py): its JSON cache and
how a cached choice is found for a workload, without a GPU."""
from __future__ import annotations

import json

import pytest

from master_b200 import autotune


def test_cache_path_honours_the_environment(tmp_path, monkeypatch):
    monkeypatch.setenv("DSMC_TUNE_CACHE", str(tmp_path / "t.json"))
    assert autotune.cache_path() == tmp_path / "t.json"
    monkeypatch.delenv("DSMC_TUNE_CACHE")
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path / "xdg"))
    assert autotune.cache_path() == tmp_path / "xdg" / "dsmc_b200" / "tuning.json"


def test_cache_round_trip_and_unreadable_files(tmp_path, monkeypatch):
    p = tmp_path / "sub" / "tuning.json"
    monkeypatch.setenv("DSMC_TUNE_CACHE", str(p))
    assert autotune.load_cache() == {}          # no file yet
    entries = {"k": {"choice": {"blocks_per_sm": [0, 4, 0, 5, 0], "ring": 0, "collide_claim": 2}}}
    autotune.save_cache(entries)
    assert autotune.load_cache() == entries
    assert not p.with_suffix(".tmp").exists()   # written through a temporary file, then renamed
    p.write_text("{not json")
    assert autotune.load_cache() == {}


def test_signature_key_ignores_field_order():
    a = {"gpu": "NVIDIA B200", "sms": 148, "cells": 1 << 21, "particles": 1 << 25, "min_ring": 96, "pipelined": 1}
    b = dict(reversed(list(a.items())))
    assert autotune._key(a) == autotune._key(b)
    assert autotune._key(a) != autotune._key({**a, "sms": 132})


@pytest.mark.parametrize("x,want", [(0, 0), (-3, 0), (1, 1), (3, 4), (5, 4), (6, 8), (1000, 1024), (31_478_288, 1 << 25)])
def test_workload_sizes_round_to_powers_of_two(x, want):
    assert autotune._pow2(x) == want


def test_apply_cached_sets_the_stored_choice(tmp_path, monkeypatch):
    monkeypatch.setenv("DSMC_TUNE_CACHE", str(tmp_path / "tuning.json"))
    sig = {"gpu": "NVIDIA B200", "sms": 148, "cells": 4096, "particles": 1 << 19, "min_ring": 64, "pipelined": 1}
    choice = {"blocks_per_sm": [2, 4, 0, 5, 0], "ring": 128, "collide_claim": 1}
    autotune.save_cache({autotune._key(sig): {"choice": choice, "default_ms": {}, "chosen_ms": {}}})
    calls = []
    monkeypatch.setattr(autotune, "set_tuning", lambda ctx, bps, ring, claim: calls.append((ctx, bps, ring, claim)))
    monkeypatch.setattr(autotune, "signature", lambda ctx: dict(sig))
    ctx = object()
    entry = autotune.apply_cached(ctx)
    assert entry["choice"] == choice
    assert calls == [(ctx, choice["blocks_per_sm"], 128, 1)]
    # another workload: nothing cached, nothing set
    monkeypatch.setattr(autotune, "signature", lambda ctx: {**sig, "cells": 8192})
    assert autotune.apply_cached(ctx) is None
    assert len(calls) == 1
    assert json.loads((tmp_path / "tuning.json").read_text())  # the cache itself untouched
