"""Host logic of the autotuner: the search, the cache key and the cache file (no GPU)."""

from __future__ import annotations

import json
import math

import pytest

from gradient_domain_b200 import autotune
from gradient_domain_b200.plan import Instance, SolveParams

START = {name: values[0] for name, values in autotune.SPACE}


def test_coordinate_descent_finds_the_separable_optimum_and_evaluates_each_once():
    target = {"sweeps": 3, "strip_target_warps": 900, "tile_cells": 1048576, "bottom_cells": 4096}
    calls = []

    def cost(choice):
        calls.append(tuple(sorted(choice.items())))
        return 10.0 + sum(0.0 if choice[k] == v else 1.0 for k, v in target.items())

    best, best_cost, history = autotune.coordinate_descent(cost, START)
    assert best == target and best_cost == 10.0
    assert len(calls) == len(set(calls)) == len(history)


def test_small_gains_and_failures_keep_the_defaults():
    def cost(choice):
        if choice["sweeps"] == 1:
            return math.inf                       # did not converge
        return 100.0 - (1.0 if choice["tile_cells"] == 65536 else 0.0)  # a 1 % gain

    best, best_cost, _ = autotune.coordinate_descent(cost, START, min_gain=0.02)
    assert best == START and best_cost == 100.0
    best, _, _ = autotune.coordinate_descent(cost, START, min_gain=0.005)
    assert best["tile_cells"] == 65536 and best["sweeps"] == 2


def test_keys_bucket_size_count_boundary_precision_and_device():
    k = autotune.tune_key([Instance(4096, 4096, "neumann", True)] * 3, device="B200")
    assert k == "neumann|cells~2^24|n<=4|mixed|B200"
    assert autotune.tune_key([Instance(1000, 1000)], device="B200") == \
        "dirichlet|cells~2^20|n<=1|mixed|B200"
    mixed = autotune.tune_key([Instance(64, 64, "masked"), Instance(128, 128, "neumann")],
                              SolveParams(precision="fp64"), device="H100")
    assert mixed == "masked+neumann|cells~2^14|n<=2|fp64|H100"
    assert autotune.tune_key([Instance(8, 8)]).endswith("|" + autotune.device_name())
    with pytest.raises(ValueError):
        autotune.tune_key([])


def test_an_entry_timed_on_another_device_is_ignored(tmp_path):
    path = str(tmp_path / "tune.json")
    insts = [Instance(128, 128, "neumann", True)]
    key = autotune.tune_key(insts)
    autotune._store(path, key, {"choice": {"sweeps": 3}, "ms": 1.0, "default_ms": 2.0,
                                "device": "another GPU"})
    assert autotune.lookup(insts, SolveParams(), path) == SolveParams()


def test_cache_round_trip_and_lookup(tmp_path):
    path = str(tmp_path / "tune.json")
    insts = [Instance(512, 512, "neumann", True)] * 2
    params = SolveParams(tolerance=1e-6)
    assert autotune.lookup(insts, params, path) == params          # nothing cached yet
    key = autotune.tune_key(insts, params)
    choice = {"sweeps": 1, "strip_target_warps": 3600, "tile_cells": 65536, "bottom_cells": 1024}
    autotune._store(path, key, {"choice": choice, "ms": 1.0, "default_ms": 1.2})
    with open(path) as fh:
        assert json.load(fh)[key]["choice"] == choice
    got = autotune.lookup(insts, params, path)
    assert (got.sweeps, got.strip_target_warps, got.tile_cells, got.bottom_cells) == (1, 3600,
                                                                                      65536, 1024)
    assert got.tolerance == 1e-6                                    # other fields kept
    # a cached entry answers tune() without timing anything (no GPU needed)
    assert autotune.tune(insts, params, path=path) == got


def test_masked_instances_need_masks(tmp_path):
    with pytest.raises(ValueError):
        autotune.tune([Instance(64, 64, "masked")], path=str(tmp_path / "t.json"))


def test_a_tuned_precision_is_applied():
    got = autotune._apply(SolveParams(), {"sweeps": 1, "precision": "fp64"})
    assert got.precision == "fp64" and got.sweeps == 1
    assert autotune._apply(SolveParams(), {"precision": "bogus"}).value("precision") == "mixed"


def test_resolve_applies_tuned_values_only_where_the_caller_kept_defaults(tmp_path):
    path = str(tmp_path / "tune.json")
    insts = [Instance(256, 256, "neumann", True)]
    assert autotune.resolve(insts, SolveParams(), path) == SolveParams()   # nothing tuned
    key = autotune.tune_key(insts, SolveParams())
    choice = {"sweeps": 3, "strip_target_warps": 900, "tile_cells": 65536, "bottom_cells": 1024,
              "precision": "fp64"}
    autotune._store(path, key, {"choice": choice, "ms": 1.0, "default_ms": 1.1})
    got = autotune.resolve(insts, SolveParams(tolerance=1e-6, zero_start=True), path)
    assert (got.sweeps, got.strip_target_warps, got.tile_cells, got.bottom_cells,
            got.precision) == (3, 900, 65536, 1024, "fp64")
    assert got.tolerance == 1e-6 and got.zero_start
    mine = autotune.resolve(insts, SolveParams(sweeps=1, tile_cells=262144), path)
    assert mine.sweeps == 1 and mine.tile_cells == 262144 and mine.strip_target_warps == 900
    # an explicit value equal to the default is the caller's choice too
    same = autotune.resolve(insts, SolveParams(sweeps=2, precision="mixed"), path)
    assert same.sweeps == 2 and same.precision == "mixed" and same.bottom_cells == 1024


def test_untuned_keys_are_read_from_the_file_once(tmp_path, monkeypatch):
    path = str(tmp_path / "tune.json")
    reads = []
    real = autotune._load
    monkeypatch.setattr(autotune, "_load", lambda p: reads.append(p) or real(p))
    insts = [Instance(96, 80, "dirichlet")]
    for _ in range(3):
        assert autotune.resolve(insts, SolveParams(), path) == SolveParams()
    assert len(reads) == 1
