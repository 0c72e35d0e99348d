"""The autotuner's host logic on the CPU: the knob table in the library
(set / get, illegal values rejected), the JSON cache, and the search picking
the cheapest setting of a synthetic cost model."""

import pytest


@pytest.fixture
def tune_mod(monkeypatch, tmp_path):
    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import autotune

    try:
        L.lib()
    except Exception as e:  # pragma: no cover - library not built
        pytest.skip(f"libygx.so not loadable: {e}")
    monkeypatch.setenv("YGGDRAX_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    saved = autotune.current()
    yield autotune
    autotune.apply(saved)


def test_knob_table_roundtrip(tune_mod):
    from yggdrax_b200 import _lib as L

    tune_mod.apply({"walk_blocks": 4, "row_grid": 8, "sort_rank": 2, "sort_skew": 100,
                    "sort_tile": 3, "sort_bits": 11})
    cur = tune_mod.current()
    assert cur["sort_bits"] == 11
    assert cur["walk_blocks"] == 4 and cur["row_grid"] == 8 and cur["sort_tile"] == 3
    assert cur["sort_rank"] == 2 and cur["sort_skew"] == 100
    for knob, bad in (("walk_blocks", 1), ("walk_blocks", 7), ("refit_warps", 3),
                      ("row_grid", 12), ("sort_rank", 3), ("sort_skew", 0), ("sort_skew", 257),
                      ("sort_tile", -1), ("sort_tile", 4), ("sort_bits", 9),
                      ("sort_bits", 16)):
        with pytest.raises(ValueError):
            tune_mod.apply({knob: bad})
        assert tune_mod.current()[knob] == cur[knob]
    with pytest.raises(ValueError):
        tune_mod.apply({"no_such_knob": 1})
    assert L.lib().ygx_tune_get(99, None) == 1


def test_search_finds_cheapest_setting(tune_mod, monkeypatch):
    # synthetic cost: best at 11-bit digits, walk_blocks=4, refit_warps=2, row_grid=32
    def cost():
        c = tune_mod.current()
        return (10.0 + abs(c["walk_blocks"] - 4) + (c["refit_warps"] != 2) * 0.5
                + (32 - c["row_grid"]) * 0.01 + (c["sort_bits"] == 8) * 0.3)

    monkeypatch.setattr(tune_mod, "time_ms", lambda fn, dev, reps=3, warmup=1: cost())
    tune_mod.apply({"walk_blocks": 6, "refit_warps": 8, "row_grid": 16, "sort_bits": 8})
    log = []
    best = tune_mod.tune(lambda: None, None, log=log)
    assert (best["walk_blocks"], best["refit_warps"], best["row_grid"]) == (4, 2, 32)
    assert best["sort_bits"] == 11
    assert tune_mod.current() == best
    assert len(log) == 1 + 1 + 3 + 2 + 3


def test_sort_stage_tunes_the_8_bit_pass_and_leaves_the_width_to_the_step(tune_mod,
                                                                           monkeypatch):
    # synthetic costs: the sort alone is cheapest at ranking 1 / tile shape 2;
    # the whole step is cheapest with 11-bit digits
    stage = {"now": "sort"}
    seen_bits = []

    def cost():
        c = tune_mod.current()
        if stage["now"] == "sort":
            seen_bits.append(c["sort_bits"])
            return 1.0 + (c["sort_rank"] != 1) * 0.2 + (c["sort_tile"] != 2) * 0.1
        return 10.0 + (c["sort_bits"] == 8) * 0.5

    def sort_step(codes, dev):
        stage["now"] = "sort"
        return lambda: None

    def step():
        pass

    def timed(fn, dev, reps=3, warmup=1):
        if fn is step:
            stage["now"] = "step"
        return cost()

    monkeypatch.setattr(tune_mod, "_sort_step", sort_step)
    monkeypatch.setattr(tune_mod, "time_ms", timed)
    tune_mod.apply({"sort_rank": 2, "sort_tile": 0, "sort_bits": 11})
    log = []
    best = tune_mod.tune(step, None, codes=object(), knobs=("sort_bits",), log=log)
    assert best["sort_rank"] == 1 and best["sort_tile"] == 2
    assert best["sort_bits"] == 11  # chosen on the step
    assert seen_bits and set(seen_bits) == {8}  # the sort stage measures the 8-bit pass
    assert tune_mod.current() == best
    assert [r["stage"] for r in log].count("sort") == len(seen_bits)


def test_cache_roundtrip(tune_mod, monkeypatch):
    calls = []
    monkeypatch.setattr(tune_mod, "tune",
                        lambda step, dev, **kw: calls.append(1) or dict(tune_mod.current(),
                                                                        walk_blocks=3))
    cfg = tune_mod.tuned("dev|kind|n2^20|leaf=16", lambda: None, None)
    assert cfg["walk_blocks"] == 3 and len(calls) == 1
    tune_mod.apply({"walk_blocks": 6})
    cfg2 = tune_mod.tuned("dev|kind|n2^20|leaf=16", lambda: None, None)
    assert cfg2["walk_blocks"] == 3 and len(calls) == 1  # from the cache
    assert tune_mod.current()["walk_blocks"] == 3
