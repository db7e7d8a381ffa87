"""Host logic of the tile-shape autotuner (autotune.tune) on CPU.

The knobs are the library's own registry (read and written through the C-ABI
with no device); the step time is a fake cost over the knob values, so the
coordinate descent, the margin rule, the per-workload cache and the
restoration of the knobs are checked without a GPU. The GPU test of the same
tuner on real steps is tests/test_autotune_gpu.py."""

import json

import pytest


@pytest.fixture()
def tuner(dpb, monkeypatch, tmp_path):
    from deepmd_kit_lr_pt_b200 import autotune

    monkeypatch.setenv("DPB_TUNE_CACHE", str(tmp_path / "tune.json"))
    # the cache key names the GPU; there is none here
    monkeypatch.setattr(autotune, "_key", lambda signature, device: f"cpu|{signature}")
    saved = autotune.current()
    yield autotune
    autotune.apply(saved)


def _fake_timer(autotune, cost):
    calls = []

    def time_step(run_step, reps=10, warmup=3, device=None):
        run_step()
        ms = cost(autotune.current())
        calls.append(ms)
        return ms

    return time_step, calls


def test_descent_finds_the_separable_optimum(tuner, monkeypatch):
    autotune = tuner
    knobs = ["desc_atoms_per_cta", "fit_n_tile"]
    want = {k: autotune.options(k)[-1] for k in knobs}
    start = {k: autotune.options(k)[0] for k in knobs}
    autotune.apply(start)

    def cost(v):  # 1 ms plus 0.2 ms per knob off its best option
        return 1.0 + sum(0.2 for k in knobs if v[k] != want[k])

    ts, calls = _fake_timer(autotune, cost)
    monkeypatch.setattr(autotune, "time_step", ts)
    recaptures = []
    res = tuner.tune(lambda: None, lambda: recaptures.append(1), knobs, signature="w1")
    assert res["knobs"] == want and not res["cached"]
    assert res["ms"] == pytest.approx(1.0) and res["baseline_ms"] == pytest.approx(1.4)
    assert autotune.current(knobs) == want  # left set
    # one timing per history entry, and the step captured again after each change
    assert len(res["history"]) == len(calls) and len(recaptures) >= len(calls)


def test_margin_keeps_the_incumbent(tuner, monkeypatch):
    """An option faster by less than the margin (1%) does not replace the
    current shape."""
    autotune = tuner
    k = "fit_n_tile"
    opts = autotune.options(k)
    autotune.set_knob(k, opts[0])
    ts, _ = _fake_timer(autotune, lambda v: 1.0 if v[k] == opts[0] else 0.995)
    monkeypatch.setattr(autotune, "time_step", ts)
    res = autotune.tune(lambda: None, lambda: None, [k], signature=None)
    assert res["knobs"][k] == opts[0] and autotune.get(k) == opts[0]


def test_cache_round_trip_applies_without_timing(tuner, monkeypatch, tmp_path):
    autotune = tuner
    knobs = ["desc_atoms_per_cta"]
    best = autotune.options(knobs[0])[-1]
    autotune.set_knob(knobs[0], autotune.options(knobs[0])[0])
    ts, calls = _fake_timer(autotune, lambda v: 1.0 if v[knobs[0]] == best else 2.0)
    monkeypatch.setattr(autotune, "time_step", ts)
    first = autotune.tune(lambda: None, lambda: None, knobs, signature="water-12288")
    n_timed = len(calls)
    stored = json.load(open(tmp_path / "tune.json"))
    assert stored["cpu|water-12288"]["knobs"] == {knobs[0]: best}
    # reset the knob; a second tune of the same workload reads the cache
    autotune.set_knob(knobs[0], autotune.options(knobs[0])[0])
    recaptured = []
    again = autotune.tune(lambda: None, lambda: recaptured.append(1), knobs,
                          signature="water-12288")
    assert again["cached"] and again["knobs"] == first["knobs"]
    assert len(calls) == n_timed and recaptured == [1]
    assert autotune.get(knobs[0]) == best
    # another knob set under the same signature is not a hit
    ts2, calls2 = _fake_timer(autotune, lambda v: 1.0)
    monkeypatch.setattr(autotune, "time_step", ts2)
    other = autotune.tune(lambda: None, lambda: None, ["fit_n_tile"], signature="water-12288")
    assert not other["cached"] and calls2
