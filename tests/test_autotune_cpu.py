"""CPU checks of the autotuner's host logic (no GPU): how a knob is picked
from timed candidates, including the re-timing of two close candidates, and
that the committed table's choices reach every setter of a context."""
from __future__ import annotations

import itertools
import json

from marigold_b200 import autotune


def make_trial(times, key, log):
    """A trial function that returns the next scripted time of each value."""
    streams = {v: iter(ts) for v, ts in times.items()}

    def trial(**change):
        v = change[key]
        ms = next(streams[v])
        log.append((v, ms))
        return {key: v, "ms": ms}

    return trial


def test_clear_winner_is_timed_once():
    log = []
    best = {"x": None}
    trial = make_trial({1: [10.0], 2: [20.0], 3: [30.0]}, "x", log)
    top = autotune.pick_knob(trial, best, "x", (1, 2, 3))
    assert best["x"] == 1 and top["x"] == 1
    assert [v for v, _ in log] == [1, 2, 3]


def test_close_pair_is_retimed_in_turn_and_the_lower_mean_wins():
    # value 2 is fastest in the first pass by luck; in the re-timings
    # value 1 is faster, and its mean is lower
    log = []
    best = {"x": None}
    trial = make_trial({1: [10.1, 9.9, 9.9, 9.9], 2: [10.0, 10.3, 10.3, 10.3], 3: [20.0]}, "x", log)
    top = autotune.pick_knob(trial, best, "x", (1, 2, 3))
    assert best["x"] == 1 and top["x"] == 1
    retimes = log[3:]
    assert len(retimes) == 2 * autotune.CONFIRM
    # in turn: the first pass's leader, then the runner-up
    assert [v for v, _ in retimes] == [2, 1] * autotune.CONFIRM


def test_close_pair_keeps_the_leader_when_it_stays_ahead():
    log = []
    best = {"x": None}
    trial = make_trial({1: [10.0, 10.0, 10.0, 10.0], 2: [10.2, 10.2, 10.2, 10.2]}, "x", log)
    autotune.pick_knob(trial, best, "x", (1, 2))
    assert best["x"] == 1


def test_pairs_further_apart_than_close_are_not_retimed():
    log = []
    best = {"x": None}
    far = 10.0 * autotune.CLOSE * 1.01
    trial = make_trial({1: [10.0], 2: [far]}, "x", log)
    autotune.pick_knob(trial, best, "x", (1, 2))
    assert best["x"] == 1 and len(log) == 2


class FakeContext:
    def __init__(self):
        self.calls = {}

    def set_tuning(self, medium_max):
        self.calls["medium_max"] = medium_max

    def set_launch_shape(self, small_threads, queue_ctas_per_sm):
        self.calls["small_threads"] = small_threads
        self.calls["queue_ctas_per_sm"] = queue_ctas_per_sm

    def set_small_occupancy(self, warps_per_sm):
        self.calls["small_warps"] = warps_per_sm

    def set_batch_mode(self, queue):
        self.calls["batch_mode"] = "queue" if queue else "levels"


def test_apply_sets_every_speed_knob_of_the_committed_table():
    with open(autotune.TABLE) as f:
        table = json.load(f)
    assert set(table) >= {"icosphere_l8", "batched_scene"}
    for name, entry in table.items():
        ctx = FakeContext()
        chosen = autotune.apply(ctx, name)
        for k in ("medium_max", "small_threads", "small_warps", "batch_mode", "queue_ctas_per_sm"):
            assert ctx.calls[k] == entry["choice"].get(k, autotune.DEFAULTS[k]), (name, k)
        assert chosen["bins"] == entry["choice"].get("bins", 0)
        # every choice is a value the tuner offers
        assert chosen["medium_max"] in autotune.MEDIUM_MAX
        assert chosen["small_threads"] in autotune.SMALL_THREADS
        assert chosen["small_warps"] in autotune.SMALL_WARPS


def test_apply_falls_back_to_defaults_for_an_unknown_workload():
    ctx = FakeContext()
    chosen = autotune.apply(ctx, "no_such_workload")
    for k, v in autotune.DEFAULTS.items():
        assert chosen[k] == v
    assert ctx.calls["small_warps"] == autotune.DEFAULTS["small_warps"]


def test_table_rows_record_the_knobs_they_timed():
    with open(autotune.TABLE) as f:
        table = json.load(f)
    for name, entry in table.items():
        for row in entry["candidates"]:
            for k in itertools.chain(autotune.DEFAULTS, ("ms", "sah")):
                assert k in row, (name, k)
