"""The built-in stage schedule table (gpurecsplit_b200/csrc/rsb_schedules.inc) is the one the
tuner measured (gpurecsplit_b200/schedules.json), and every entry is a valid schedule."""
import json
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "gpurecsplit_b200", "csrc", "rsb_schedules.inc")
JSON = os.path.join(ROOT, "gpurecsplit_b200", "schedules.json")


def _inc_entries():
    rows = re.findall(r"\{(\d+), (\d+), (\d+), (\d+), (\d+)\}", open(INC).read())
    return [tuple(int(x) for x in r) for r in rows]


def test_table_entries_are_valid():
    seen = set()
    for leaf, stage, cls, s, pct in _inc_entries():
        assert 2 <= leaf <= 24 and cls in (0, 1, 2) and 1 <= pct <= 100
        assert s in ((4, 8, 12, 16) if stage in (17, 18) else (4, 8, 12)) and stage in (17, 18, 19)
        assert (leaf, stage, cls) not in seen
        seen.add((leaf, stage, cls))


def test_table_matches_the_measurements():
    if not os.path.exists(JSON):
        pytest.skip("no tuning run recorded")
    entries = json.load(open(JSON))["entries"]
    want = sorted((e["leaf"], e["stage"], e["size_class"], e["seeds_per_lane"], e["occupancy_pct"]) for e in entries)
    assert sorted(_inc_entries()) == want
    for e in entries:
        if "copied_from_size_class" in e:
            continue
        chosen = f"{e['seeds_per_lane']}/{e['occupancy_pct']}"
        if "score" in e:  # measured at several sizes: least summed relative time
            assert e["score"][chosen] <= min(e["score"].values()) + 1e-9
        else:
            assert e["ms_best"] <= min(e["ms"].values()) + 1e-9


def test_tuner_choice_over_sizes():
    """A schedule that wins narrowly at the small end of a size class but loses clearly at its
    large end is not chosen; with one size the fastest is."""
    from gpurecsplit_b200.tune import choose
    small = {(4, 75): 0.0686, (12, 75): 0.0646, (8, 100): 0.0809}
    large = {(4, 75): 0.2099, (12, 75): 0.2735, (8, 100): 0.2325}
    best, score = choose([small, large])
    assert best == (4, 75) and score[(4, 75)] < score[(12, 75)]
    assert choose([small])[0] == (12, 75)
    assert abs(choose([small])[1][(12, 75)] - 1.0) < 1e-12
