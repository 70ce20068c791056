"""Stage schedules (rsb_engine_set_schedule, the table gpurecsplit_b200/tune.py writes): every
schedule - candidates per lane of a window, occupancy share - builds the same function, since
each search returns the minimum seed whatever the window size; invalid schedules are refused,
and an engine reports the built-in (tuned) schedule until it is overridden."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AGGR = (4, 8, 12, 16)
LEAF = (4, 8, 12)


@pytest.mark.parametrize("leaf,b,n", [(4, 25, 20_000), (8, 100, 60_000), (12, 1000, 60_000), (16, 2000, 8_000),
                                      (20, 2000, 400)])
def test_every_schedule_builds_the_same_function(rsb, oracle_mod, leaf, b, n):
    keys = oracle_mod.keygen_hash128(4242 + leaf, n)
    e = rsb.Engine(0)
    try:
        want = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=e).serialize()
        assert want == oracle_mod.build_mphf(keys, leaf, b).bytes.tobytes()
        for s17, s18, s19 in itertools.product(AGGR, AGGR, LEAF):
            if len({s17, s18}) > 1 and s19 != 8:
                continue  # every value of every stage, without the full product
            for st, s in ((17, s17), (18, s18), (19, s19)):
                e.set_schedule(leaf, st, 0, s, 100 if s19 != 4 else 60)
            got = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=e).serialize()
            assert got == want, (s17, s18, s19)
    finally:
        e.close()


def test_schedule_arguments(rsb):
    e = rsb.Engine(0)
    try:
        builtin = e.schedule(16, 18, 1)
        assert builtin[0] in AGGR and 1 <= builtin[1] <= 100
        e.set_schedule(16, 18, 1, 16, 90)
        assert e.schedule(16, 18, 1) == (16, 90)
        e.set_schedule(16, 18, 1, 0)
        assert e.schedule(16, 18, 1) == builtin
        e.set_schedule(16, 18, 2, 8, 75)  # size classes are separate entries
        assert e.schedule(16, 18, 2) == (8, 75) and e.schedule(16, 18, 1) == builtin
        lower0 = e.schedule(16, 18, 0)
        e.set_schedule(16, 17, 2, 16, 60)  # the entry of stage 17, class 2 is not stage 18's
        assert e.schedule(16, 17, 2) == (16, 60) and e.schedule(16, 18, 0) == lower0
        for args in ((16, 18, 1, 6, 100), (16, 19, 1, 16, 100), (16, 18, 3, 8, 100), (16, 20, 0, 8, 100),
                     (1, 18, 0, 8, 100), (16, 18, 0, 8, 0), (16, 18, 0, 8, 101)):
            with pytest.raises(rsb.RSBError) as err:
                e.set_schedule(*args)
            assert err.value.name == "BAD_ARG"
    finally:
        e.close()
