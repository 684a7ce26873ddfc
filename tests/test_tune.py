"""The launch tuner's host logic (voluma_b200/tune.py): the candidate tail configurations of a
hierarchy, the size-class lookup, and the committed per-device table's shape."""
import json
import os

from voluma_b200 import tune


def test_candidates_split_levels_differently():
    levels = [2097152, 523326, 130427, 32489, 8072, 2002, 491, 120, 59]
    c = tune.candidates(levels)
    assert c and len(set(c)) == len(c)
    for cl, max_rows, full_rows in c:
        assert cl in (1, 2, 4, 8)
        # a row limit is a padded level size the cluster covers at four rows per thread at most
        assert max_rows <= 1024 * cl * 4 or full_rows > 1
    # the whole V-cycle in the tail only for systems that fit it
    assert all(full == 1 for _, _, full in c)
    small = tune.candidates([4096, 1024, 256, 64])
    assert any(full > 1 for _, _, full in small)


def test_lookup_takes_the_nearest_class_of_the_same_kind():
    entries = [dict(case="a", rows0=4096, nsys=1), dict(case="b", rows0=2097152, nsys=1),
               dict(case="c", rows0=1 << 20, nsys=8)]
    assert tune.lookup(entries, 3000, 1)["case"] == "a"
    assert tune.lookup(entries, 1_500_000, 1)["case"] == "b"
    assert tune.lookup(entries, 10_000_000, 4)["case"] == "c"
    assert tune.lookup([e for e in entries if e["nsys"] == 1], 100, 4) is None


def test_committed_table_shape():
    d = os.path.join(os.path.dirname(tune.__file__), "tuning")
    tables = [f for f in os.listdir(d) if f.endswith(".json")]
    assert tables
    for f in tables:
        t = json.load(open(os.path.join(d, f)))
        assert t["device"] and t["entries"]
        for e in t["entries"]:
            assert e["cluster"] in (1, 2, 4, 8) and e["max_rows"] >= 0 and e["full_rows"] >= 0
            assert e["ms"] <= e["default_ms"] * 1.001  # the kept configuration is never slower than the default
