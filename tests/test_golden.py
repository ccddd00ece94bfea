"""The oracle against its committed golden fixtures (tests/golden/make_golden.py).

These pin the oracle's restatement of the reference against regressions: the
seeded random streams, the Maclaurin roots, the pair table, the body builder,
the seat table and one scheduled step (bit for bit).  They are the oracle's
own outputs, not the reference's -- the reference cannot run here.
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_matches_its_golden_fixtures(orc):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import golden
    want = json.load(open(os.path.join(HERE, "golden", "oracle_golden.json")))
    got = json.loads(json.dumps(golden()))
    for key in want:
        assert got[key] == want[key], key
