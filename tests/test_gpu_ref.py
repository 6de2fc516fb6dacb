"""The engine against the reference's own build (tests/golden/ref_counts.json).

Each fixture run is repeated through the C ABI with the same method: unit,
orientation or pivoting, partition size, encoding, graph orientation and k.
Where the reference counts exactly (every run outside tests/ref_rules.py's
deviations: all node-unit methods and most edge-unit ones) the engine must
print the same number; under a deviation the engine must give the exact
count, which the oracle supplies.
"""
import sys
from pathlib import Path

import pytest

import kcgpu_b200 as kc
from oracle.oracle import OracleGraph
from tests import ref_rules as R

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import ref_graphs as RG  # noqa: E402

pytestmark = pytest.mark.gpu


def test_engine_matches_reference_build(ctx):
    fx = R.load_fixture()
    runs = {}
    for r in fx["runs"]:
        runs.setdefault((r["graph"], r["orient"]), []).append(r)
    same = exact = 0
    for (name, orient), rs in sorted(runs.items()):
        s, d, n = RG.make(name)
        assert RG.sha(s, d) == fx["graphs"][name]["sha256"]
        og = OracleGraph(s, d, n)
        og.orient(orient)
        with kc.Graph.from_edges(ctx, s, d, n) as g:
            g.orient(orient)
            for r in rs:
                mode, part, enc = R.parse_spec(r["spec"])
                k = int(r["k"])
                got = g.count(k, mode=mode, unit=r["unit"], part=part, encoding=enc)
                if R.rule(r) is None:
                    assert got == int(r["count"]), (name, orient, r)
                    same += 1
                else:
                    assert got == og.count(k, "pivot", closed=True), (name, orient, r)
                    exact += 1
    assert same == 514 and exact == 270
