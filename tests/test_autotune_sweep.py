"""Host side of the measured autotuner (kcgpu_b200/autotune_sweep.py): the
bucket bands, the method names and the generated table header, which must
compile and agree with the committed sweep record. CPU only."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from kcgpu_b200 import autotune_sweep as S  # noqa: E402


def test_bands_and_buckets():
    assert S.band(3, S.K_BANDS) == 0 and S.band(5, S.K_BANDS) == 0
    assert S.band(6, S.K_BANDS) == 1 and S.band(12, S.K_BANDS) == 2
    assert S.band(32, S.OUT_BANDS) == 0 and S.band(33, S.OUT_BANDS) == 1 and S.band(10**6, S.OUT_BANDS) == 4
    # density 2m / (n (n - 1))
    assert S.bucket_of(4, 10, 100, 10) == (0, 0, 0)
    assert S.bucket_of(9, 100, 100, 495) == (2, 2, 2)  # density 0.1
    assert S.bucket_of(7, 40, 1000, 10_000) == (1, 1, 1)  # density 0.02


def test_method_names_round_trip():
    names = [S.spec_name(*m) for m in S.methods()]
    assert len(names) == len(set(names)) == len(S.MODES) * len(S.UNITS) * len(S.PARTS) * len(S.ENCS)
    assert S.spec_name("auto", "node", 0, "bitmap") == "aAb-node"
    assert S.spec_name("pivot", "edge", 32, "list") == "p32n-edge"


def test_generated_header_compiles(tmp_path):
    table = {(0, 0, 0): ("pivot", "node", 32, "bitmap"), (2, 4, 2): ("orient", "edge", 4, "list")}
    h = tmp_path / "t.h"
    S.write_header(table, h, "test table")
    src = tmp_path / "t.cpp"
    src.write_text('#include "t.h"\n'
                   'static_assert(kc::tune::kTable[0][0][0].valid == 1 && kc::tune::kTable[0][0][0].mode == 1 &&\n'
                   '              kc::tune::kTable[0][0][0].part == 32, "entry");\n'
                   'static_assert(kc::tune::kTable[2][4][2].unit == 1 && kc::tune::kTable[2][4][2].encoding == 1, "entry");\n'
                   'static_assert(kc::tune::kTable[1][1][1].valid == 0, "empty bucket");\n'
                   'int main() { return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-I", str(tmp_path), "-c", str(src), "-o", str(tmp_path / "t.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_committed_table_matches_the_sweep_record():
    rec_path = ROOT / "kcgpu_b200" / "autotune_sweep.json"
    if not rec_path.exists():
        pytest.skip("no sweep record committed")
    rec = json.loads(rec_path.read_text())
    header = (ROOT / "kcgpu_b200" / "csrc" / "autotune_table.h").read_text()
    assert rec["decision"] in header
    # every bucket of the record's engine table is in the header with its method
    entries = []
    for ln in header.splitlines():
        s = ln.strip()
        if s.startswith("{{") or s.startswith("{0,") or s.startswith("{1,"):
            row = s.strip("{},").split("}, {")
            entries.append([tuple(int(x) for x in e.strip("{} ,").split(",")) for e in row])
    nk, no, nd = len(S.K_BANDS), len(S.OUT_BANDS), len(S.DENS_BANDS)
    assert len(entries) == nk * no
    for key, name in rec["engine_table"].items():
        a, b, c = json.loads(key)
        valid, mode, unit, part, enc = entries[a * no + b][c]
        assert valid == 1
        assert S.spec_name(["orient", "pivot", "auto"][mode], ["node", "edge"][unit], part,
                           ["bitmap", "list"][enc]) == name
