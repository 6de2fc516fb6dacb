"""Python-side helpers of the binding (no GPU): u128 results from ctypes
arrays, and per-graph method dicts to kc_params."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import kcgpu_b200 as kc  # noqa: E402
from kcgpu_b200._lib import KcU128  # noqa: E402


def test_u128_list():
    a = (KcU128 * 5)()
    for i in range(5):
        a[i].lo = 2**64 - 1 - i
    assert kc._u128_list(a, 5) == [2**64 - 1 - i for i in range(5)]
    a[2].hi = 7
    assert kc._u128_list(a, 5)[2] == (7 << 64) | (2**64 - 3)
    assert kc._u128_list(a, 0) == []


def test_params_from_dict():
    p = kc._params({"mode": "pivot", "unit": "edge", "part": 16, "encoding": "list"})
    assert (p.mode, p.unit, p.part, p.encoding) == (1, 1, 16, 1)
    p = kc._params({"mode": 2, "unit": 0})
    assert (p.mode, p.unit, p.part, p.encoding) == (2, 0, 0, 0)
