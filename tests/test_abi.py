"""The C ABI library: loads without a GPU, exports every declared symbol, and
its host-only entry points (spec parsing, generators, footprint model) behave."""
import re
from pathlib import Path

import numpy as np
import pytest

import kcgpu_b200 as kc
from kcgpu_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(kc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = kc.lib()
    names = declared_functions()
    assert len(names) >= 35
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) == names


def test_parse_spec_reference_grammar():
    # include/Config.h:235-271: defaults o8b; 'p' first -> pivoting; digits -> partition; 'n' -> list
    assert kc.parse_spec("o8b") == {"mode": 0, "part": 8, "encoding": 0}
    assert kc.parse_spec("p16n") == {"mode": 1, "part": 16, "encoding": 1}
    assert kc.parse_spec("o1b") == {"mode": 0, "part": 1, "encoding": 0}
    assert kc.parse_spec("p32b") == {"mode": 1, "part": 32, "encoding": 0}
    assert kc.parse_spec("o4h") == {"mode": 0, "part": 4, "encoding": 0}  # 'h' is parsed but unused upstream
    assert kc.parse_spec("") == {"mode": 0, "part": 8, "encoding": 0}
    assert kc.parse_spec("p") == {"mode": 0, "part": 8, "encoding": 0}  # length <= 2 keeps defaults
    for bad in ("o3b", "p0b", "o64b", "oxb"):
        with pytest.raises(kc.KCError) as e:
            kc.parse_spec(bad)
        assert e.value.name == "KC_ERR_INVALID_ARG"


def test_context_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(kc.KCError) as e:
        kc.Context(0)
    assert e.value.name in ("KC_ERR_CUDA", "KC_ERR_INVALID_ARG")
    assert kc.lib().kc_last_error()


def test_generators_are_seeded_and_shaped():
    a = kc.gen_er(2000, 0.01, 1).arrays()
    b = kc.gen_er(2000, 0.01, 1).arrays()
    c = kc.gen_er(2000, 0.01, 2).arrays()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not (a[0].size == c[0].size and np.array_equal(a[0], c[0]))
    n_pairs = 2000 * 1999 / 2
    assert abs(a[0].size - 0.01 * n_pairs) < 6 * np.sqrt(0.01 * n_pairs)
    assert np.all(a[0] > a[1])  # pairs are emitted as (larger, smaller)
    s, d, n = kc.gen_rmat(10, 16, seed=1).arrays()
    assert n == 1024 and s.size == 16 * 1024 and s.max() < 1024 and d.max() < 1024
    s, d, n = kc.gen_sbm(400, 4, 0.3, 0.0, 3).arrays()
    assert np.all(s // 100 == d // 100)  # p_out = 0: no edge leaves its block
    el = kc.gen_er(300, 0.0, 1)
    el.plant_cliques(2, 10, 10, 7)
    s, d, n = el.arrays()
    assert s.size == 2 * 45 and len(set(s.tolist()) | set(d.tolist())) == 20


def test_batch_generator_distribution():
    e = kc.gen_batch(200, 5)
    s, d, n = e.arrays()
    off, nn, kk, fam = e.batch_meta()
    assert off[0] == 0 and off[-1] == s.size and np.all(np.diff(off) >= 0)
    assert nn.min() >= 50 and nn.max() <= 5000
    assert kk.min() >= 4 and kk.max() <= 12
    assert set(fam.tolist()) == {0, 1, 2}
    for g in range(0, 200, 17):
        seg = slice(off[g], off[g + 1])
        if off[g + 1] > off[g]:
            assert s[seg].max() < nn[g] and d[seg].max() < nn[g]
    # same seed, same batch
    s2, _, _ = kc.gen_batch(200, 5).arrays()
    assert np.array_equal(s, s2)


def test_footprint_model_monotone():
    a = kc.footprint_bytes(1000, 10_000, 50)
    b = kc.footprint_bytes(1000, 100_000, 50)
    c = kc.footprint_bytes(100_000, 100_000, 50)
    assert 0 < a < b < c
    assert kc.footprint_bytes(4_000_000, 40_000_000, 2000) < 180e9
