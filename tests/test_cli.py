"""The reference-compatible command line: graph readers (CPU) and one count
through the whole command (GPU)."""
import math
import subprocess
import sys

import numpy as np
import pytest

from kcgpu_b200.cli import read_graph


def test_readers_agree(tmp_path):
    # a triangle plus a pendant edge in every supported file format
    (tmp_path / "g.tsv").write_text("# comment\n0 1\n1 2 7\n\n2 0\n2 3\n")
    (tmp_path / "g.mtx").write_text("%%MatrixMarket matrix coordinate pattern symmetric\n4 4 4\n"
                                    "1 2\n2 3\n3 1\n3 4\n")
    np.array([[1, 0, 1], [2, 1, 1], [0, 2, 1], [3, 2, 1]], dtype=np.uint64).tofile(tmp_path / "g.bel")
    want = {(0, 1), (1, 2), (0, 2), (2, 3)}
    for name in ("g.tsv", "g.mtx", "g.bel"):
        s, d, n = read_graph(str(tmp_path / name))
        assert {tuple(sorted(e)) for e in zip(s.tolist(), d.tolist())} == want, name


def test_generator_specs():
    s, d, n = read_graph("gen:er:200:0.05:3")
    assert n == 200 and s.size == d.size and s.size > 0
    s2, d2, _ = read_graph("gen:er:200:0.05:3")
    assert np.array_equal(s, s2) and np.array_equal(d, d2)


@pytest.mark.gpu
def test_cli_counts_complete_graph(tmp_path):
    n = 12
    lines = [f"{i} {j}" for i in range(n) for j in range(i + 1, n)]
    (tmp_path / "k12.tsv").write_text("\n".join(lines) + "\n")
    for q, p in (("o8b", "node"), ("p8b", "edge"), ("p32n", "node")):
        out = subprocess.run([sys.executable, "-m", "kcgpu_b200.cli", "-g", str(tmp_path / "k12.tsv"), "-m", "kc",
                              "-o", "degen", "-k", "5", "-p", p, "-q", q], capture_output=True, text=True, check=True)
        counter = [ln for ln in out.stdout.splitlines() if ln.startswith("Counter = ")]
        assert counter == [f"Counter = {math.comb(n, 5)}"], (q, p, out.stdout)


@pytest.mark.gpu
def test_cli_local_counts(tmp_path):
    n = 10
    lines = [f"{i} {j}" for i in range(n) for j in range(i + 1, n)]
    (tmp_path / "k10.tsv").write_text("\n".join(lines) + "\n")
    out = subprocess.run([sys.executable, "-m", "kcgpu_b200.cli", "-g", str(tmp_path / "k10.tsv"), "-m", "lkc",
                          "-o", "degree", "-k", "4", "-p", "node", "-q", "o8b"], capture_output=True, text=True,
                         check=True)
    rows = [ln.split("\t") for ln in out.stdout.splitlines() if "\t" in ln]
    assert rows == [[str(v), str(math.comb(n - 1, 3))] for v in range(n)]
