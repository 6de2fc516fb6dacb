"""Graph files parsed by the library's host readers (kc_edgelist_from_file):
text edge lists, Matrix Market and the reference's .bel records."""
import numpy as np
import pytest

import kcgpu_b200 as kc


def test_text_variants(tmp_path):
    f = tmp_path / "g.txt"
    f.write_bytes(b"# header\r\n% also a comment\n\n0 1\n1\t2 0.5\n  2,3\r\n3 0 7 9\n")
    s, d, n = kc.read_edgelist(f).arrays()
    assert s.tolist() == [0, 1, 2, 3] and d.tolist() == [1, 2, 3, 0] and n == 4


def test_matrix_market(tmp_path):
    f = tmp_path / "g.mtx"
    f.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% comment\n6 6 3\n1 2\n2 3\n3 1\n")
    s, d, n = kc.read_edgelist(f).arrays()
    assert s.tolist() == [0, 1, 2] and d.tolist() == [1, 2, 0]
    assert n == 6  # the size line keeps the isolated vertices 3..5


def test_bel_records(tmp_path):
    f = tmp_path / "g.bel"
    np.array([[1, 0, 9], [2, 1, 9], [0, 2, 9]], dtype=np.uint64).tofile(f)  # {dst, src, weight}
    s, d, n = kc.read_edgelist(f).arrays()
    assert s.tolist() == [0, 1, 2] and d.tolist() == [1, 2, 0] and n == 3


def test_errors(tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("0 1\n1 x\n")
    with pytest.raises(kc.KCError) as e:
        kc.read_edgelist(bad)
    assert e.value.name == "KC_ERR_INVALID_ARG" and "line 2" in str(e.value)
    big = tmp_path / "big.txt"
    big.write_text("0 4294967295\n")
    with pytest.raises(kc.KCError):
        kc.read_edgelist(big)
    short = tmp_path / "g.bel"
    short.write_bytes(b"\0" * 25)
    with pytest.raises(kc.KCError):
        kc.read_edgelist(short)
    with pytest.raises(kc.KCError):
        kc.read_edgelist(tmp_path / "missing.txt")
    mtx = tmp_path / "zero.mtx"
    mtx.write_text("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n0 1\n")  # 1-based ids
    with pytest.raises(kc.KCError):
        kc.read_edgelist(mtx)


def test_large_file_matches_and_is_ordered(tmp_path):
    rng = np.random.default_rng(3)
    m = 2_000_000
    e = rng.integers(0, 1 << 20, size=(m, 2), dtype=np.uint64)
    f = tmp_path / "large.tsv"
    np.savetxt(f, e, fmt="%d", delimiter="\t")
    s, d, n = kc.read_edgelist(f, format="text").arrays()
    assert np.array_equal(s, e[:, 0].astype(np.uint32)) and np.array_equal(d, e[:, 1].astype(np.uint32))
    assert n == int(e.max()) + 1


@pytest.mark.gpu
def test_graph_from_file_counts(tmp_path, ctx):
    s, d, n = kc.gen_er(500, 0.05, 4).arrays()
    f = tmp_path / "er.bel"
    np.stack([d.astype(np.uint64), s.astype(np.uint64), np.ones(s.size, np.uint64)], axis=1).tofile(f)
    with kc.Graph.from_edges(ctx, s, d, n) as a, kc.Graph.from_file(ctx, f) as b:
        a.orient("degen")
        b.orient("degen")
        assert a.info()["m"] == b.info()["m"]
        for k in (3, 4, 5):
            assert a.count(k) == b.count(k)
