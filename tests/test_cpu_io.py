"""METIS .graph reader / .part writer (the reference's file formats)."""
import os

import numpy as np
import pytest

from hunyuansc25_b200 import graphs


def test_roundtrip(tmp_path):
    g = graphs.grid3d(7, 6, 5, seed=2, wmin=1, wmax=10)
    p = str(tmp_path / "g.graph")
    graphs.write_metis(p, g)
    h = graphs.read_metis(p)
    for a in ("xadj", "adjncy", "vwgt", "adjwgt"):
        assert np.array_equal(getattr(g, a), getattr(h, a)), a


def test_formats(tmp_path):
    p = tmp_path / "t.graph"
    # 4-cycle, unweighted, with comments (fmt 0)
    p.write_text("% comment\n4 4\n2 4\n1 3\n% inner comment\n2 4\n3 1\n")
    g = graphs.read_metis(str(p))
    assert list(g.xadj) == [0, 2, 4, 6, 8]
    assert list(g.adjncy) == [1, 3, 0, 2, 1, 3, 2, 0]
    assert np.all(g.adjwgt == 1) and np.all(g.vwgt == 1)
    # vertex weights + edge weights (fmt 11)
    p.write_text("3 2 11\n5 2 7\n1 1 7 3 9\n2 2 9\n")
    g = graphs.read_metis(str(p))
    assert list(g.vwgt) == [5, 1, 2]
    assert list(g.adjwgt) == [7, 7, 9, 9]
    # vertex sizes are skipped (fmt 111)
    p.write_text("2 1 111\n4 3 2 6\n8 1 1 6\n")
    g = graphs.read_metis(str(p))
    assert list(g.vwgt) == [3, 1] and list(g.adjncy) == [1, 0] and list(g.adjwgt) == [6, 6]


@pytest.mark.parametrize("text,msg", [
    ("2 1\n3\n1\n", "out of range"),
    ("2 2\n2\n1\n", "header gives"),
    ("2 1 1\n2 0\n1 0\n", "must be positive"),
    ("3 1\n2\n1\n", "premature end"),
    ("x y\n", "header"),
])
def test_errors(tmp_path, text, msg):
    p = tmp_path / "bad.graph"
    p.write_text(text)
    with pytest.raises(ValueError, match=msg):
        graphs.read_metis(str(p))


def test_write_partition(tmp_path):
    f = str(tmp_path / "g.graph")
    out = graphs.write_partition(f, np.array([0, 3, 1], np.int32), 4)
    assert out.endswith("g.graph.part.4")
    assert open(out).read() == "0\n3\n1\n"


def _mtx_reference(n, entries):
    """Pattern of A + A^T without the diagonal, rows sorted and unique (the
    reference converter's result, matrix_to_graph/matrix_to_graph.c)."""
    adj = [set() for _ in range(n)]
    for i, j in entries:
        if i != j:
            adj[i].add(j)
            adj[j].add(i)
    xadj = np.zeros(n + 1, np.int64)
    for i in range(n):
        xadj[i + 1] = xadj[i] + len(adj[i])
    return xadj, np.array([j for i in range(n) for j in sorted(adj[i])], np.int64)


def test_mtx_general_and_symmetric(tmp_path):
    rng = np.random.default_rng(4)
    n = 40
    ent = [(int(a), int(b)) for a, b in rng.integers(0, n, size=(150, 2))]
    ent += [(3, 3), (5, 7), (5, 7), (7, 5)]      # diagonal and duplicates
    p = tmp_path / "a.mtx"
    lines = ["%%MatrixMarket matrix coordinate real general", "% a comment", f"{n} {n} {len(ent)}"]
    lines += [f"{i + 1} {j + 1} {0.5 * (i + j)}" for i, j in ent]
    p.write_text("\n".join(lines) + "\n")
    g = graphs.read_mtx(str(p))
    xadj, adj = _mtx_reference(n, ent)
    assert np.array_equal(g.xadj, xadj) and np.array_equal(g.adjncy, adj)
    assert np.all(g.adjwgt == 1) and np.all(g.vwgt == 1)
    # symmetric storage (lower triangle only) gives the same graph
    low = sorted({(max(i, j), min(i, j)) for i, j in ent})
    q = tmp_path / "s.mtx"
    q.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n"
                 f"{n} {n} {len(low)}\n" + "".join(f"{i + 1} {j + 1}\n" for i, j in low))
    h = graphs.read_mtx(str(q))
    assert np.array_equal(h.xadj, xadj) and np.array_equal(h.adjncy, adj)
    # conversion to METIS next to the input, readable by the METIS reader
    out = graphs.mtx_to_metis(str(q))
    assert out.endswith("s.graph")
    r = graphs.read_metis(out)
    assert np.array_equal(r.xadj, xadj) and np.array_equal(r.adjncy, adj)


def test_mtx_errors(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(ValueError, match="coordinate"):
        graphs.read_mtx(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 4 1\n1 2 1.0\n")
    with pytest.raises(ValueError, match="square"):
        graphs.read_mtx(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 2 1.0\n")
    with pytest.raises(ValueError, match="premature"):
        graphs.read_mtx(str(p))
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 1\n1 9 1.0\n")
    with pytest.raises(ValueError, match="bad entry"):
        graphs.read_mtx(str(p))
    with pytest.raises(ValueError):
        graphs.read_mtx(str(tmp_path / "missing.mtx"))


def test_cli_argument_errors(capsys):
    from hunyuansc25_b200.__main__ import main
    with pytest.raises(SystemExit):
        main([])
    with pytest.raises(SystemExit):
        main(["only_a_graph.graph"])
