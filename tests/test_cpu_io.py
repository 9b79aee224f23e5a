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
