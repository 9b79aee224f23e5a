"""The command-line partitioner (python -m hunyuansc25_b200): the reference CLI's
output lines, the .part.k file, and the same cut as the library call."""
import re

import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs
from hunyuansc25_b200.__main__ import main

pytestmark = pytest.mark.gpu


def test_cli_metis_file(tmp_path, capsys):
    g = graphs.grid2d(40, 30, seed=3, wmin=1, wmax=7)
    path = str(tmp_path / "g.graph")
    graphs.write_metis(path, g)
    assert main([path, "6", "--iters", "2", "--write-part"]) == 0
    out = capsys.readouterr().out
    assert out.startswith(f"graph:{path} {g.nvtxs} {g.nedges // 2} 6 0")
    assert out.count("Hunyuangraph-Partition-end") == 2
    cuts = [int(x) for x in re.findall(r"edge-cut=\s+(\d+)", out)]
    best = int(re.search(r"best_edgecut=\s+(\d+)", out).group(1))
    assert len(cuts) == 2 and cuts[0] == cuts[1] == best
    part = np.loadtxt(path + ".part.6", dtype=np.int64)
    assert part.shape == (g.nvtxs,) and part.min() >= 0 and part.max() < 6
    assert oracle.edgecut(g, part.astype(np.int32)) == best
    imb = [float(x) for x in re.findall(r"imbalance=\s+([\d.]+)", out)]
    assert all(x <= 1.03 + 1e-6 for x in imb)
