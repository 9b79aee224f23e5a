"""Device primitives through the C ABI: decoupled look-back scan, exact cut."""
import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 31, 4095, 4096, 4097, 100000, 1 << 22, 10_000_019])
def test_scan_exclusive(ctx, n):
    import torch
    rng = np.random.default_rng(n)
    a = rng.integers(0, 50, size=n, dtype=np.int32)
    d = torch.from_numpy(a).cuda()
    out = ctx.scan_exclusive(d).cpu().numpy()
    ref = np.zeros(n + 1, np.int64)
    ref[1:] = np.cumsum(a, dtype=np.int64)
    assert np.array_equal(out.astype(np.int64), ref)


def test_scan_in_place(ctx):
    import torch
    a = np.arange(1, 300001, dtype=np.int32) % 7
    buf = torch.zeros(a.size + 1, dtype=torch.int32, device="cuda")
    buf[:-1] = torch.from_numpy(a).cuda()
    ctx.scan_exclusive(buf[:-1], buf)
    ref = np.concatenate([[0], np.cumsum(a)])
    assert np.array_equal(buf.cpu().numpy(), ref)


def test_edgecut_device(ctx):
    import torch
    g = graphs.rmat(14, 16, seed=3)
    where = (np.arange(g.nvtxs) * 2654435761 % 97).astype(np.int32)
    t = [torch.from_numpy(x).cuda() for x in (g.xadj, g.adjncy, g.adjwgt, where)]
    assert ctx.edgecut_device(t[0], t[1], t[2], t[3]) == oracle.edgecut(g, where)
    unit = graphs.Graph(g.xadj, g.adjncy, g.vwgt, np.ones_like(g.adjwgt))
    assert ctx.edgecut_device(t[0], t[1], None, t[3]) == oracle.edgecut(unit, where)
