"""Parity at the benchmark configurations' full sizes: the R-MAT scale-22 graph
at k = 256 and the 2^24-point geometric graph at k = 1024, every level (CSR,
vertex and edge weights, matching, cmap, both partitions, both cuts) equal to
the oracle's, under the workloads' committed tuning files (the tuned row
classes are the ones the benchmark runs); and a 64-graph sample of the
1,024-graph batch specification, every graph of one batched call equal to the
oracle's partition of it.  The hub and long-row classes that only large R-MAT
levels reach, and the dense k = 1024 gain rows, are covered here."""
import os

import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs, tune

from test_gpu_parity import compare_runs

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _threads():
    n = os.cpu_count() or 1
    graphs.set_threads(n)
    oracle.set_threads(n)
    yield


def _tuned(ctx, workload):
    path = tune.resolve_tuning("auto", workload)
    if path:
        ctx.load_tuning(path)


def test_full_rmat22_k256(ctx):
    """BASELINE configuration 3 (plain refiner): R-MAT scale 22, edge factor 16,
    weights U{1..100}, k = 256, imbalance 1.03."""
    g = graphs.config_rmat(22)
    _tuned(ctx, "rmat22")
    try:
        part, cut, st = compare_runs(ctx, g, 256, 1.03)
    finally:
        ctx.set_tuning(None)
    assert st.max_excess <= 0
    assert st.nlevels > 10


def test_full_rgg24_k1024(ctx):
    """BASELINE configuration 4 (plain refiner): 2^24 points, mean degree 12,
    w = int(1000 (1 - d/r)) + 1, k = 1024, imbalance 1.05."""
    g = graphs.config_rgg(1 << 24)
    _tuned(ctx, "rgg24")
    try:
        part, cut, st = compare_runs(ctx, g, 1024, 1.05)
    finally:
        ctx.set_tuning(None)
    assert st.max_excess <= 0


def test_batch_sample_of_1024(ctx):
    """64 graphs of the 1,024-graph batch (every 16th of graphs.batch_specs(1024,
    seed=5), generated with the benchmark's seeds): one batched call, each
    graph's partition and cut equal to the oracle's."""
    specs = graphs.batch_specs(1024, seed=5)
    idx = list(range(0, 1024, 16))
    gs = [graphs.batch_graph(specs[i][0], specs[i][1], seed=1000 + i) for i in idx]
    ks = [specs[i][2] for i in idx]
    parts, cuts = ctx.partition_batch(gs, ks, 1.03)
    for g, k, p, c in zip(gs, ks, parts, cuts):
        op, oc, _ = oracle.partition(g, k, 1.03)
        assert oc == c
        assert np.array_equal(op, p)
