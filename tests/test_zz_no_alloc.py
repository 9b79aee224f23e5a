"""hp_scan_exclusive_i32_noalloc: the scan entry point for callers that cannot
call cudaMalloc (their device memory belongs to a framework allocator, or a
cudaMalloc's implicit device synchronisation is too costly mid-pipeline).  It
takes no context and keeps its scratch in a fixed array of the library's
device image.  Checked through the C ABI against the context-based scan on
two calls in a row (the second smaller, so stale scratch from the first must
not leak into it), and directly against numpy's cumsum at the scan's tile
boundaries (4096 elements per tile), at the largest size it accepts, and in
place.  Kept in its own file so that it runs last."""
import ctypes as C

import numpy as np
import pytest

import hunyuansc25_b200 as hp
from hunyuansc25_b200._abi import HP_ERR_UNSUPPORTED, HP_OK, HP_SCAN_NOALLOC_MAX_N

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_in, d_out, n, stream):
    return lib.hp_scan_exclusive_i32_noalloc(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), n,
                                             C.c_void_p(stream.cuda_stream))


def _cumsum_excl(a):
    ref = np.zeros(a.size + 1, np.int64)
    ref[1:] = np.cumsum(a, dtype=np.int64)
    return ref


def test_noalloc_scan_matches_context_scan():
    import torch
    lib = hp.load_library()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    ctx = hp.Context(0)
    rng = np.random.default_rng(7)
    for n in (3_000_001, 40_000):   # two calls in a row, the second smaller
        a = torch.from_numpy(rng.integers(0, 100, size=n, dtype=np.int32)).to(dev)
        out_na = torch.full((n + 1,), -1, dtype=torch.int32, device=dev)
        assert _noalloc(lib, a, out_na, n, stream) == HP_OK
        out_ctx = ctx.scan_exclusive(a)
        torch.cuda.synchronize()
        assert torch.equal(out_na, out_ctx)   # integer scan: bit-exact
    ctx.close()


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, HP_SCAN_NOALLOC_MAX_N])
def test_noalloc_scan_matches_cumsum(n):
    import torch
    lib = hp.load_library()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(n + 11)
    # values small enough that the total of 2^26 elements stays below 2^31
    a = rng.integers(0, 16, size=n, dtype=np.int32)
    d_in = torch.from_numpy(a).to(dev) if n else torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.full((n + 1,), -1, dtype=torch.int32, device=dev)
    assert _noalloc(lib, d_in, out, n, stream) == HP_OK
    assert np.array_equal(out.cpu().numpy().astype(np.int64), _cumsum_excl(a))


def test_noalloc_scan_in_place_then_smaller():
    """In place (d_in == d_out), then a smaller call whose result must not
    depend on the tile words the larger call left in the shared array."""
    import torch
    lib = hp.load_library()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    for n in (1_000_003, 9_000):
        a = (np.arange(1, n + 1, dtype=np.int64) * 7919 % 13).astype(np.int32)
        buf = torch.zeros(n + 1, dtype=torch.int32, device=dev)
        buf[:-1] = torch.from_numpy(a).to(dev)
        assert _noalloc(lib, buf, buf, n, stream) == HP_OK
        assert np.array_equal(buf.cpu().numpy().astype(np.int64), _cumsum_excl(a))


def test_noalloc_scan_rejects_oversize():
    import torch
    lib = hp.load_library()
    small = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _noalloc(lib, small, small, HP_SCAN_NOALLOC_MAX_N + 1, torch.cuda.current_stream())
    assert rc == HP_ERR_UNSUPPORTED
