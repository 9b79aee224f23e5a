"""MLP weight blob (versioned, SHA-256 checked) and initialisation; no GPU."""
import numpy as np
import pytest

from hunyuansc25_b200 import learn
from hunyuansc25_b200._abi import HP_MLP_NPARAM


def test_weight_blob_roundtrip(tmp_path):
    p = learn.init_params(9)
    f = str(tmp_path / "w.bin")
    learn.save_params(f, p, -0.25, "unit")
    q, thr, meta = learn.load_params(f)
    assert np.array_equal(p, q) and thr == pytest.approx(-0.25) and meta == "unit"
    data = bytearray(open(f, "rb").read())
    data[60] ^= 1
    open(f, "wb").write(bytes(data))
    with pytest.raises(ValueError):
        learn.load_params(f)
    assert p.shape[0] == HP_MLP_NPARAM


def test_init_params_shapes():
    p = learn.init_params(0)
    assert p.dtype == np.float32 and p.shape == (HP_MLP_NPARAM,)
    assert np.all(p[256:288] == 0) and np.all(p[1312:1344] == 0) and p[1376] == 0
