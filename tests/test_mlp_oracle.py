"""CPU checks of the warm-start network's reference implementation."""
import numpy as np
import torch

from oracle import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e4, 1000), [0.0, -0.0, 1.0, 3.0e38]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_blob_layout():
    assert M.NPARAMS == 4993 and M.BLOB == 5016
    from warpsph_b200 import _lib
    from warpsph_b200.learned import init_blob

    rng = np.random.default_rng(1)
    f = rng.normal(0, 1, (256, M.NF)).astype(np.float32)
    t = rng.normal(0, 3, 256).astype(np.float32)
    blob = init_blob(f, t)
    assert blob.size == _lib.SPH_MLP_BLOB
    w = M.unpack(blob)
    assert w["W1"].shape == (11, 64) and w["W2"].shape == (64, 64)
    loss, grad, y = M.loss_and_grad(blob, f, t)
    assert grad.size == M.NPARAMS and np.isfinite(loss)
