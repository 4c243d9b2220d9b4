"""Learned warm start on the GPU: the tensor-core forward/backward kernels
against the CPU reference, training, and the effect on the pressure solve."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from tests.helpers import normrel

pytestmark = pytest.mark.gpu


def _data(n=4096, seed=0):
    rng = np.random.default_rng(seed)
    nf = M.NF
    f = rng.normal(0, 1, (n, nf)).astype(np.float32) * np.linspace(0.5, 3, nf, dtype=np.float32)
    f += np.linspace(-2, 2, nf, dtype=np.float32)
    t = (np.maximum(f[:, 7], 0) * 2.0 + 0.3 * f[:, 3] + 0.1 * f[:, 0] ** 2).astype(np.float32)
    return f, t


def test_forward_and_gradient_match_oracle():
    from warpsph_b200 import learned

    f, t = _data()
    blob = learned.init_blob(f, t, seed=3)
    pred, loss, grad = learned.evaluate(blob, f, t)
    loss_o, grad_o, y_o = M.loss_and_grad(blob, f, t)
    # the tensor-core inference against the oracle that accumulates as it does
    assert normrel(pred, M.forward(blob, f, tc=True)["y"]) < 1e-5
    assert normrel(pred, y_o) < 2e-3
    assert abs(loss - loss_o) < 1e-4 * loss_o
    assert normrel(grad, grad_o) < 1e-3
    # per-block: every parameter group agrees
    off = 0
    for name, shape in M.SIZES:
        k = int(np.prod(shape))
        assert normrel(grad[off:off + k], grad_o[off:off + k]) < 2e-3, name
        off += k


def test_training_reduces_loss():
    from warpsph_b200 import learned

    f, t = _data(n=60000, seed=1)
    r = learned.residual_target(f, t)  # what the network regresses: t - max(input 3, input 10)
    blob0 = learned.init_blob(f, r, seed=0)
    l0 = M.loss_and_grad(blob0, f[:4096], r[:4096])[0]
    blob, losses = learned.train(f, t, epochs=8, batch=2048, lr=1e-3, seed=0, blob=blob0)
    assert losses[-1] < 0.2 * losses[0]
    l1 = M.loss_and_grad(blob, f[:4096], r[:4096])[0]
    assert l1 < 0.2 * l0
    # the prediction adds the skip input back
    y = learned.evaluate(blob, f[:64])
    want = np.maximum(f[:64, 3], f[:64, 10]) + np.minimum(y * blob[2 * learned.NF], 0.5)
    assert np.allclose(learned.predict(blob, f[:64]), want, rtol=0, atol=1e-6)


def test_learned_warm_start_reduces_iterations():
    """Trained on a few small dam breaks, the network must cut the Jacobi
    iterations of an unseen one against p = 0, while the solve's own
    convergence test still decides (avg_err <= eta or the cap)."""
    from warpsph_b200 import learned
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import dam_break
    from warpsph_b200.solver import IISPH

    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    train_scenes = [dam_break(fluid=(14 + 2 * k, 16, 10), spacing=0.02, box=(0.8, 0.5, 0.22), jitter=1e-4,
                              seed=10 + k) for k in range(3)]
    f, t = learned.collect(train_scenes, steps=120, per_step=400, params_for=lambda s: params, seed=0)
    blob, losses = learned.train(f, t, epochs=10, batch=2048, lr=1e-3, seed=0)
    assert losses[-1] < losses[0]
    test_scene = dam_break(fluid=(18, 18, 12), spacing=0.02, box=(0.9, 0.5, 0.26), jitter=1e-4, seed=99)
    iters = {}
    for mode in ("zero", "mlp"):
        p = params.replace(warm_start=mode, extra={"mlp_blob": blob})
        sol = IISPH(stage_path=None, params=p, scene=test_scene)
        sol.steps(100)
        hist = sol.stats_history(100)
        iters[mode] = sum(h["iterations"] for h in hist)
        for h in hist:
            assert h["avg_err"] <= params.eta or h["iterations"] == 101
        assert np.all(sol.p.numpy() >= 0)
        sol.close()
    assert iters["mlp"] < iters["zero"], iters


def test_shipped_network_beats_half_start():
    """The shipped network against the plain 0.5 p_prev start (the variant
    at IISPH.py:174, the config's comparator) on a dam break that is not in
    its training data, over the first 100 steps including the start-up
    transient: fewer Jacobi iterations, with the solve's own test deciding
    convergence in both."""
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import dam_break
    from warpsph_b200.solver import IISPH

    params = SolverParams(diameter=0.01, gravity=9.81, w_table_size=1024, g_table_size=1024)
    scene = dam_break(fluid=(40, 36, 30), spacing=0.01, box=(1.1, 0.6, 0.4), jitter=5e-5, seed=123)
    iters = {}
    for mode in ("half", "mlp"):
        sol = IISPH(stage_path=None, params=params.replace(warm_start=mode), scene=scene)
        sol.steps(100)
        hist = sol.stats_history(100)
        iters[mode] = sum(h["iterations"] for h in hist)
        for h in hist:
            assert h["avg_err"] <= params.eta or h["iterations"] == params.max_loop + 1
        sol.close()
    assert iters["mlp"] < iters["half"], iters
