"""The solve's failure path on the GPU, without a fault: every grid-wide wait
of the persistent solve is bounded (SphParams.timeout_ms).  A test hook makes
one block skip its first barrier arrival, so every block's wait runs out; the
step must come back as SPH_E_TIMEOUT with the state, time and dt untouched,
and the context must step on normally once the hook is off."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_barrier_timeout_reports_and_leaves_state():
    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH

    params = preset_params("dam_break_8k", timeout_ms=50)
    scene = preset_scene("dam_break_8k")
    sol = IISPH(stage_path=None, params=params, scene=scene)
    ref = IISPH(stage_path=None, params=params, scene=scene)
    sol.steps(3)
    ref.steps(4)
    x0, v0, p0, t0, dt0 = sol.x.numpy(), sol.v.numpy(), sol.p.numpy(), sol.sim_time, sol.dt

    _lib.check(sol._ctx, sol._lib.sph_test_stall_barrier(sol._ctx, 0))
    with pytest.raises(_lib.SphError) as err:
        sol.step()
    assert err.value.code == _lib.SPH_E_TIMEOUT
    assert np.array_equal(sol.x.numpy(), x0) and np.array_equal(sol.v.numpy(), v0)
    assert np.array_equal(sol.p.numpy(), p0)
    assert sol.stats_history(1)[0]["step_index"] == 3  # no step was recorded

    # hook off: the same step again gives what an undisturbed run gives
    _lib.check(sol._ctx, sol._lib.sph_test_stall_barrier(sol._ctx, -1))
    sol.step()
    assert sol.sim_time == ref.sim_time and sol.dt == ref.dt
    assert np.array_equal(sol.x.numpy(), ref.x.numpy())
    assert np.array_equal(sol.v.numpy(), ref.v.numpy())
    assert np.array_equal(sol.p.numpy(), ref.p.numpy())
    assert sol.sim_time > t0 and dt0 > 0
    sol.close()
    ref.close()


def test_inference_wait_timeout_frees_tensor_memory():
    """The learned warm start's tensor-core kernel with its MMAs withheld: its
    bounded mbarrier wait runs out, it frees its tensor memory and flags the
    step, the solve stops at its first barrier, and the step reports
    SPH_E_TIMEOUT with the state untouched.  Afterwards inference allocates
    tensor memory again and the retried step equals an undisturbed run's."""
    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH

    params = preset_params("dam_break_8k", warm_start="mlp", timeout_ms=50)
    scene = preset_scene("dam_break_8k")
    sol = IISPH(stage_path=None, params=params, scene=scene)
    ref = IISPH(stage_path=None, params=params, scene=scene)
    sol.steps(3)
    ref.steps(4)
    x0, p0 = sol.x.numpy(), sol.p.numpy()

    _lib.check(sol._ctx, sol._lib.sph_test_withhold_mma(sol._ctx, 1))
    with pytest.raises(_lib.SphError) as err:
        sol.step()
    assert err.value.code == _lib.SPH_E_TIMEOUT
    assert np.array_equal(sol.x.numpy(), x0) and np.array_equal(sol.p.numpy(), p0)

    _lib.check(sol._ctx, sol._lib.sph_test_withhold_mma(sol._ctx, 0))
    sol.step()
    assert np.array_equal(sol.x.numpy(), ref.x.numpy())
    assert np.array_equal(sol.p.numpy(), ref.p.numpy())
    sol.close()
    ref.close()
