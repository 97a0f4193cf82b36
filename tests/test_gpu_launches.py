"""The library's own count of the kernels it launches (hf_kernel_launches),
which the bench lines report as gpu_launches: direct launches outside graph
capture plus every kernel node of each graph launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hydroflux_b200 import _lib, workloads
    return _lib, workloads


def test_run_steps_launch_count(gpu):
    """run_steps(K) launches its set-run kernel and K steps of three kernels
    each (control, stage 1, stage 2), replayed from 64-, 8- and 1-step graphs."""
    _lib, workloads = gpu
    s = workloads.step_regime("all_wet", 256)
    with workloads.simulation_for(s) as sm:
        sm.run_steps(5)  # graph capture, initial CFL
        for k in (1, 8, 77, 100):
            before = _lib.kernel_launches()
            sm.run_steps(k)
            assert _lib.kernel_launches() - before == 3 * k + 1


def test_capture_is_not_counted(gpu):
    """Capturing a graph launches nothing: the first run_steps of a chunk
    size counts the same as later ones."""
    _lib, workloads = gpu
    s = workloads.step_regime("all_wet", 128)
    with workloads.simulation_for(s) as sm:
        sm.run_steps(1)
        before = _lib.kernel_launches()
        sm.run_steps(64)  # captures the 64-step graph, then launches it
        first = _lib.kernel_launches() - before
        before = _lib.kernel_launches()
        sm.run_steps(64)
        assert first == _lib.kernel_launches() - before == 3 * 64 + 1


def test_ensemble_launches_four_kernels_per_batch_step(gpu):
    """A batch step is control, stage 1, stage 2 and clock commit."""
    _lib, workloads = gpu
    from hydroflux_b200.ensemble import Ensemble
    scns = [workloads.valley(n=n, dx=5.0, seed=k, t_end=1e9) for k, n in enumerate((48, 96))]
    with Ensemble(scns) as e:
        e.set_schedule(1)
        e.run(8)
        before = _lib.kernel_launches()
        e.run(72)  # one 64-step and one 8-step chunk
        assert _lib.kernel_launches() - before == 4 * 72
        assert all(e.info(k)["steps"] == 80 for k in range(2))


def test_ensemble_solo_scenarios_add_two_launches_per_batch_step(gpu):
    """A scenario of at least 512 tiles of 32 x 32 runs its two stages as its
    own launches: 4 + 2 kernels per batch step with one such scenario."""
    _lib, workloads = gpu
    from hydroflux_b200.ensemble import Ensemble
    scns = [workloads.valley(n=48, dx=5.0, seed=1, t_end=1e9),
            workloads.valley(n=736, dx=5.0, seed=2, t_end=1e9)]
    with Ensemble(scns) as e:
        e.set_schedule(1)
        e.run(8)
        before = _lib.kernel_launches()
        e.run(72)
        assert _lib.kernel_launches() - before == 6 * 72
