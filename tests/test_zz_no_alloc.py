"""hf_ssprk2_step_noalloc: the SSP-RK2 step for callers that cannot allocate
device memory (hosts whose caching allocator has reserved the GPU up front,
loops that must not trigger cudaMalloc's device-wide synchronization). It
keeps its scratch in a fixed array inside the library instead of an
hf_workspace. This file is collected last so that a failure here leaves
every other test already run; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

from hydroflux_b200 import abi
from tests.gpu_util import assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _case(nr, nc, seed):
    rng = np.random.default_rng(seed)
    z = rng.uniform(-0.3, 0.3, (nr, nc)) + 0.01 * np.arange(nc)[None, :]
    h = rng.uniform(0.1, 1.5, (nr, nc))
    h[rng.uniform(size=(nr, nc)) > 0.8] = 0.0
    hu = rng.normal(0, 0.3, (nr, nc)) * (h > 0)
    hv = rng.normal(0, 0.3, (nr, nc)) * (h > 0)
    return z, h, hu, hv


# (1024, 1024) is exactly HF_NOALLOC_MAX_CELLS: its stage buffer reaches the
# last element of the fixed scratch array.
@pytest.mark.parametrize("shape", [(37, 53), (512, 512), (1024, 1024)])
def test_noalloc_step_matches_workspace_step(torch_cuda, shape):
    torch = torch_cuda
    from hydroflux_b200 import sim, step
    from hydroflux_b200._lib import last_error, lib
    nr, nc = shape
    z, h, hu, hv = _case(nr, nc, seed=nr + nc)
    mesh = step.DeviceMesh(z, 2.0, 1.5, 0.03)
    bcs = sim.Boundaries2D(sim.Boundary.wall(), sim.Boundary.transmissive(),
                           sim.Boundary.discharge(0.2), sim.Boundary.depth(0.5))
    ws = step.StepWorkspace2D(nr, nc)
    dev = torch.cuda.current_device()
    ref = [torch.tensor(a, device="cuda") for a in (h, hu, hv)]
    got = [torch.tensor(a, device="cuda") for a in (h, hu, hv)]
    grid = mesh.grid()
    cb = bcs.to_c()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # two calls in a row share (and reuse) the scratch array
        dt = 0.01 * (call + 1)
        step.ssprk2_step(*ref, mesh, bcs, dt, ws)
        rc = lib().hf_ssprk2_step_noalloc(C.byref(grid), *[C.c_void_p(t.data_ptr()) for t in got],
                                          C.byref(cb), dt, dev, stream)
        assert rc == 0, last_error()
        torch.cuda.synchronize()
        a = [t.cpu().numpy() for t in got]
        b = [t.cpu().numpy() for t in ref]
        assert_parity(a, b, what=f"call {call}: ")
        assert all(np.array_equal(x, y) for x, y in zip(a, b)), f"call {call}: not bitwise"


def test_noalloc_rejects_grids_beyond_its_scratch(torch_cuda):
    from hydroflux_b200._lib import last_error, lib
    # 1025 x 1024 cells is one row more than the fixed scratch holds; the call
    # is rejected before any pointer is touched, so placeholders suffice.
    grid = abi.hf_grid(1025, 1024, 1.0, 1.0, C.c_void_p(1), None)
    dummy = C.c_void_p(1)
    rc = lib().hf_ssprk2_step_noalloc(C.byref(grid), dummy, dummy, dummy, None, 0.01, 0, None)
    assert rc == abi.HF_ERR_INVALID_ARG
    assert "exceeds" in last_error()
