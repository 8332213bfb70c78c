"""The allocation-free cell-list entry point, edm_cell_list_static.

It serves callers that cannot allocate device memory at call time: code
running inside a device memory pool or arena that a host framework sized in
advance, or a loop where cudaMalloc, which can synchronise the device, is
not acceptable.  Its scratch is a static device array instead of an
allocation.  Its result must equal the cell list the engine builds through
its normal entry points (edm_create, edm_set_state, edm_dynamics_step,
edm_get_cells) for the same positions, on two calls in a row: the second
call reuses the shared scratch left by the first.
"""
import ctypes as C

import numpy as np
import pytest

from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu


def _static_cells(L, positions: np.ndarray, dp):
    import torch
    nc = dp.nx * dp.ny
    pos = torch.as_tensor(np.ascontiguousarray(positions), device="cuda")
    start = torch.full((nc + 1,), -7, dtype=torch.int32, device="cuda")
    mem = torch.full((positions.shape[0],), -7, dtype=torch.int32, device="cuda")
    rc = L.edm_cell_list_static(C.c_void_p(pos.data_ptr()), positions.shape[0], dp.Lx, dp.Ly, dp.nx, dp.ny,
                                C.c_void_p(start.data_ptr()), C.c_void_p(mem.data_ptr()), None)
    assert rc == 0, L.edm_last_error()
    torch.cuda.synchronize()
    return start.cpu().numpy(), mem.cpu().numpy()


def test_static_cell_list_equals_engine_cell_list_on_two_calls():
    from flim_microscopy_simulator_with_causal_inference_b200 import engine as E
    L = E.load_library()
    P = Pair(cases.get("rich_small"), precision=64, photons=False)
    dp = P.dp
    nc = dp.nx * dp.ny
    for call in range(2):
        before = P.gpu_state()["positions"]   # the positions the next step sorts into cells
        P.eng.dynamics_step(1)
        ref_start, ref_mem = P.eng.cells(0)   # the engine's cell list of `before`
        start, mem = _static_cells(L, before, dp)
        assert np.array_equal(start, ref_start), f"cell starts differ on call {call + 1}"
        for c in range(nc):
            a, b = start[c], start[c + 1]
            assert np.array_equal(mem[a:b], np.sort(ref_mem[ref_start[c]:ref_start[c + 1]])), (call, c)


def test_static_cell_list_rejects_grids_beyond_its_scratch():
    from flim_microscopy_simulator_with_causal_inference_b200 import engine as E
    L = E.load_library()
    too_many = 1 << 11  # (2^11)^2 cells > EDM_STATIC_MAX_CELLS = 2^20
    rc = L.edm_cell_list_static(None, 0, 10.0, 10.0, too_many, too_many, None, None, None)
    assert rc == -1
    assert b"EDM_STATIC_MAX_CELLS" in L.edm_last_error()
