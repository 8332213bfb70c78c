"""The allocation-free cell-list entry point, edm_cell_list_static.

It serves callers that cannot allocate device memory at call time: code
running inside a device memory pool or arena that a host framework sized in
advance, or a loop where cudaMalloc, which can synchronise the device, is
not acceptable.  Its scratch is a static device array instead of an
allocation.  Its result must equal the cell list the engine builds through
its normal entry points (edm_create, edm_set_state, edm_dynamics_step,
edm_get_cells) for the same positions, on two calls in a row: the second
call reuses the shared scratch left by the first.  Edge cases (no particles,
a rectangular grid, points outside the box, thousands of points in one cell)
are checked against a numpy restatement of the reference's cell assignment
(ed_mrdt/dynamics.py:177-196: cx = int(x / cell) clamped into the grid).
"""
import ctypes as C

import numpy as np
import pytest

from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu


def _static_cells_raw(L, positions: np.ndarray, Lx, Ly, nx, ny):
    import torch
    n = positions.shape[0]
    pos = torch.as_tensor(np.ascontiguousarray(positions, dtype=np.float64).reshape(n, 2), device="cuda")
    start = torch.full((nx * ny + 1,), -7, dtype=torch.int32, device="cuda")
    mem = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    rc = L.edm_cell_list_static(C.c_void_p(pos.data_ptr()) if n else None, n, Lx, Ly, nx, ny,
                                C.c_void_p(start.data_ptr()), C.c_void_p(mem.data_ptr()), None)
    assert rc == 0, L.edm_last_error()
    torch.cuda.synchronize()
    return start.cpu().numpy(), mem.cpu().numpy()[:n]


def _static_cells(L, positions: np.ndarray, dp):
    return _static_cells_raw(L, positions, dp.Lx, dp.Ly, dp.nx, dp.ny)


def _numpy_cells(positions: np.ndarray, Lx, Ly, nx, ny):
    """Cell starts and members (ascending index) of the reference's cell
    assignment: cx = int(x / (Lx / nx)) clamped to [0, nx-1], likewise cy,
    key cx*ny + cy."""
    cx = np.clip(np.trunc(positions[:, 0] / (Lx / nx)), 0, nx - 1).astype(np.int64)
    cy = np.clip(np.trunc(positions[:, 1] / (Ly / ny)), 0, ny - 1).astype(np.int64)
    key = cx * ny + cy
    start = np.zeros(nx * ny + 1, dtype=np.int64)
    start[1:] = np.cumsum(np.bincount(key, minlength=nx * ny))
    return start.astype(np.int32), np.argsort(key, kind="stable").astype(np.int32)


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


def _edge_cases():
    rng = np.random.default_rng(2024)
    out = {"no particles": (np.zeros((0, 2)), 4.0, 3.0, 5, 7)}
    # a rectangular grid (nx != ny) with points below 0, at the box side and beyond it
    pts = rng.uniform(0.0, 1.0, (2000, 2)) * [6.5, 2.5]
    pts[:40] = rng.uniform(-3.0, 0.0, (40, 2))
    pts[40:80] = rng.uniform(1.0, 4.0, (40, 2)) * [6.5, 2.5]
    pts[80:90] = [6.5, 2.5]
    out["rectangular grid, points outside"] = (pts, 6.5, 2.5, 13, 5)
    # 3,000 points clamped into cell 0 beside 1,000 spread ones (shared-memory ranking)
    pts = rng.uniform(0.0, 10.0, (4000, 2))
    pts[rng.permutation(4000)[:3000]] = rng.uniform(-5.0, -0.001, (3000, 2))
    out["3,000 points in one cell"] = (pts, 10.0, 10.0, 40, 40)
    # 12,000 of 20,000 points beyond the box, clamped into the last cell (index-order scan)
    pts = rng.uniform(0.0, 10.0, (20000, 2))
    pts[rng.permutation(20000)[:12000]] = rng.uniform(10.0, 1.0e6, (12000, 2))
    out["12,000 points in one cell"] = (pts, 10.0, 10.0, 64, 32)
    return out


@pytest.mark.parametrize("name", list(_edge_cases()))
def test_static_cell_list_edge_cases_match_numpy_restatement(name):
    from flim_microscopy_simulator_with_causal_inference_b200 import engine as E
    L = E.load_library()
    pts, Lx, Ly, nx, ny = _edge_cases()[name]
    ref_start, ref_mem = _numpy_cells(pts, Lx, Ly, nx, ny)
    for call in range(2):
        start, mem = _static_cells_raw(L, pts, Lx, Ly, nx, ny)
        assert np.array_equal(start, ref_start), (name, call)
        assert np.array_equal(mem, ref_mem), (name, call)


def test_static_cell_list_rejects_too_many_particles():
    from flim_microscopy_simulator_with_causal_inference_b200 import engine as E
    L = E.load_library()
    rc = L.edm_cell_list_static(None, (1 << 24) + 1, 10.0, 10.0, 8, 8, None, None, None)
    assert rc == -1
    assert b"EDM_STATIC_MAX_PARTICLES" in L.edm_last_error()
