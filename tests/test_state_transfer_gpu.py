"""State transfers overlapped with computation (edm_set_state_async, or its
halves edm_stage_state_async + edm_install_state, and edm_get_state_async): a
pipelined frame loop (the next frame's state goes up while this frame's result
comes down) gives, frame by frame, the states the synchronous edm_set_state /
edm_get_state loop gives."""
import numpy as np
import pytest

from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("split", [False, True])
def test_pipelined_async_frames_equal_synchronous_frames(precision, split):
    import torch
    raw = cases.get("rich_small")
    A = Pair(raw, precision=precision, photons=True)
    B = Pair(raw, precision=precision, photons=True)
    st = A.state
    host = dict(positions=st.positions.astype(np.float64), species=st.species_id.astype(np.int32),
                alive=st.is_alive.astype(np.uint8), bond=st.bond_partner.astype(np.int32),
                has_dye=st.has_dye.astype(np.uint8), dye=st.dye_type_id.astype(np.int32),
                ctmc=st.ctmc_state.astype(np.int8), bleached=st.is_bleached.astype(np.uint8))
    pinned = {k: _pinned(v) for k, v in host.items()}
    N = B.eng.N
    outs = [{k: _pinned(np.zeros((N, w) if w > 1 else N, dtype=dt)) for k, dt, w in B.eng.STATE_FIELDS}
            for _ in range(3)]
    s = torch.cuda.Stream()
    frames = 3
    want = []
    for _ in range(frames):  # synchronous loop
        A.eng.set_state(*(pinned[k] for k in ("positions", "species", "alive", "bond", "has_dye", "dye", "ctmc",
                                               "bleached")), stream=s)
        A.eng.pipeline_steps(10, True, 10, stream=s)
        want.append(A.eng.get_state(stream=s))
    # pipelined loop: upload frame k + 1 before frame k's result has come down
    # (split: the upload is queued before this frame's read, the installation after)
    B.eng.set_state_async(pinned, stream=s)
    for k in range(frames):
        B.eng.pipeline_steps(10, True, 10, stream=s)
        if split and k + 1 < frames:
            B.eng.stage_state_async(pinned)
        B.eng.get_state_async(outs[k], stream=s)
        if k + 1 < frames:
            if split:
                B.eng.install_state(stream=s)
            else:
                B.eng.set_state_async(pinned, stream=s)
    B.eng.transfers_wait()
    s.synchronize()
    for k in range(frames):
        for key in want[k]:
            assert np.array_equal(outs[k][key], want[k][key]), (k, key)
    assert not np.array_equal(outs[0]["positions"], outs[1]["positions"]), "frames should differ (step counter)"
    assert np.array_equal(A.eng.counters(), B.eng.counters())
