"""The launch-shape autotuner (edm_autotune): every candidate shape computes
the same state, so tuning is just the first steps of a run.  An engine tuned
on real steps ends bit-identical (float64 path) to an engine of the same
system stepped the same number of times with the fixed default shapes, and
the chosen shapes are reported and reused by the next engine of its kind."""
import numpy as np
import pytest

from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu


def test_autotuned_engine_matches_default_shapes_bitwise():
    import torch
    raw = cases.get("rich_small")
    plain = Pair(raw, precision=64, photons=False)   # created before any tuning: default shapes
    tuned = Pair(raw, precision=64, photons=False)
    s = torch.cuda.Stream()
    shapes = tuned.eng.autotune(2, retune=True, stream=s)
    s.synchronize()
    steps = tuned.eng.get_step()
    # candidates of k_scatter, k_move, k_contacts (by sweeper, by neighbour column,
    # over the move's sweeper list: no binding pass here) x (1 + 2 timed) steps
    assert steps == (3 + 8 + 8) * 3
    for k, v in shapes.items():
        assert v["block"] in (128, 256, 512) and v["candidates"] >= 3, (k, v)
        assert 0.0 < v["tuned_ms"] <= v["default_ms"], (k, v)
    plain.eng.dynamics_step(steps)
    a, b = tuned.gpu_state(), plain.gpu_state()
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(tuned.eng.counters(), plain.eng.counters())
    # a later engine of the same kind starts with the tuned shapes
    again = Pair(raw, precision=64, photons=False)
    got = again.eng.launch_shapes()
    for k in shapes:
        assert got[k]["candidate"] == shapes[k]["candidate"], (k, got[k], shapes[k])
