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
    assert steps == (5 + 8 + 8) * 3
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


@pytest.mark.parametrize("precision", [32, 64])
def test_every_scatter_and_move_shape_gives_the_same_run(precision):
    """The order in which k_scatter's cursor atomics place the slots of one
    bucket, and the contact search's order of appends, differ from shape to
    shape (one or two slots per thread, block sizes, the contact search's
    forms); nothing downstream depends on them.  Fresh ensembles of jittered
    replicas, stepped through graph chunks with photons at each fixed shape,
    end with the same state, counters and stacks bit for bit."""
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    raws = W.ensemble_replicas(6, seed=17, n_min=600, n_max=2000)
    ref = None
    for scatter, move, contacts in ((0, 0, 0), (1, 5, 7), (2, 2, 3), (3, 5, 6), (4, 7, 1)):
        ens = Ensemble(raws, precision=precision, photons=True, device=0)
        eng = ens.engine
        got = eng.set_launch_shapes([scatter, move, contacts])
        assert got["k_scatter"]["candidate"] == scatter and got["k_move"]["candidate"] == move
        assert got["k_contacts"]["candidate"] == contacts
        s = torch.cuda.Stream()
        eng.pipeline_steps(60, True, 30, stream=s)
        s.synchronize()
        run = (eng.get_state(stream=s), eng.counters(), [eng.flim(r).copy() for r in range(ens.R)])
        eng.close()
        if ref is None:
            ref = run
            continue
        for key in ref[0]:
            assert np.array_equal(ref[0][key], run[0][key]), (scatter, move, key)
        assert np.array_equal(ref[1], run[1]), (scatter, move)
        for x, y in zip(ref[2], run[2]):
            assert np.array_equal(x, y), (scatter, move)
