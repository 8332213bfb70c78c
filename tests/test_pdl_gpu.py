"""Programmatic dependent launches of the BD step's kernels.

Each kernel of the step's chain goes as a programmatic dependent of the
kernel before it on the stream and waits, as its first statement, for that
kernel's completion.  The results must not depend on it: an engine created
with EDM_PDL=0 (ordinary launches) and one created without it give the same
state, counters and stacks bit for bit, through the graph chunks and the
eager steps, on systems whose schedules hold every kind of reaction pass
(binding, dissociation, catalytic passes with their contact search,
recruitment, detachment, conversion, the adaptation field and the local
recruitment CDF).
"""
import os

import numpy as np
import pytest
import torch

from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu


def _with_pdl(flag, make):
    old = os.environ.get("EDM_PDL")
    try:
        if flag:
            os.environ.pop("EDM_PDL", None)
        else:
            os.environ["EDM_PDL"] = "0"
        return make()
    finally:
        if old is None:
            os.environ.pop("EDM_PDL", None)
        else:
            os.environ["EDM_PDL"] = old


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "adaptive_local", "exchange_heavy"])
@pytest.mark.parametrize("precision", [64, 32])
def test_chained_launches_give_the_ordinary_results(case, precision):
    raw = cases.get(case)
    runs = []
    for flag in (False, True):
        P = _with_pdl(flag, lambda: Pair(raw, precision=precision, photons=True))
        s = torch.cuda.Stream()
        P.eng.pipeline_steps(40, True, 20, stream=s)  # graph chunks
        P.eng.dynamics_step(5, stream=s)  # eager steps
        s.synchronize()
        runs.append((P.gpu_state(), P.eng.counters(), P.eng.flim(0).copy(), P.eng.status()))
    (a, ca, fa, sa), (b, cb, fb, sb) = runs
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(ca, cb)
    assert np.array_equal(fa, fb)
    assert sa == sb


def test_chained_launches_on_a_jittered_ensemble():
    raws = W.ensemble_replicas(8, seed=5, n_min=600, n_max=2000)
    out = []
    for flag in (False, True):
        ens = _with_pdl(flag, lambda: Ensemble(raws, precision=32, photons=True, device=0))
        eng = ens.engine
        s = torch.cuda.Stream()
        eng.pipeline_steps(100, True, 100, stream=s)
        s.synchronize()
        out.append((eng.get_state(stream=s), eng.counters(), [eng.flim(r).copy() for r in range(ens.R)]))
    (a, ca, fa), (b, cb, fb) = out
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(ca, cb)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)
