"""Sides of the catalytic contact sweep (edm_contact_sides).

Each catalytic reaction's direct pairs can be found by sweeping from its
enzyme species or from its substrate species; the pairs whose partner an
earlier pass converts are looked up by the converting pass.  Whichever sides
are chosen, the float64 path must reproduce the oracle (the reference's
single pair-list sweep) bit for bit: event counts, species, positions.  The
catalytic rates of these systems are scaled up, so conversions that feed a
later pass of the same step (the late pairs) happen every few steps.
"""
import numpy as np
import pytest

from tests import cases
from tests.harness import Pair, compare_state

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12  # µm


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "adaptive_local"])
@pytest.mark.parametrize("sides", ["enzyme", "substrate", "counted"])
def test_every_sweep_side_matches_the_oracle(case, sides):
    P = Pair(cases.get(case), precision=64, photons=False)
    n_cat = len(P.cfg.catalytic_reactions)
    full = (1 << n_cat) - 1
    if sides == "enzyme":
        assert P.eng.contact_sides(full) == full
    elif sides == "substrate":
        assert P.eng.contact_sides(0) == 0
    else:  # the sides the first state's species counts chose
        assert 0 <= P.eng.contact_sides() <= full
    for t in range(40):
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        if t % 10 == 9:
            compare_state(P.gpu_state(), P.orc, F64_TOL)
    g = P.eng.counters()[0]
    assert np.array_equal(g[:6], P.orc.counters[:6]), (g[:6], P.orc.counters[:6])
    assert P.orc.counters[2] > 0, "no catalytic events: the test would not exercise the contact lists"
    assert P.eng.status() == 0


def test_float32_sides_agree():
    """float32 path: both sides give the same state step for step (the
    float32 pair tests are symmetric in the two particles)."""
    raw = cases.get("rich_small")
    runs = []
    for mask in (0, 0x7FFFFFFF):
        P = Pair(raw, precision=32, photons=False)
        P.eng.contact_sides(mask)
        P.eng.dynamics_step(30)
        runs.append((P.gpu_state(), P.eng.counters()))
    (a, ca), (b, cb) = runs
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(ca, cb)


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "adaptive_local"])
@pytest.mark.parametrize("shape", [1, 3, 6, 7])
def test_contact_search_forms_match_the_oracle(case, shape):
    """The contact search by (sweeper, neighbour column) within a warp (1),
    balanced over the block (3) and over the global sweeper list (6, 7): the
    float64 path reproduces the oracle bit for bit with each."""
    P = Pair(cases.get(case), precision=64, photons=False)
    assert P.eng.set_launch_shapes([-1, -1, shape])["k_contacts"]["candidate"] == shape
    for t in range(40):
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        if t % 10 == 9:
            compare_state(P.gpu_state(), P.orc, F64_TOL)
    g = P.eng.counters()[0]
    assert np.array_equal(g[:6], P.orc.counters[:6]), (g[:6], P.orc.counters[:6])
    assert P.orc.counters[2] > 0, "no catalytic events: the test would not exercise the contact lists"
    assert P.eng.status() == 0
