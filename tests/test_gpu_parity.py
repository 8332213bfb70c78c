"""CUDA engine vs the CPU oracle (the reference's algorithm restated in C).

float64 path: same inputs, same keyed noise -> identical cell lists, event
sets, counters and photon streams; positions equal to <= 1e-12 µm (bit-exact
except where the device's exp/sin/log differ from the host libm by an ulp:
the D(x) field and photon arrival times).
float32 path (cell-relative positions): lockstep, i.e. the oracle's state is
loaded before every step; positions within 1e-5 µm per step, identical event
sets.
"""
import numpy as np
import pytest

from tests import cases
from tests.harness import Pair, compare_state, cell_sets_oracle

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12      # µm, float64 path vs oracle, free running
F32_TOL = 1e-5       # µm per step, float32 path vs oracle, lockstep


def test_noise_streams_bit_identical():
    from flim_microscopy_simulator_with_causal_inference_b200.engine import device_normals, device_uniforms
    from oracle import oracle as O
    keys = np.arange(0, 200000, 7, dtype=np.int64)
    for seed, step, stream in ((42, 0, 1), (2 ** 40 + 3, 123456789012, 122), (7, 5, 32)):
        assert np.array_equal(device_normals(seed, step, stream, keys), O.normals(seed, step, stream, keys))
        b = keys[::-1].copy()
        assert np.array_equal(device_uniforms(seed, step, stream, keys, b), O.uniforms(seed, step, stream, keys, b, two=True))


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "harmonic_small", "exchange_heavy",
                                  "adaptive_local"])
def test_fp64_free_running_matches_oracle(case):
    P = Pair(cases.get(case), precision=64)
    steps = 40
    for t in range(steps):
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        if t % 10 == 9 or t == 0:
            compare_state(P.gpu_state(), P.orc, F64_TOL)
    g = P.eng.counters()[0]
    assert np.array_equal(g[:6], P.orc.counters[:6]), (g[:6], P.orc.counters[:6])
    if case in ("rich_small", "binding_regions"):
        assert P.orc.counters[:6].sum() > 0, "test system produced no reaction events"
    if case == "exchange_heavy":  # recruitments, detachments and conversions all fired
        assert (P.orc.counters[3:6] > 0).all(), P.orc.counters[:6]
        assert P.eng.status() == 0
    if case == "adaptive_local":  # catalysis under adaptation and local recruitment both fired
        assert P.orc.counters[2] > 0 and P.orc.counters[3] > 0, P.orc.counters[:6]


def test_fp64_cell_lists_match_oracle():
    P = Pair(cases.get("rich_small"), precision=64)
    for _ in range(3):
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        start, mem = P.eng.cells(0)
        gsets = [sorted(mem[start[c]:start[c + 1]].tolist()) for c in range(P.dp.nx * P.dp.ny)]
        assert gsets == cell_sets_oracle(P.orc, P.dp.nx, P.dp.ny)


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "proximity_small"])
def test_fp64_pipeline_photons_and_tcspc_match_oracle(case):
    P = Pair(cases.get(case), precision=64)
    total = 0
    for t in range(30):
        P.eng.dynamics_step(1)
        P.eng.photon_step()
        P.eng.scope_process()
        ob = P.orc.bd_step()
        pid, tt, ch, fr = P.eng.photons(0)
        assert np.array_equal(pid, ob[0]), f"photon emitters differ at step {t}"
        assert np.array_equal(ch, ob[2]) and np.array_equal(fr, ob[3])
        np.testing.assert_allclose(tt, ob[1], rtol=1e-14, atol=0)
        total += pid.size
        if t % 10 == 9:
            assert np.array_equal(P.eng.flim(0), P.orc.flim), f"TCSPC stacks differ at step {t}"
    assert total > 0
    P.eng.finalize(0)
    of = P.orc.finalize_frame()
    assert np.array_equal(P.eng.flim(0), of)
    compare_state(P.gpu_state(), P.orc, F64_TOL)


def test_fp64_graph_chunks_match_eager():
    raw = cases.get("rich_small")
    A = Pair(raw, precision=64)
    B = Pair(raw, precision=64)
    import torch
    s = torch.cuda.Stream()
    A.eng.pipeline_steps(40, True, 10, stream=s)
    s.synchronize()
    B.eng.pipeline_steps(40, True, 0)
    ga, gb = A.gpu_state(), B.gpu_state()
    for k in ga:
        assert np.array_equal(ga[k], gb[k]), k
    assert np.array_equal(A.eng.flim(0), B.eng.flim(0))
    assert np.array_equal(A.eng.counters(), B.eng.counters())


@pytest.mark.parametrize("case", ["rich_small", "binding_regions", "sine_small", "exchange_heavy",
                                  "adaptive_local"])
def test_fp32_lockstep_matches_oracle(case):
    P = Pair(cases.get(case), precision=32)
    worst = 0.0
    for t in range(25):
        P.load_oracle_state_into_gpu()
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        worst = max(worst, compare_state(P.gpu_state(), P.orc, F32_TOL))
    assert worst < F32_TOL


def test_sine_field_fp64_close():
    P = Pair(cases.get("sine_small"), precision=64)
    for t in range(20):
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
    compare_state(P.gpu_state(), P.orc, 1e-9)


def test_determinism_two_runs_bitwise():
    raw = cases.get("rich_small")
    runs = []
    for _ in range(2):
        P = Pair(raw, precision=32)
        P.eng.pipeline_steps(30, True, 0)
        runs.append((P.gpu_state(), P.eng.flim(0), P.eng.counters()))
    for k in runs[0][0]:
        assert np.array_equal(runs[0][0][k], runs[1][0][k]), k
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


def test_fp64_proximity_photons_before_any_dynamics_step():
    """Proximity FRET right after the state is set (no cell list yet): the
    all-pairs search gives the oracle's photons."""
    P = Pair(cases.get("proximity_small"), precision=64)
    P.eng.photon_step()
    ob = P.orc.photon_step()
    pid, tt, ch, fr = P.eng.photons(0)
    assert pid.size > 0
    assert np.array_equal(pid, ob[0]) and np.array_equal(ch, ob[2]) and np.array_equal(fr, ob[3])
    np.testing.assert_allclose(tt, ob[1], rtol=1e-14, atol=0)


def test_fp32_lockstep_large_membrane_no_cell_jumps():
    """The float32 path against the float64 path on the 1.3M-particle membrane
    (1.86M with pools), one step at a time from the float64 state: positions
    within 1e-5 µm per step with identical species and alive flags.  This
    covers strongly overlapping harmonic pairs, whose moves hit the
    displacement cap and keep only the direction of the pair force, and
    particles whose offset lands within rounding of a cell's lower side,
    which must stay there, not a cell (0.165 µm) away."""
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    raw = W.config2(n_frames=1)
    s = torch.cuda.Stream()
    ens = {p: Ensemble([raw], precision=p, photons=True, device=0) for p in (32, 64)}
    e32, e64 = ens[32].engine, ens[64].engine
    dye = ens[64].host["dye"]
    e64.pipeline_steps(5, True, 0, stream=s)
    worst = 0.0
    for _ in range(4):
        st = e64.get_state(stream=s)
        e32.set_state(st["positions"], st["species"], st["alive"], st["bond"], st["has_dye"], dye, st["ctmc"],
                      st["bleached"], stream=s)
        e32.set_step(e64.get_step())
        e64.pipeline_steps(1, True, 0, stream=s)
        e32.pipeline_steps(1, True, 0, stream=s)
        a64, a32 = e64.get_state(stream=s), e32.get_state(stream=s)
        assert np.array_equal(a32["species"], a64["species"]) and np.array_equal(a32["alive"], a64["alive"])
        d = np.abs(a32["positions"] - a64["positions"])
        d = np.minimum(d, 100.0 - d)  # periodic 100 µm box
        worst = max(worst, float(d.max()))
    assert worst < F32_TOL, worst
    del ens
    torch.cuda.empty_cache()
