"""The benchmarked configurations on the GPU against the CPU oracle.

* The 10x10 µm^2 PIP3/PTEN membrane (3,500 membrane + 1,500 dormant
  particles, WCA, 150 nm contacts, 64x64 px) and its 13,000-particle version
  with the sine D(x) field (128x128 px): 40 free-running float64 BD steps with
  photons and detection, then 25 float32 steps in lockstep (the oracle's state
  loaded before every step).
* A batched ensemble of 8 replicas drawn like the headline ensemble (uneven
  particle counts, boxes scaled to the density, per-replica k_cat / K_half
  jitter and seeds) in ONE engine: every replica's float64 state, counters and
  TCSPC stack after 30 pipeline steps (CUDA-graph chunks) must equal an oracle
  run of that replica alone.  This checks the replica-offset layout (particle,
  cell, grid, Hill-table, photon and stack offsets) and the per-replica draw
  thresholds behind the benchmark's number.
* Free diffusion on the float32 path: MSD = 4 D t (the reference's
  tests/test_dynamics.py:130-213 check, with its 5 % and 10 % bounds).

Tolerances: float64 free running <= 1e-12 µm (<= 1e-9 µm with the sine field,
whose device sin/cos may differ from the host's by an ulp); float32 lockstep
<= 1e-5 µm per step; event sets, counters, photon streams and TCSPC stacks
identical.
"""
import numpy as np
import pytest

from tests import cases
from tests.harness import Pair, compare_state

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
SINE_TOL = 1e-9
F32_TOL = 1e-5


def _configs():
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    return {"membrane_10um": (W.config0(), F64_TOL),
            "membrane_13k_sine": (W.config1(n_frames=1), SINE_TOL)}


@pytest.mark.parametrize("name", ["membrane_10um", "membrane_13k_sine"])
def test_benchmark_config_fp64_free_running_matches_oracle(name):
    raw, tol = _configs()[name]
    P = Pair(raw, precision=64)
    photons = 0
    for t in range(40):
        P.eng.dynamics_step(1)
        P.eng.photon_step()
        P.eng.scope_process()
        ob = P.orc.bd_step()
        pid, tt, ch, fr = P.eng.photons(0)
        assert np.array_equal(pid, ob[0]), f"photon emitters differ at step {t}"
        assert np.array_equal(ch, ob[2]) and np.array_equal(fr, ob[3])
        np.testing.assert_allclose(tt, ob[1], rtol=1e-14, atol=0)
        photons += pid.size
        if t % 10 == 9:
            compare_state(P.gpu_state(), P.orc, tol)
    assert photons > 0
    assert np.array_equal(P.eng.counters()[0][:6], P.orc.counters[:6])
    P.eng.finalize(0)
    assert np.array_equal(P.eng.flim(0), P.orc.finalize_frame()), "TCSPC stacks differ"


@pytest.mark.parametrize("name", ["membrane_10um", "membrane_13k_sine"])
def test_benchmark_config_fp32_lockstep_matches_oracle(name):
    raw, _ = _configs()[name]
    P = Pair(raw, precision=32, photons=False)
    worst = 0.0
    for _ in range(25):
        P.load_oracle_state_into_gpu()
        P.eng.dynamics_step(1)
        P.orc.dynamics_step()
        P.orc.step_index += 1
        worst = max(worst, compare_state(P.gpu_state(), P.orc, F32_TOL))
    assert worst < F32_TOL


def test_jittered_ensemble_replicas_match_oracle_one_by_one():
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
    from oracle import oracle as O
    raws = cases.jittered_ensemble(8)
    ens = Ensemble(raws, precision=64, photons=True, device=0)
    assert len(set(ens.n_particles.tolist())) == ens.R  # uneven sizes
    steps = 30
    s = torch.cuda.Stream()
    ens.engine.pipeline_steps(steps, True, 10, stream=s)
    g = ens.engine.get_state(stream=s)
    counters = ens.engine.counters(stream=s)
    fired = np.zeros(6, dtype=np.int64)
    for r, cfg in enumerate(ens.configs):
        st = ParticleState(cfg)
        dp, _, _ = PR.build_dyn_params(cfg, st.N)
        duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
        _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
        sp, _ = PR.build_scope_params(cfg)
        orc = O.OracleSimulation(cfg, st, dp, pd, sp, duty)
        for _ in range(steps):
            orc.bd_step()
        sl = ens.replica_slice(r)
        gr = {k: v[sl] for k, v in g.items()}
        compare_state(gr, orc, F64_TOL)
        assert np.array_equal(counters[r][:6], orc.counters[:6]), (r, counters[r][:6], orc.counters[:6])
        assert np.array_equal(ens.engine.flim(r, stream=s), orc.flim), f"TCSPC stack of replica {r} differs"
        fired += orc.counters[:6]
    assert (fired[2:6] > 0).all(), fired  # catalysis, recruitment, detachment and conversion all fired


@pytest.mark.parametrize("precision", [32, 64])
def test_free_diffusion_msd_is_4Dt(precision):
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    ens = Ensemble([cases.free_diffusion()], precision=precision, photons=False, device=0)
    eng = ens.engine
    s = torch.cuda.Stream()
    start = eng.get_state(stream=s)
    prev = start["positions"].copy()
    unwrapped = prev.copy()
    steps = 1000
    for _ in range(steps // 100):  # unwrap every 100 steps (<= 0.3 µm apart, box 100 µm)
        eng.pipeline_steps(100, False, 100, stream=s)
        p = eng.get_state(stream=s)["positions"]
        d = p - prev
        unwrapped += d - 100.0 * np.round(d / 100.0)
        prev = p.copy()
    r2 = np.sum((unwrapped - start["positions"]) ** 2, axis=1)
    t = steps * 1e-4
    species = start["species"]
    for sp, D, bound in ((0, 1.0, 0.05), (1, 0.05, 0.10)):
        msd = r2[species == sp].mean()
        assert abs(msd - 4.0 * D * t) < bound * 4.0 * D * t, (precision, D, msd, 4.0 * D * t)
