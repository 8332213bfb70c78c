"""Sub-frame record and per-frame ground truth on the device, against the
reference.

The golden fixtures hold, for each test system, the reference's own per-step
sub-frame series (pipeline.py:567-642) over 24 BD steps with keyed draws,
and the ground truth of the frame (its _extract_ground_truth after
update_fret_rates).  The engine records one census row per step inside its
CUDA-graph chunks (edm_record_enable / edm_record_read) and evaluates the
ground truth on the device (edm_ground_truth).  Integer series and the
ground-truth arrays must be identical; the mean FRET efficiency, a sum over
donors taken in another order, within 1e-12 relative.
"""
from pathlib import Path

import numpy as np
import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
from tests import cases
from tests.harness import Pair

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["rich_small", "binding_regions", "proximity_small", "exchange_heavy"])
@pytest.mark.parametrize("precision", [64, 32])
def test_recorded_subframe_series_and_ground_truth_match_reference(name, precision):
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200.api import subframe_series
    g = dict(np.load(GOLDEN / f"{name}.npz"))
    P = Pair(cases.get(name), precision=precision)
    eng = P.eng
    eng.record_enable(24)
    s = torch.cuda.Stream()
    prev = eng.counters(stream=s)[0][:7].copy()
    eng.pipeline_steps(24, True, 8, stream=s)  # three captured chunks of 8 steps
    rows = eng.record_read(0, 24, stream=s)[:, 0, :]
    e_cls = np.array(eng._phot[0].fret_E[0][:PR.MAX_FCLASS])
    ser = subframe_series(rows, prev, P.cfg, e_cls)
    if precision == 64:  # float32 trajectories may part from the reference's after a few steps
        for k in ("n_complexes", "n_bindings", "n_dissociations", "n_bleached", "total_photons", "n_catalytic",
                  "n_recruited", "n_detached", "n_converted"):
            assert np.array_equal(ser[k], g[f"sf_{k}"]), (k, ser[k], g[f"sf_{k}"])
        for i, sp in enumerate(P.cfg.species):
            assert np.array_equal(ser["species"][sp.name], g["sf_species"][:, i]), sp.name
        np.testing.assert_allclose(ser["mean_fret_E"], g["sf_mean_fret_E"], rtol=1e-12, atol=0)
    eng.finalize(0, stream=s)
    fret_E, tau_DA, census = eng.ground_truth(stream=s)
    st = eng.get_state(stream=s)
    c = census[0]
    # the census always describes the engine's own state
    assert int(c[PR.CEN_BOND_ALL]) == int(np.sum(st["bond"] >= 0))
    assert int(c[PR.CEN_BLEACHED]) == int(np.sum(st["bleached"]))
    for i in range(len(P.cfg.species)):
        assert int(c[PR.CEN_SPECIES + i]) == int(np.sum((st["species"] == i) & st["alive"].astype(bool)))
    if precision == 64:
        assert np.array_equal(fret_E, g["gt_fret_E"])
        assert np.array_equal(tau_DA, g["gt_tau_DA"])
        assert int(c[PR.CEN_BOND_ALL]) // 2 == int(g["gt_n_complexes"])
        assert int(c[PR.CEN_BLEACHED]) == int(g["gt_n_bleached"])
        n_free = sum(int(c[PR.CEN_FREE_DYE + fi]) for fp in P.cfg.fret_pairs
                     for fi, f in enumerate(P.cfg.fluorophores) if f.name == fp.donor_type)
        assert n_free == int(g["gt_n_free_donors"])
        assert np.array_equal(c[PR.CEN_SPECIES:PR.CEN_SPECIES + len(P.cfg.species)], g["gt_species_counts"])
    eng.record_enable(0)


def test_recorded_series_of_a_jittered_ensemble_match_oracle_replicas():
    """Census rows of 8 replicas in one engine: each replica's rows equal the
    reference expressions on an oracle run of that replica alone."""
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200.api import subframe_series
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
    from oracle import oracle as O
    from tests import census as CS
    raws = cases.jittered_ensemble(8)
    ens = Ensemble(raws, precision=64, photons=True, device=0)
    eng = ens.engine
    steps = 20
    eng.record_enable(steps)
    s = torch.cuda.Stream()
    prev_all = eng.counters(stream=s)[:, :7].copy()
    eng.pipeline_steps(steps, True, 10, stream=s)
    rows = eng.record_read(0, steps, stream=s)
    gt_E, gt_tau, gt_cen = eng.ground_truth(stream=s)
    for r, cfg in enumerate(ens.configs):
        st = ParticleState(cfg)
        dp, _, _ = PR.build_dyn_params(cfg, st.N)
        duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
        _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
        sp, _ = PR.build_scope_params(cfg)
        orc = O.OracleSimulation(cfg, st, dp, pd, sp, duty)
        ser = subframe_series(rows[:, r, :], prev_all[r], cfg, np.array(eng._phot[r].fret_E[0][:PR.MAX_FCLASS]))
        prev = orc.counters[:6].copy()
        for t in range(steps):
            batch = orc.bd_step()
            want = CS.subframe_step(orc, cfg, batch[0].size, prev, pd.tau_all[0])
            prev = orc.counters[:6].copy()
            for k, v in want.items():
                if k == "species":
                    got = np.array([ser["species"][sp_.name][t] for sp_ in cfg.species])
                    assert np.array_equal(got, v), (r, t)
                elif k == "mean_fret_E":
                    assert abs(ser[k][t] - v) <= 1e-12 * abs(v), (r, t, ser[k][t], v)
                else:
                    assert ser[k][t] == v, (r, t, k, ser[k][t], v)
        gt = CS.ground_truth(orc, cfg, pd)
        sl = ens.replica_slice(r)
        assert np.array_equal(gt_E[sl], gt["fret_E"]) and np.array_equal(gt_tau[sl], gt["tau_DA"]), r
        assert int(gt_cen[r][PR.CEN_BOND_ALL]) // 2 == gt["n_complexes"]
        assert int(gt_cen[r][PR.CEN_BLEACHED]) == gt["n_bleached"]
        assert np.array_equal(gt_cen[r][PR.CEN_SPECIES:PR.CEN_SPECIES + len(cfg.species)], gt["species"])
    eng.record_enable(0)


def test_pipeline_run_with_subframe_recording_keeps_graphs_and_matches_plain_run():
    """SimulationPipeline.run(record_subframe=True) steps through the same
    CUDA-graph chunks as a run without recording: identical frames, and the
    recorded series add up to the frame counters."""
    from flim_microscopy_simulator_with_causal_inference_b200.api import SimulationPipeline
    from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
    raw = cases.get("binding_regions")
    raw["scan"]["n_frames"] = 3
    raw["scan"]["frame_interval"] = 20 * raw["bd_timestep"]
    raw["simulation_time"] = 3 * raw["scan"]["frame_interval"]
    runs = {}
    for rec in (False, True):
        pipe = SimulationPipeline(config_from_dict(raw), progress_callback=lambda *a: None, record_subframe=rec,
                                  precision=64, graph_chunk=10)
        runs[rec] = pipe.run()
    a, b = runs[False], runs[True]
    for fa, fb in zip(a.frames, b.frames):
        assert np.array_equal(fa.flim_frame.flim_stack, fb.flim_frame.flim_stack)
        assert np.array_equal(fa.ground_truth.positions, fb.ground_truth.positions)
        assert np.array_equal(fa.ground_truth.fret_efficiency_exact, fb.ground_truth.fret_efficiency_exact)
        assert fa.ground_truth.n_complexes == fb.ground_truth.n_complexes
    sf = b.subframe_data
    assert sf is not None and sf.n_complexes.size == 60
    assert int(sf.total_photons.sum()) == b.total_photons_emitted
    assert int(sf.n_bindings.sum()) == b.total_bindings and int(sf.n_dissociations.sum()) == b.total_dissociations
