"""The oracle and the host constant derivation, pinned to the reference.

Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from
the reference itself with keyed draws injected) hold the reference's derived
constants and its state after 10 and 24 BD steps.  These CPU tests rebuild
each system with this package's config / ParticleState / parameter builder,
replay the same steps on the oracle and require bit equality.
"""
from pathlib import Path

import numpy as np
import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
from oracle import oracle as O
from tests import cases

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = sorted(cases.CASES)


def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def _build(name):
    cfg = config_from_dict(cases.get(name))
    st = ParticleState(cfg)
    return cfg, st


@pytest.mark.parametrize("name", NAMES)
def test_initial_state_matches_reference(name):
    g = _load(name)
    _, st = _build(name)
    assert np.array_equal(st.positions, g["init_positions"])
    assert np.array_equal(st.species_id, g["init_species"])
    assert np.array_equal(st.is_alive, g["init_alive"])
    assert np.array_equal(st.has_dye, g["init_has_dye"])
    assert np.array_equal(st.dye_type_id, g["init_dye"])


@pytest.mark.parametrize("name", NAMES)
def test_derived_constants_match_reference(name):
    g = _load(name)
    cfg, st = _build(name)
    dp, hill, d = PR.build_dyn_params(cfg, st.N)
    assert d.cutoff_um == g["cutoff_um"]
    assert d.max_displacement == g["max_displacement"]
    assert (d.nx, d.ny) == (int(g["nx"]), int(g["ny"]))
    assert np.array_equal([c["prob"] for c in d.catalytic], g["prob_cat"])
    assert np.array_equal([e["prob_on"] for e in d.exchanges], g["prob_on"])
    assert np.array_equal([e["prob_off"] for e in d.exchanges], g["prob_off"])
    assert np.array_equal([c["prob"] for c in d.conversions], g["prob_conv"])
    assert np.array_equal([r["prob_bind"] for r in d.reactions], g["prob_bind"])
    duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
    _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
    for k, v in (("T_step", pd.T_step), ("T_step_fret", pd.T_step_fret), ("mean_ph", pd.mean_ph),
                 ("mean_ph_fret", pd.mean_ph_fret), ("mean_fret", pd.mean_fret), ("tau_all", pd.tau_all),
                 ("k_fret_bound", pd.k_fret_bound)):
        assert np.array_equal(v, g[k]), k
    assert pd.max_photons == int(g["max_photons"])
    _, sd = PR.build_scope_params(cfg)
    assert np.array_equal([sd.sigma_um[k] for k in sorted(sd.sigma_um)], g["psf_sigma"])
    assert sd.psf_range_px == int(g["psf_range_px"])
    assert sd.sigma_irf == float(g["sigma_irf"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_replays_reference_bit_exact(name):
    g = _load(name)
    cfg, st = _build(name)
    dp, hill, d = PR.build_dyn_params(cfg, st.N)
    duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
    _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
    sp, _ = PR.build_scope_params(cfg)
    orc = O.OracleSimulation(cfg, st, dp, pd, sp, duty)
    batch = None
    for t in range(24):
        batch = orc.bd_step()
        if t + 1 == 10:
            assert np.array_equal(orc.pos, g["snap_positions"])
            assert np.array_equal(orc.species, g["snap_species"])
            assert np.array_equal(orc.alive.astype(bool), g["snap_alive"])
    flim = orc.finalize_frame()
    assert np.array_equal(orc.pos, g["final_positions"])
    assert np.array_equal(orc.species, g["final_species"])
    assert np.array_equal(orc.alive.astype(bool), g["final_alive"])
    assert np.array_equal(orc.bond, g["final_bond"])
    assert np.array_equal(orc.ctmc, g["final_ctmc"])
    assert np.array_equal(orc.bleached.astype(bool), g["final_bleached"])
    assert np.array_equal(orc.counters[:6], g["counters"])
    assert np.array_equal(batch[0], g["last_batch_particle"])
    assert np.array_equal(batch[1], g["last_batch_time"])
    assert np.array_equal(batch[2], g["last_batch_channel"])
    assert np.array_equal(flim, g["flim"])
    assert orc.last_dark == int(g["n_dark"]) and orc.last_ap == int(g["n_ap"])
    assert orc.scope_stats.n_detected == int(g["photons_detected"])


def test_hill_table_is_sequential_density_sum():
    """The tabulated Hill factor at count k equals the reference expression
    at the k-fold sequential float64 sum of 1/cell_area."""
    inv_area = 1.0 / (0.5 * 0.5)
    tab = PR.hill_table(inv_area, 15.0, 2.0, False, 0.05, 64)
    rho = 0.0
    for k in range(64):
        ratio = rho / 15.0
        rn = ratio ** 2.0
        assert tab[k] == 0.05 + (1.0 - 0.05) * (rn / (1.0 + rn))
        rho += inv_area


@pytest.mark.parametrize("name", NAMES)
def test_oracle_subframe_series_and_ground_truth_match_reference(name):
    """The reference's per-step sub-frame record and frame ground truth
    (golden sf_* / gt_*, from its own state and _extract_ground_truth) equal
    the same expressions on the oracle's replay."""
    from tests import census as CS
    g = _load(name)
    cfg, st = _build(name)
    dp, hill, d = PR.build_dyn_params(cfg, st.N)
    duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
    _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
    sp, _ = PR.build_scope_params(cfg)
    orc = O.OracleSimulation(cfg, st, dp, pd, sp, duty)
    prev = orc.counters[:6].copy()
    for t in range(24):
        batch = orc.bd_step()
        row = CS.subframe_step(orc, cfg, batch[0].size, prev, pd.tau_all[0])
        prev = orc.counters[:6].copy()
        for k, v in row.items():
            if k == "species":
                assert np.array_equal(v, g["sf_species"][t]), (t, k)
            else:
                assert v == g[f"sf_{k}"][t], (t, k, v, g[f"sf_{k}"][t])
    orc.finalize_frame()
    gt = CS.ground_truth(orc, cfg, pd)
    assert np.array_equal(gt["fret_E"], g["gt_fret_E"])
    assert np.array_equal(gt["tau_DA"], g["gt_tau_DA"])
    assert gt["n_complexes"] == int(g["gt_n_complexes"])
    assert gt["n_bleached"] == int(g["gt_n_bleached"])
    assert gt["n_free_donors"] == int(g["gt_n_free_donors"])
    assert np.array_equal(gt["species"], g["gt_species_counts"])
