"""Configuration loader: same defaults and errors as the reference's
(ed_mrdt/config.py:579-1094); engine-unsupported features fail loudly."""
import copy

import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
from flim_microscopy_simulator_with_causal_inference_b200.config import ConfigError, config_from_dict, load_config
from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState


def test_defaults_not_read_from_yaml():
    cfg = config_from_dict(W.config0())
    assert cfg.displacement_cap_fraction == 0.5
    assert cfg.region_smoothing_width == 0.05
    assert cfg.psf.sigma_xy == 0.0
    assert cfg.tcspc.bin_width == 2.5e-8 / 256


def test_unknown_species_reference_raises():
    raw = W.config0()
    raw["catalytic_reactions"][0]["enzyme"] = "NOPE"
    with pytest.raises(ConfigError, match="NOPE"):
        config_from_dict(raw)


def test_bad_basal_fraction_raises():
    raw = W.config0()
    raw["feedback_rules"][0]["basal_fraction"] = 1.5
    with pytest.raises(ConfigError, match="basal_fraction"):
        config_from_dict(raw)


def test_keq_mode_derives_kon():
    raw = W.config0()
    raw["reactions"] = [{"name": "b", "reactants": ["PIP3", "PI3K"], "products": ["PIP2"], "Keq": 2.0, "koff": 0.5}]
    cfg = config_from_dict(raw)
    assert cfg.reactions[0].kon == 1.0


def test_f_bound_mode_requires_ligand_density():
    raw = W.config0()
    raw["reactions"] = [{"name": "b", "reactants": ["PIP3", "PI3K"], "products": ["PIP2"], "f_bound": 0.5,
                         "koff": 0.5}]
    with pytest.raises(ConfigError, match="ligand_density"):
        config_from_dict(raw)


def test_missing_file(tmp_path):
    with pytest.raises(FileNotFoundError):
        load_config(tmp_path / "none.yaml")


def test_yaml_roundtrip(tmp_path):
    import yaml
    p = tmp_path / "c.yaml"
    p.write_text(yaml.safe_dump(W.config0()))
    cfg = load_config(p)
    assert cfg.n_species == 5 and cfg.initial_populations["PIP2"] == 2500


def test_particle_layout_pools_and_dyes():
    cfg = config_from_dict(W.config0())
    st = ParticleState(cfg)
    assert st.N == 3500 + 1500
    assert int(st.is_alive.sum()) == 3500
    assert int(st.has_dye.sum()) == 125  # PIP3 labelled with efficiency 1
    assert st.species_ranges["PIP2"] == (0, 2500)


def test_unsupported_features_fail_loudly():
    # config 0's 0.5 µm feedback grids are larger than the 1 µm adaptation grid: the reference would read
    # past its adaptation array there (dynamics.py:1078)
    cfg = config_from_dict(W.config0())
    cfg.use_adaptation = True
    with pytest.raises(NotImplementedError, match="adaptation"):
        PR.build_dyn_params(cfg, 10)
    raw = W.config0()
    raw["catalytic_reactions"][0]["product"] = "PI3K"
    with pytest.raises(NotImplementedError):
        PR.build_dyn_params(config_from_dict(raw), 10)


def test_workload_sizes():
    c1 = W.config1()
    assert sum(c1["initial_populations"].values()) == 13000
    c2 = W.config2()
    assert sum(c2["initial_populations"].values()) == 1_300_000
    reps = W.ensemble_replicas(64, seed=1)
    n = [sum(r["initial_populations"].values()) for r in reps]
    assert min(n) >= 1000 and max(n) <= 50000


def test_script_attributes_and_adaptation_plan():
    raw = W.config0()
    for fb in raw["feedback_rules"]:
        fb["grid_resolution"] = 1.0
    raw["_script_attributes"] = {"use_adaptation": True, "adaptation_tau_w": 30.0, "adaptation_K_w": 5.0,
                                 "adaptation_n_w": 3.0, "use_local_pi3k_recruitment": True, "recruit_sigma": 0.25}
    cfg = config_from_dict(raw)
    assert cfg.use_adaptation and cfg.use_local_pi3k_recruitment and cfg.recruit_sigma == 0.25
    P, _, d = PR.build_dyn_params(cfg, 5000)
    names = [s.name for s in cfg.species]
    # the adaptation grid counts PIP3 on max(3, int(L / 1 µm)) cells per side; here it is the PIP3 feedback grid
    g = d.grids[d.adapt_grid]
    assert g[0] == names.index("PIP3") and (g[1], g[2]) == (10, 10)
    assert P.adapt_grid == d.adapt_grid and P.adapt_inv_tau == cfg.bd_timestep / 30.0
    assert (P.adapt_K, P.adapt_n, P.recruit_sigma) == (5.0, 3.0, 0.25)
    # only catalytic reactions whose enzyme name holds 'PI3K' (and have feedback) are modulated
    mask = [k for k, c in enumerate(cfg.catalytic_reactions) if "PI3K" in c.enzyme and d.catalytic[k]["rule"] >= 0]
    assert P.adapt_cat_mask == sum(1 << k for k in mask) and mask
    # local recruitment: single feedback rules named '...pip3_activation...'
    for ex, e in zip(cfg.compartment_exchanges, P.exch[:P.n_exch]):
        want = bool(ex.feedback_rule) and "pip3_activation" in ex.feedback_rule and not ex.secondary_feedback_rule
        assert e.local_recruit == int(want), ex.name
    assert any(e.local_recruit for e in P.exch[:P.n_exch])


def test_unknown_script_attribute_rejected():
    raw = W.config0()
    raw["_script_attributes"] = {"use_adaptaton": True}
    with pytest.raises(ConfigError, match="unknown script attribute"):
        config_from_dict(raw)
