"""Small seeded test systems (YAML-equivalent dicts) shared by the tests."""
from __future__ import annotations

import copy

from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W


def rich_small(seed: int = 7, box: float = 3.0, rate_scale: float = 500.0) -> dict:
    """PIP3/PTEN chemistry at ~1,200 particles with rates scaled up so that
    catalysis, recruitment, detachment and conversions all fire within tens
    of steps; dark counts and afterpulsing switched on."""
    d = W.membrane_pip3_pten(counts={"PIP2": 600, "PIP3": 120, "PI3K": 60, "PTEN_T1": 150, "PTEN_T2": 80},
                             pools={"PI3K": 60, "PTEN_T1": 100}, box=box, pixels=16, pixel_size_nm=150.0,
                             seed=seed, k_cat_scale=rate_scale)
    for ex in d["compartment_exchanges"]:
        ex["k_on"] *= 400.0
        ex["k_off"] *= 2.0
        ex["max_recruits_per_step"] = 2
    for cv in d["unimolecular_conversions"]:
        cv["rate"] *= 20.0
    d["detector"]["afterpulsing_prob"] = 0.01
    d["detector"]["dark_count_rate"] = 2.0e5
    d["laser"]["power"] = 5.0e-4
    return d


def binding_regions(seed: int = 11) -> dict:
    """A sensor that binds the lipid (A + B -> AB, reversible) inside a box
    with a slow-diffusion disc: exercises binding, dissociation, the sigmoid
    D(x) regions and bond-mode intramolecular FRET."""
    d = W.membrane_pip3_pten(counts={"PIP2": 300, "PIP3": 200, "PI3K": 40, "PTEN_T1": 60, "PTEN_T2": 30},
                             pools={"PI3K": 40, "PTEN_T1": 60}, box=2.5, pixels=16, pixel_size_nm=150.0,
                             seed=seed, k_cat_scale=200.0)
    d["species"].append({"name": "Sensor", "diffusion_coefficient": 0.08, "radius": 3.0})
    d["species"].append({"name": "Sensor_PIP3", "diffusion_coefficient": 0.06, "radius": 3.5})
    d["initial_populations"]["Sensor"] = 150
    d["reactions"] = [{"name": "bind", "reactants": ["Sensor", "PIP3"], "products": ["Sensor_PIP3"],
                       "kon": 5.0, "koff": 40.0, "contact_radius": 20.0}]
    d["diffusion_field"] = {"type": "regions",
                            "regions": [{"shape": "circle", "center": [1.25, 1.25], "radius": 0.6, "D_factor": 0.3}]}
    d["dye_attachments"] = [{"species": "Sensor", "fluorophore": "mTFP1", "labeling_efficiency": 0.9},
                            {"species": "PIP3", "fluorophore": "Venus", "labeling_efficiency": 0.5}]
    d["fret_pairs"] = [{"donor_type": "mTFP1", "acceptor_type": "Venus", "R0": 5.4,
                        "intra_complex_distance": 5.0, "fret_mode": "bond", "intramolecular": False}]
    d["laser"]["power"] = 5.0e-4
    return d


def harmonic_small(seed: int = 5) -> dict:
    """Dense harmonic soft repulsion (many simultaneous overlaps).  Contact
    radii are short (10 nm) so the candidate pair list stays below the
    reference's silent cap of min(30 N, 500000) pairs (dynamics.py:233)."""
    d = W.membrane_pip3_pten(counts={"PIP2": 3000, "PIP3": 300, "PI3K": 100, "PTEN_T1": 200, "PTEN_T2": 100},
                             pools={"PI3K": 50, "PTEN_T1": 50}, box=0.6, potential="harmonic", pixels=8,
                             pixel_size_nm=70.0, seed=seed, k_cat_scale=5000.0)
    for c in d["catalytic_reactions"]:
        c["contact_radius"] = 10.0
    for p in d["potentials"]:
        p["parameters"]["sigma"] = 12.0
        p["parameters"]["spring_constant"] = 2.0e5
        p["parameters"]["interaction_distance"] = 12.0
    return d


def sine_small(seed: int = 3) -> dict:
    d = rich_small(seed=seed)
    d["diffusion_field"] = {"type": "sine_x", "amplitude": 0.5, "wavelength": 5.0}
    return d


def proximity_small(seed: int = 13) -> dict:
    d = rich_small(seed=seed)
    d["fret_pairs"] = [{"donor_type": "mTFP1", "acceptor_type": "Venus", "R0": 5.4, "fret_mode": "proximity",
                        "proximity_radius": 60.0, "proximity_E_high": 0.5, "proximity_E_low": 0.05,
                        "proximity_target_species": "PTEN_T1"}]
    return d


def exchange_heavy(seed: int = 17) -> dict:
    """rich_small with recruitment, detachment and conversion probabilities
    of 0.01-0.9 per step, so that a particle is recruited and detached, or
    converted twice (PTEN_T1 -> PTEN_T2 -> PTEN_T1), within one step."""
    d = rich_small(seed=seed)
    for ex in d["compartment_exchanges"]:
        ex["k_on"] *= 5.0
        ex["k_off"] *= 1000.0
        ex["max_recruits_per_step"] = 8
    for cv in d["unimolecular_conversions"]:
        cv["rate"] *= 400.0
    return d


def adaptive_local(seed: int = 19) -> dict:
    """rich_small with the two script-set switches of the reference's PIP3/PTEN
    wave script: the adaptation field (tau_w shortened to 10 ms so that w
    follows the PIP3 density within the test) and density-biased local PI3K
    recruitment; feedback grids at 1 µm, as that script sets them."""
    d = rich_small(seed=seed)
    for fb in d["feedback_rules"]:
        fb["grid_resolution"] = 1.0
    for ex in d["compartment_exchanges"]:
        ex["k_on"] *= 5.0
    d["_script_attributes"] = {"use_adaptation": True, "adaptation_tau_w": 0.01, "adaptation_K_w": 10.0,
                               "adaptation_n_w": 2.0, "use_local_pi3k_recruitment": True,
                               "recruit_sigma": 0.5}
    return d


CASES = {
    "rich_small": rich_small,
    "binding_regions": binding_regions,
    "harmonic_small": harmonic_small,
    "sine_small": sine_small,
    "proximity_small": proximity_small,
    "exchange_heavy": exchange_heavy,
    "adaptive_local": adaptive_local,
}


def get(name: str) -> dict:
    return copy.deepcopy(CASES[name]())


def jittered_ensemble(n_replicas: int = 8, seed: int = 99, n_min: int = 400, n_max: int = 4000) -> list:
    """Replicas drawn like the batched ensemble (particle count log-uniform,
    box scaled to the membrane density, k_cat and K_half each jittered by
    U(0.5, 1.5), a seed per replica), at sizes the oracle runs in seconds,
    with the rates raised as in rich_small so that catalysis, recruitment,
    detachment and conversions fire within tens of steps.  Every replica keeps
    its own jitter on top of the common scaling."""
    out = []
    for d in W.ensemble_replicas(n_replicas, seed=seed, n_min=n_min, n_max=n_max, pixels=16):
        for c in d["catalytic_reactions"]:
            c["k_cat"] *= 500.0
        for ex in d["compartment_exchanges"]:
            ex["k_on"] *= 400.0
            ex["k_off"] *= 2.0
            ex["max_recruits_per_step"] = 2
        for cv in d["unimolecular_conversions"]:
            cv["rate"] *= 200.0
        d["laser"]["power"] = 5.0e-4
        out.append(d)
    return out


def free_diffusion(n_per_species: int = 20000, seed: int = 123) -> dict:
    """Two species without forces or reactions (D = 1.0 and 0.05 µm^2/s) in a
    periodic 100x100 µm^2 box at dt = 0.1 ms: the reference's MSD = 4Dt check
    (tests/test_dynamics.py:130-213), with more particles per species."""
    return {"name": "free diffusion", "membrane": {"size": [100.0, 100.0], "periodic": [True, True]},
            "species": [{"name": "A", "diffusion_coefficient": 1.0, "radius": 1.0},
                        {"name": "B", "diffusion_coefficient": 0.05, "radius": 1.0}],
            "initial_populations": {"A": n_per_species, "B": n_per_species},
            "bd_timestep": 1e-4, "simulation_time": 0.1, "random_seed": seed}
