"""Synthetic workloads of the benchmark configurations, as YAML-equivalent dicts.

There is no public dataset for this path; these seeded synthetic systems are
the workload.  All derive from the PIP3/PTEN chemistry of the reference's
shipped `ed_mrdt/examples/pip3_pten_flim.yaml` with the parameters stated for
the benchmark:

* membrane_pip3_pten(...)   -- the 10x10 µm^2 PIP3/PTEN membrane ("config 0"),
  scalable in particle count ("config 1": 13,000 membrane particles) and box
  size ("config 2": 100x100 µm^2, 1.3M particles, harmonic repulsion);
* ensemble_replicas(...)    -- "config 3": replicas with log-uniform particle
  counts, box side scaled to keep the density, k_cat and K_half jittered;
* the FLIM-acquisition workload ("config 4") lives in flim_acquire.py.

Open choices of the benchmark description, fixed here:
* dwell_time 20 µs and frame_interval = 100 BD steps (scan duty 2e-3);
* the donor FRET pair keeps the shipped bond-mode pair (R0 5.4 nm at 5.0 nm,
  E = 0.6134); with no binding reaction every donor is unquenched;
* config 1/2 keep the config-0 species ratios; cytosolic pools scale with
  the membrane count (500 PI3K and 1000 PTEN_T1 per 3,500 membrane particles);
* "config-0 densities" for 1.3M particles on 100x100 µm^2 is read as the
  config-1 areal density (130 /µm^2), the one consistent with 1.3M.
"""
from __future__ import annotations

import copy
import math
from typing import Dict, List, Optional

import numpy as np

C0_COUNTS = {"PIP2": 2500, "PIP3": 125, "PI3K": 125, "PTEN_T1": 500, "PTEN_T2": 250}
C0_POOLS = {"PI3K": 500, "PTEN_T1": 1000}

_FLUOROPHORES = [
    {"name": "mTFP1",
     "states": [{"name": "S0", "is_fluorescent": False, "is_absorbing": True},
                {"name": "S1", "is_fluorescent": True, "quantum_yield": 0.85, "emission_wavelength": 492.0},
                {"name": "T1", "is_fluorescent": False, "is_absorbing": False},
                {"name": "bleached", "is_fluorescent": False, "is_absorbing": False, "is_terminal": True}],
     "thermal_rates": {"S1": {"S0": 3.57e8, "T1": 1.0e6, "bleached": 1.0e3},
                       "T1": {"S0": 1.0e4, "bleached": 1.0e2}},
     "absorption_cross_section": 2.5e-16, "excitation_wavelength": 462.0},
    {"name": "Venus",
     "states": [{"name": "S0", "is_fluorescent": False, "is_absorbing": True},
                {"name": "S1", "is_fluorescent": True, "quantum_yield": 0.57, "emission_wavelength": 528.0},
                {"name": "T1", "is_fluorescent": False, "is_absorbing": False},
                {"name": "bleached", "is_fluorescent": False, "is_absorbing": False, "is_terminal": True}],
     "thermal_rates": {"S1": {"S0": 3.33e8, "T1": 5.0e5, "bleached": 5.0e2},
                       "T1": {"S0": 5.0e3, "bleached": 50.0}},
     "absorption_cross_section": 1.5e-16, "excitation_wavelength": 515.0},
]

_SPECIES = ["PIP2", "PIP3", "PI3K", "PTEN_T1", "PTEN_T2"]
_D = {"PIP2": 0.15, "PIP3": 0.15, "PI3K": 0.10, "PTEN_T1": 0.08, "PTEN_T2": 0.08}
_R = {"PIP2": 0.5, "PIP3": 0.5, "PI3K": 4.0, "PTEN_T1": 4.0, "PTEN_T2": 4.0}

_FEEDBACK = [
    ("pip3_inhibition", "PIP3", "hill_inhibition", 40.0, 4.0, 0.0),
    ("pip3_activation", "PIP3", "hill_activation", 15.0, 2.0, 0.05),
    ("pip3_activation_pten", "PIP3", "hill_activation", 15.0, 2.0, 0.05),
    ("pip3_detachment_boost", "PIP3", "hill_activation", 40.0, 2.0, 0.2),
    ("pten_self_activation", "PTEN_T2", "hill_activation", 30.0, 2.0, 0.1),
]


def membrane_pip3_pten(counts: Optional[Dict[str, int]] = None, pools: Optional[Dict[str, int]] = None,
                       box: float = 10.0, potential: str = "wca", n_frames: int = 20,
                       steps_per_frame: int = 100, pixels: int = 64, pixel_size_nm: float = 156.0,
                       sine_d_field: bool = False, seed: int = 42, k_cat_scale: float = 1.0,
                       K_half_scale: float = 1.0, dt: float = 1e-4) -> dict:
    """The PIP3/PTEN membrane system as a YAML-equivalent dict."""
    counts = dict(C0_COUNTS if counts is None else counts)
    pools = dict(C0_POOLS if pools is None else pools)
    d: dict = {"name": "PIP3/PTEN membrane", "membrane": {"size": [box, box], "periodic": [True, True]}}
    if sine_d_field:
        d["diffusion_field"] = {"type": "sine_x", "amplitude": 0.5, "wavelength": 5.0}
    else:
        d["diffusion_field"] = {"type": "uniform"}
    d["species"] = [{"name": n, "diffusion_coefficient": _D[n], "radius": _R[n]} for n in _SPECIES]
    kc = k_cat_scale
    d["catalytic_reactions"] = [
        {"name": "PI3K_cat", "enzyme": "PI3K", "substrate": "PIP2", "product": "PIP3",
         "k_cat": 0.0083 * kc, "contact_radius": 150.0, "feedback_rule": "pip3_activation"},
        {"name": "T1_cat", "enzyme": "PTEN_T1", "substrate": "PIP3", "product": "PIP2",
         "k_cat": 0.05 * kc, "contact_radius": 150.0},
        {"name": "T2_cat", "enzyme": "PTEN_T2", "substrate": "PIP3", "product": "PIP2",
         "k_cat": 0.005 * kc, "contact_radius": 150.0},
    ]
    d["compartment_exchanges"] = [
        {"name": "PI3K_ex", "species": "PI3K", "k_on": 0.4, "k_off": 0.4,
         "cytosol_pool": pools.get("PI3K", 0), "max_recruits_per_step": 20, "feedback_rule": "pip3_activation"},
        {"name": "T1_ex", "species": "PTEN_T1", "k_on": 0.6, "k_off": 4.7,
         "cytosol_pool": pools.get("PTEN_T1", 0), "max_recruits_per_step": 20,
         "feedback_rule": "pip3_inhibition", "secondary_feedback_rule": "pten_self_activation"},
        {"name": "T2_ex", "species": "PTEN_T2", "k_on": 0.0, "k_off": 1.1, "cytosol_pool": 0,
         "max_recruits_per_step": 20, "detachment_feedback_rule": "pip3_detachment_boost"},
    ]
    d["unimolecular_conversions"] = [
        {"name": "T1_to_T2", "from_species": "PTEN_T1", "to_species": "PTEN_T2", "rate": 0.35,
         "feedback_rule": "pip3_activation_pten"},
        {"name": "T2_to_T1", "from_species": "PTEN_T2", "to_species": "PTEN_T1", "rate": 0.015},
    ]
    d["feedback_rules"] = [
        {"name": n, "sensor_species": s, "function_type": f, "K_half": K * K_half_scale, "n_hill": nh,
         "grid_resolution": 0.5, "basal_fraction": b} for (n, s, f, K, nh, b) in _FEEDBACK]
    pots = []
    for i, a in enumerate(_SPECIES):
        for b in _SPECIES[i:]:
            if potential == "wca":
                pots.append({"species_a": a, "species_b": b, "potential_type": "wca",
                             "parameters": {"sigma": 5.0, "epsilon": 1.0}})
            else:
                pots.append({"species_a": a, "species_b": b, "potential_type": "harmonic_repulsion",
                             "parameters": {"sigma": 5.0, "spring_constant": 1.0e7,
                                            "interaction_distance": 5.0}})
    d["potentials"] = pots
    d["initial_populations"] = counts
    d["fluorophores"] = copy.deepcopy(_FLUOROPHORES)
    d["fret_pairs"] = [{"donor_type": "mTFP1", "acceptor_type": "Venus", "R0": 5.4,
                        "intra_complex_distance": 5.0, "fret_mode": "bond", "intramolecular": True}]
    d["dye_attachments"] = [{"species": "PIP3", "fluorophore": "mTFP1", "labeling_efficiency": 1.0}]
    d["objective"] = {"NA": 0.7071}
    d["laser"] = {"wavelength": 462.0, "repetition_rate": 4.0e7, "pulse_width": 1.0e-10,
                  "power": 5.0e-6, "beam_waist": 250.0}
    d["detector"] = {"dark_count_rate": 100.0, "detection_efficiency": 0.4, "timing_jitter": 5.0e-11,
                     "dead_time": 1.0e-7, "afterpulsing_prob": 0.0}
    d["scan"] = {"pixel_size": pixel_size_nm, "pixels_x": pixels, "pixels_y": pixels, "dwell_time": 2.0e-5,
                 "n_frames": n_frames, "frame_interval": steps_per_frame * dt}
    d["tcspc"] = {"n_bins": 256, "time_range": 2.5e-8}
    d["psf"] = {"type": "gaussian", "emission_wavelength": 492.0}
    d["simulation_time"] = n_frames * steps_per_frame * dt
    d["bd_timestep"] = dt
    d["random_seed"] = seed
    return d


def scaled_counts(n_membrane: int) -> Dict[str, int]:
    """Membrane counts in the config-0 species ratios summing to n_membrane."""
    tot = sum(C0_COUNTS.values())
    out = {k: int(round(v * n_membrane / tot)) for k, v in C0_COUNTS.items()}
    out["PIP2"] += n_membrane - sum(out.values())
    return out


def scaled_pools(n_membrane: int) -> Dict[str, int]:
    tot = sum(C0_COUNTS.values())
    return {k: int(round(v * n_membrane / tot)) for k, v in C0_POOLS.items()}


def config0() -> dict:
    """10x10 µm^2, 3,500 membrane + 1,500 dormant, WCA, 2,000 steps, 64x64 px."""
    return membrane_pip3_pten()


def config1(n_frames: int = 200) -> dict:
    """13,000 membrane particles, sine D(x), 20,000 steps, 128x128 frame per 100 steps."""
    n = 13000
    return membrane_pip3_pten(counts=scaled_counts(n), pools=scaled_pools(n), sine_d_field=True,
                              n_frames=n_frames, pixels=128, pixel_size_nm=10000.0 / 128)


def config2(n_frames: int = 20) -> dict:
    """100x100 µm^2, 1.3M membrane particles, harmonic repulsion, 200x200 density grid."""
    n = 1_300_000
    return membrane_pip3_pten(counts=scaled_counts(n), pools=scaled_pools(n), box=100.0,
                              potential="harmonic", n_frames=n_frames, pixels=256,
                              pixel_size_nm=100000.0 / 256)


def ensemble_replicas(n_replicas: int = 512, seed: int = 2024, n_min: int = 1000,
                      n_max: int = 50000, pixels: int = 64) -> List[dict]:
    """Replicas with N ~ log-uniform(n_min, n_max), box L = 10 sqrt(N/3500) µm,
    k_cat and K_half each scaled by U(0.5, 1.5); seed per replica."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n_replicas):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        box = 10.0 * math.sqrt(n / 3500.0)
        kc = float(rng.uniform(0.5, 1.5))
        kh = float(rng.uniform(0.5, 1.5))
        rseed = int(rng.integers(1, 2 ** 31 - 1))
        out.append(membrane_pip3_pten(counts=scaled_counts(n), pools=scaled_pools(n), box=box,
                                      k_cat_scale=kc, K_half_scale=kh, seed=rseed, pixels=pixels,
                                      pixel_size_nm=min(156.0, box * 1000.0 / pixels)))
    return out
