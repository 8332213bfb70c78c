"""A small seeded simulation result for HDF5 layout tests (test
infrastructure): the rich_small system's configuration with two frames, and
synthetic frame contents (TCSPC stacks, ground truth, statistics) built from
one seed, so that the reference's writer and this package's writer can be
fed the same values."""
from __future__ import annotations

import numpy as np

from tests import cases

N_FRAMES = 2


def raw_config() -> dict:
    raw = cases.get("rich_small")
    raw["scan"]["n_frames"] = N_FRAMES
    raw["name"] = "layout check"
    return raw


def frame_arrays(n_particles: int, n_species: int, px: int, py: int, n_bins: int, seed: int = 5) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for f in range(N_FRAMES):
        stack = rng.poisson(0.05, (2, px, py, n_bins)).astype(np.uint32)
        bond = np.full(n_particles, -1, dtype=np.int32)
        pairs = rng.permutation(n_particles)[:20].reshape(10, 2)
        bond[pairs[:, 0]], bond[pairs[:, 1]] = pairs[:, 1], pairs[:, 0]
        out.append({
            "frame_index": f, "bio_time": (f + 1) * 0.01, "flim_stack": stack,
            "intensity": stack.sum(axis=-1).astype(np.float64), "n_signal": int(rng.integers(0, 1000)),
            "n_dark": int(rng.integers(0, 100)), "n_ap": int(rng.integers(0, 10)),
            "positions": rng.uniform(0, 3, (n_particles, 2)), "species_id": rng.integers(0, n_species, n_particles).astype(np.int32),
            "bond_partner": bond, "is_alive": rng.random(n_particles) < 0.8, "has_dye": rng.random(n_particles) < 0.2,
            "dye_type_id": rng.integers(-1, 2, n_particles).astype(np.int32), "is_bleached": rng.random(n_particles) < 0.05,
            "fret_E": rng.random(n_particles) * 0.5, "tau_DA": rng.random(n_particles) * 3e-9,
            "n_complexes": 10, "n_bleached": int(rng.integers(0, 50)), "n_free_donors": int(rng.integers(0, 50)),
            "emitted": int(rng.integers(0, 10 ** 6)), "detected": int(rng.integers(0, 10 ** 5)),
            "wall": float(rng.random()),
        })
    return out


TOTALS = {"total_wall_time": 12.5, "peak_ram_mb": 345.0, "total_bindings": 17, "total_dissociations": 4}


def build_frames(arrays: list, FLIMFrame, GroundTruth, FrameResult) -> list:
    """Frame objects of either implementation (same field names)."""
    frames = []
    for a in arrays:
        fl = FLIMFrame(flim_stack=a["flim_stack"], intensity=a["intensity"], frame_index=a["frame_index"],
                       n_signal_photons=a["n_signal"], n_dark_counts=a["n_dark"], n_afterpulses=a["n_ap"])
        gt = GroundTruth(positions=a["positions"], species_id=a["species_id"], bond_partner=a["bond_partner"],
                         is_alive=a["is_alive"], has_dye=a["has_dye"], dye_type_id=a["dye_type_id"],
                         is_bleached=a["is_bleached"], fret_efficiency_exact=a["fret_E"],
                         donor_lifetime_exact=a["tau_DA"], n_complexes=a["n_complexes"], n_bleached=a["n_bleached"],
                         n_free_donors=a["n_free_donors"], species_counts={})
        frames.append(FrameResult(frame_index=a["frame_index"], bio_time=a["bio_time"], flim_frame=fl,
                                  ground_truth=gt, n_photons_emitted=a["emitted"], n_photons_detected=a["detected"],
                                  wall_time_s=a["wall"]))
    return frames
