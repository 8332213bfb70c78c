"""The reference's sub-frame series and ground truth evaluated on an oracle
state (test infrastructure): the expressions of pipeline.py:567-642 (one BD
step of SimulationPipeline.run with record_subframe=True) and of
_extract_ground_truth, pipeline.py:357-455, after update_fret_rates."""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import oracle as O

COUNTER_NAMES = ("n_bindings", "n_dissociations", "n_catalytic", "n_recruited", "n_detached", "n_converted")


def subframe_step(orc, cfg, n_photons: int, prev_counters: np.ndarray, tau_all0: float) -> dict:
    """One step's record; prev_counters = the oracle's first six counters
    before the step."""
    alive = orc.alive.astype(bool)
    bleached = orc.bleached.astype(bool)
    n_bound = int(np.sum(orc.bond[alive] >= 0) // 2)
    out = {"n_complexes": n_bound, "n_bleached": int(np.sum(bleached)), "total_photons": int(n_photons)}
    cur = orc.counters[:6]
    for k, name in enumerate(COUNTER_NAMES):
        out[name] = int(cur[k] - prev_counters[k])
    mean = 0.0
    if cfg.fret_pairs:
        fp = cfg.fret_pairs[0]
        donors = orc.has_dye.astype(bool) & alive & ~bleached & (orc.dye_type == 0)
        n_don = int(np.sum(donors))
        if getattr(fp, "fret_mode", "bond") == "proximity" and n_don > 0:
            k = orc.k_fret[donors]
            mean = float(np.mean(k * tau_all0 / (1.0 + k * tau_all0)))
        elif getattr(fp, "fret_mode", "bond") != "proximity" and n_don > 0:
            e_const = 1.0 / (1.0 + (fp.intra_complex_distance / fp.R0) ** 6)
            mean = e_const * n_bound / (n_bound + (n_don - n_bound))
    out["mean_fret_E"] = mean
    out["species"] = np.array([np.sum((orc.species == i) & alive) for i in range(len(cfg.species))], dtype=np.int64)
    return out


def ground_truth(orc, cfg, pd) -> dict:
    """update_fret_rates on the oracle's state, then the frame's ground truth."""
    O.lib().orc_update_fret_rates(C.byref(orc.pp), C.byref(orc.phot))
    N = orc.N
    has_dye = orc.has_dye.astype(bool)
    bleached = orc.bleached.astype(bool)
    fret_E = np.zeros(N)
    tau_DA = np.zeros(N)
    for fp in cfg.fret_pairs:
        di = next((i for i, f in enumerate(cfg.fluorophores) if f.name == fp.donor_type), None)
        if di is None:
            continue
        tau_D = pd.tau_all[di]
        if tau_D <= 0 or np.isinf(tau_D):
            continue
        for i in range(N):
            if not has_dye[i] or bleached[i] or orc.dye_type[i] != di:
                continue
            k = orc.k_fret[i]
            if k > 0:
                fret_E[i] = k * tau_D / (1.0 + k * tau_D)
                tau_DA[i] = tau_D / (1.0 + k * tau_D)
            else:
                fret_E[i] = 0.0
                tau_DA[i] = tau_D
    n_free = 0
    for fp in cfg.fret_pairs:
        for fi, f in enumerate(cfg.fluorophores):
            if f.name == fp.donor_type:
                n_free += int(np.sum(has_dye & (orc.dye_type == fi) & ~bleached & (orc.bond < 0)))
    alive = orc.alive.astype(bool)
    return {"fret_E": fret_E, "tau_DA": tau_DA, "n_complexes": int(np.sum(orc.bond >= 0)) // 2,
            "n_bleached": int(np.sum(bleached)), "n_free_donors": n_free,
            "species": np.array([np.sum((orc.species == i) & alive) for i in range(len(cfg.species))],
                                dtype=np.int64)}
