"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run where the reference source tree is present, with EDM_REFERENCE_ROOT set to
it (the directory holding ed_mrdt/):

    python tests/golden/make_golden.py [name ...]   (default: every system)

For every test system of tests/cases.py the reference's own DynamicsEngine,
PhotonSimulator and VirtualMicroscope run K BD steps with the keyed draws
injected (oracle/refshim.py), then one finalize_frame.  Saved per system:
the reference's derived constants, the state after step 10 and after step
K, the counters, the last photon batch and the finalized FLIM stack.  The
CPU tests replay the same steps on the oracle and require bit equality.

Also saved: the per-step series SimulationPipeline.run(record_subframe=True)
records (pipeline.py:567-642), evaluated here on the reference's state and
counters after each step with the same expressions ("sf_*"), and the frame's
ground truth from the reference's own SimulationPipeline._extract_ground_truth
after PhotonSimulator.update_fret_rates (pipeline.py:653-654, "gt_*").
"""
from __future__ import annotations

import sys
import types
import warnings
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refshim as RS  # noqa: E402
from tests import cases  # noqa: E402

STEPS = 24
SNAP = 10


def generate(name: str) -> dict:
    RS.import_reference()
    from ed_mrdt.dynamics import DynamicsEngine
    from ed_mrdt.microscope import VirtualMicroscope
    from ed_mrdt.particles import ParticleState
    from ed_mrdt.photophysics import PhotonSimulator

    raw = cases.get(name)
    cfg = RS.ref_config_from_dict(raw)
    st = ParticleState(cfg)
    eng = DynamicsEngine(cfg, st)
    duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
    ps = PhotonSimulator(cfg, st, scan_duty_fraction=duty)
    vm = VirtualMicroscope(cfg, st)
    seed = cfg.random_seed
    sine = (0.5, 5.0) if raw.get("diffusion_field", {}).get("type") == "sine_x" else None
    dyn = RS.ShimmedDynamics(eng, seed, sine_field=sine)
    ph = RS.ShimmedPhotons(ps, seed)
    sc = RS.ShimmedMicroscope(vm, seed)
    out = {
        "init_positions": st.positions.copy(), "init_species": st.species_id.copy(),
        "init_alive": st.is_alive.copy(), "init_has_dye": st.has_dye.copy(), "init_dye": st.dye_type_id.copy(),
        "cutoff_um": eng.cutoff_um, "max_displacement": eng.max_displacement,
        "nx": eng.cell_list.nx, "ny": eng.cell_list.ny,
        "prob_cat": np.array([c["prob_cat"] for c in eng._catalytic_reactions]),
        "prob_on": np.array([e["prob_on"] for e in eng._compartment_exchanges]),
        "prob_off": np.array([e["prob_off"] for e in eng._compartment_exchanges]),
        "prob_conv": np.array([c["prob"] for c in eng._unimolecular_conversions]),
        "prob_bind": np.array([r["prob_bind"] for r in eng._reactions]),
        "T_step": ps._T_step_all, "T_step_fret": ps._T_step_fret_all,
        "mean_ph": ps._mean_ph_all, "mean_ph_fret": ps._mean_ph_fret_all,
        "mean_fret": ps._mean_fret_all, "tau_all": ps._tau_all, "k_fret_bound": ps._k_fret_bound_all,
        "max_photons": ps._max_photons,
        "psf_sigma": np.array([vm.psf.sigma_um[k] for k in sorted(vm.psf.sigma_um)]),
        "psf_range_px": vm.scanner.psf_range_px, "sigma_irf": vm.tcspc.sigma_irf,
    }
    sf = {k: np.zeros(STEPS, dtype=np.int64) for k in
          ("n_complexes", "n_bindings", "n_dissociations", "n_bleached", "total_photons", "n_catalytic",
           "n_recruited", "n_detached", "n_converted")}
    sf["mean_fret_E"] = np.zeros(STEPS)
    sf["species"] = np.zeros((STEPS, len(cfg.species)), dtype=np.int64)
    names = ("n_bindings", "n_dissociations", "n_catalytic", "n_recruited", "n_detached", "n_converted")
    prev = [getattr(eng, k) for k in names]
    for t in range(STEPS):
        dyn.step()
        batch = ph.evolve(t)
        sc.process(batch, t)
        # the sub-frame record of pipeline.py:567-642
        n_bound = int(np.sum(st.bond_partner[st.is_alive] >= 0) // 2)
        sf["n_complexes"][t] = n_bound
        cur = [getattr(eng, k) for k in names]
        for k, a, b in zip(names, cur, prev):
            sf[k][t] = a - b
        prev = cur
        sf["n_bleached"][t] = np.sum(st.is_bleached)
        sf["total_photons"][t] = batch.n_photons
        if cfg.fret_pairs:
            fp = cfg.fret_pairs[0]
            donors = st.has_dye & st.is_alive & ~st.is_bleached & (st.dye_type_id == 0)
            n_don = int(np.sum(donors))
            if getattr(fp, "fret_mode", "bond") == "proximity" and n_don > 0:
                k = ps._k_fret[donors]
                tau_d = ps._tau_all[0]
                sf["mean_fret_E"][t] = float(np.mean(k * tau_d / (1.0 + k * tau_d)))
            elif getattr(fp, "fret_mode", "bond") != "proximity" and n_don > 0:
                e_const = 1.0 / (1.0 + (fp.intra_complex_distance / fp.R0) ** 6)
                sf["mean_fret_E"][t] = e_const * n_bound / (n_bound + (n_don - n_bound))
        for i in range(len(cfg.species)):
            sf["species"][t, i] = np.sum((st.species_id == i) & st.is_alive)
        if t + 1 == SNAP:
            out["snap_positions"] = st.positions.copy()
            out["snap_species"] = st.species_id.copy()
            out["snap_alive"] = st.is_alive.copy()
    dyn.restore()
    frame = sc.finalize()
    from ed_mrdt.pipeline import SimulationPipeline
    ps.update_fret_rates()
    gt = SimulationPipeline._extract_ground_truth(types.SimpleNamespace(_state=st, config=cfg, _photon_sim=ps))
    out.update({f"sf_{k}": v for k, v in sf.items()})
    out.update({"gt_fret_E": gt.fret_efficiency_exact, "gt_tau_DA": gt.donor_lifetime_exact,
                "gt_n_complexes": gt.n_complexes, "gt_n_bleached": gt.n_bleached,
                "gt_n_free_donors": gt.n_free_donors,
                "gt_species_counts": np.array([gt.species_counts[sp.name] for sp in cfg.species], dtype=np.int64)})
    out.update({
        "final_positions": st.positions.copy(), "final_species": st.species_id.copy(),
        "final_alive": st.is_alive.copy(), "final_bond": st.bond_partner.copy(),
        "final_ctmc": st.ctmc_state.copy(), "final_bleached": st.is_bleached.copy(),
        "counters": np.array([eng.n_bindings, eng.n_dissociations, eng.n_catalytic, eng.n_recruited,
                              eng.n_detached, eng.n_converted], dtype=np.int64),
        "last_batch_particle": batch.particle_idx, "last_batch_time": batch.arrival_time,
        "last_batch_channel": batch.channel,
        "flim": frame.flim_stack, "n_dark": frame.n_dark_counts, "n_ap": frame.n_afterpulses,
        "photons_detected": vm.total_photons_detected,
    })
    return out


def main():
    warnings.filterwarnings("ignore")
    here = Path(__file__).resolve().parent
    for name in sys.argv[1:] or list(cases.CASES):
        data = generate(name)
        np.savez_compressed(here / f"{name}.npz", **data)
        print(name, "counters", data["counters"].tolist(), "flim counts", int(data["flim"].sum()))


if __name__ == "__main__":
    main()
