"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a container that has the reference source tree (EDM_REFERENCE_ROOT,
default /root/reference):

    python tests/golden/make_golden.py [name ...]   (default: every system)

For every test system of tests/cases.py the reference's own DynamicsEngine,
PhotonSimulator and VirtualMicroscope run K BD steps with the keyed draws
injected (oracle/refshim.py), then one finalize_frame.  Saved per system:
the reference's derived constants, the state after step 10 and after step
K, the counters, the last photon batch and the finalized FLIM stack.  The
CPU tests replay the same steps on the oracle and require bit equality.
"""
from __future__ import annotations

import sys
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
    for t in range(STEPS):
        dyn.step()
        batch = ph.evolve(t)
        sc.process(batch, t)
        if t + 1 == SNAP:
            out["snap_positions"] = st.positions.copy()
            out["snap_species"] = st.species_id.copy()
            out["snap_alive"] = st.is_alive.copy()
    dyn.restore()
    frame = sc.finalize()
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
