"""Builds the GPU engine and the CPU oracle for the same system."""
from __future__ import annotations

import numpy as np

from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
from oracle import oracle as O


class Pair:
    """One system on the GPU engine and on the oracle, same initial state."""

    def __init__(self, raw: dict, precision: int = 64, photons: bool = True):
        from flim_microscopy_simulator_with_causal_inference_b200.engine import Engine
        self.cfg = config_from_dict(raw)
        self.state = ParticleState(self.cfg)
        st = self.state
        self.dp, self.hill, self.dd = PR.build_dyn_params(self.cfg, st.N)
        self.duty = min(1.0, self.cfg.scan.dwell_time / self.cfg.scan.frame_interval)
        self.pp = self.pd = self.sp = None
        phot = scope = None
        if photons:
            self.pp, self.pd = PR.build_phot_params(self.cfg, st.N, int(st.has_dye.sum()), self.duty)
            self.sp, _ = PR.build_scope_params(self.cfg)
            phot, scope = [self.pp], [self.sp]
        self.eng = Engine([self.dp], self.hill, phot, scope, precision=precision)
        self.eng.set_state(st.positions, st.species_id, st.is_alive, st.bond_partner, st.has_dye, st.dye_type_id,
                           st.ctmc_state, st.is_bleached)
        self.orc = O.OracleSimulation(self.cfg, st, self.dp, self.pd if photons else None,
                                      self.sp if photons else None, self.duty)

    def gpu_state(self) -> dict:
        return self.eng.get_state()

    def load_oracle_state_into_gpu(self):
        o = self.orc
        self.eng.set_state(o.pos, o.species, o.alive, o.bond, o.has_dye, o.dye_type, o.ctmc, o.bleached)
        self.eng.set_step(o.step_index)


def compare_state(g: dict, o: O.OracleSimulation, pos_tol: float) -> float:
    """Assert species / alive / bonds / photophysical state equal; return the
    max position error (asserted <= pos_tol)."""
    assert np.array_equal(g["species"], o.species), "species differ"
    assert np.array_equal(g["alive"].astype(bool), o.alive.astype(bool)), "alive differs"
    assert np.array_equal(g["bond"], o.bond), "bond partners differ"
    assert np.array_equal(g["ctmc"], o.ctmc), "ctmc states differ"
    assert np.array_equal(g["bleached"].astype(bool), o.bleached.astype(bool)), "bleaching differs"
    err = float(np.max(np.abs(g["positions"] - o.pos))) if o.N else 0.0
    assert err <= pos_tol, f"position error {err} > {pos_tol}"
    return err


def cell_sets_oracle(o: O.OracleSimulation, nx: int, ny: int):
    """Cell -> member set from the oracle's head/next chains of the last step."""
    import ctypes as C
    head = np.ctypeslib.as_array(C.cast(o.dyn.head, C.POINTER(C.c_int32)), shape=(nx * ny,))
    nxt = np.ctypeslib.as_array(C.cast(o.dyn.next, C.POINTER(C.c_int32)), shape=(o.N,))
    out = []
    for c in range(nx * ny):
        mem = []
        j = head[c]
        while j >= 0:
            mem.append(int(j))
            j = nxt[j]
        out.append(sorted(mem))
    return out
