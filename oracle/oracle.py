"""ctypes driver of the CPU float64 oracle (oracle/edm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference arm, never by the product package.

`OracleSimulation` advances one replica through the reference's per-BD-step
loop body (ed_mrdt/pipeline.py:554-564): DynamicsEngine.step(),
PhotonSimulator.evolve_one_bd_step(), VirtualMicroscope.process_photons(),
and VirtualMicroscope.finalize_frame() at frame ends, with every random draw
taken from the keyed generator.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc, no external dependencies)."""
    srcs = [HERE / "edm_oracle.c", HERE / "edm_oracle.h", HERE.parent / "include" / "edm_b200.h"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE)], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        vp, i64, i32, u64, dp = C.c_void_p, C.c_int64, C.c_int32, C.c_uint64, C.POINTER(C.c_double)
        L.orc_uniform2.argtypes = [u64, i64, i32, u64, u64, dp, dp]
        L.orc_normal2.argtypes = [u64, i64, i32, u64, dp, dp]
        L.orc_ln.argtypes = [C.c_double]
        L.orc_ln.restype = C.c_double
        L.orc_fill_uniform.argtypes = [u64, i64, i32, vp, vp, i64, vp, i32]
        L.orc_fill_normal.argtypes = [u64, i64, i32, vp, i64, vp, i32]
        L.orc_poisson_knuth.argtypes = [u64, i64, i32, u64, C.c_double]
        L.orc_poisson_knuth.restype = i64
        L.orc_dyn_alloc.argtypes = [vp, vp, i64]
        L.orc_dyn_free.argtypes = [vp]
        L.orc_dyn_step.argtypes = [vp, vp, i64]
        L.orc_update_fret_rates.argtypes = [vp, vp]
        L.orc_photon_step.argtypes = [vp, vp, i64]
        L.orc_process_photons.argtypes = [vp, u64, i64, vp, i64, vp, vp, vp, i64, vp, vp]
        L.orc_finalize_frame.argtypes = [vp, u64, i64, vp, vp, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ---- keyed noise, vectorised (used by the reference shim and the tests) ----
def uniforms(seed: int, step: int, stream: int, a, b=None, two: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int64)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.int64)
    out = np.empty((a.size, 2) if two else a.size, dtype=np.float64)
    lib().orc_fill_uniform(seed, step, stream, _p(a), None if bb is None else _p(bb), a.size, _p(out), int(two))
    return out


def normals(seed: int, step: int, stream: int, a, two: bool = True) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int64)
    out = np.empty((a.size, 2) if two else a.size, dtype=np.float64)
    lib().orc_fill_normal(seed, step, stream, _p(a), a.size, _p(out), int(two))
    return out


def poisson_knuth(seed: int, step: int, stream: int, key: int, exp_neg_lambda: float) -> int:
    return int(lib().orc_poisson_knuth(seed, step, stream, key, exp_neg_lambda))


# ---- oracle structs --------------------------------------------------------
NCOUNTERS = 14
MAXF = 4


class OrcDyn(C.Structure):
    _fields_ = [("N", C.c_int64), ("pos", C.c_void_p), ("species", C.c_void_p),
                ("alive", C.c_void_p), ("bond", C.c_void_p),
                ("counters", C.c_int64 * NCOUNTERS), ("head", C.c_void_p), ("next", C.c_void_p),
                ("pairs", C.c_void_p), ("n_pairs", C.c_int64), ("max_pairs", C.c_int64),
                ("forces", C.c_void_p), ("adapt_w", C.c_void_p)]


class OrcPhotParams(C.Structure):
    _fields_ = [
        ("n_fluoro", C.c_int32),
        ("T_step", ((C.c_double * 3) * 3) * MAXF), ("T_step_fret", ((C.c_double * 3) * 3) * MAXF),
        ("mean_ph", (C.c_double * 2) * MAXF), ("mean_ph_fret", (C.c_double * 2) * MAXF),
        ("mean_fret", (C.c_double * 2) * MAXF), ("mean_fret_fret", (C.c_double * 2) * MAXF),
        ("tau_all", C.c_double * MAXF), ("k_fret_bound", C.c_double * MAXF),
        ("ground", C.c_int32 * MAXF), ("excited", C.c_int32 * MAXF), ("t1", C.c_int32 * MAXF),
        ("bl", C.c_int32 * MAXF),
        ("n_bond", C.c_int32),
        ("bond_R0", C.c_double * MAXF), ("bond_tauD", C.c_double * MAXF), ("bond_icd", C.c_double * MAXF),
        ("bond_donor", C.c_int32 * MAXF), ("bond_acceptor", C.c_int32 * MAXF), ("bond_intra", C.c_int32 * MAXF),
        ("n_prox", C.c_int32),
        ("prox_radius_um", C.c_double * MAXF), ("prox_khigh", C.c_double * MAXF),
        ("prox_klow", C.c_double * MAXF),
        ("prox_donor", C.c_int32 * MAXF), ("prox_target", C.c_int32 * MAXF),
        ("max_photons", C.c_int64), ("est_photons", C.c_int64),
        ("Lx", C.c_double), ("Ly", C.c_double), ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("seed", C.c_uint64),
    ]


class OrcPhot(C.Structure):
    _fields_ = [("N", C.c_int64), ("pos", C.c_void_p), ("species", C.c_void_p), ("alive", C.c_void_p),
                ("bond", C.c_void_p), ("has_dye", C.c_void_p), ("dye_type", C.c_void_p),
                ("ctmc", C.c_void_p), ("bleached", C.c_void_p), ("k_fret", C.c_void_p),
                ("acc_idx", C.c_void_p), ("ph_particle", C.c_void_p), ("ph_time", C.c_void_p),
                ("ph_channel", C.c_void_p), ("ph_is_fret", C.c_void_p), ("n_photons", C.c_int64)]


class OrcScopeStats(C.Structure):
    _fields_ = [("n_received", C.c_int64), ("n_detected", C.c_int64)]


def orc_phot_params(pd, config, seed: int) -> OrcPhotParams:
    """Reference-style photophysics arrays (PhotonSimulator fields) from a
    PhotDerived, for the oracle's restatement of _evolve_pss_kernel."""
    P = OrcPhotParams()
    P.n_fluoro = pd.n_fluoro
    for t in range(pd.n_fluoro):
        for a in range(3):
            for b in range(3):
                P.T_step[t][a][b] = pd.T_step[t, a, b]
                P.T_step_fret[t][a][b] = pd.T_step_fret[t, a, b]
        for s in range(2):
            P.mean_ph[t][s] = pd.mean_ph[t, s]
            P.mean_ph_fret[t][s] = pd.mean_ph_fret[t, s]
            P.mean_fret[t][s] = pd.mean_fret[t, s]
            P.mean_fret_fret[t][s] = pd.mean_fret_fret[t, s]
        P.tau_all[t] = pd.tau_all[t]
        P.k_fret_bound[t] = pd.k_fret_bound[t]
        rm = pd.rates[t]
        P.ground[t], P.excited[t], P.t1[t], P.bl[t] = rm.ground, rm.excited, rm.t1, rm.bl
    P.n_bond = len(pd.bond_pairs)
    for k, bp in enumerate(pd.bond_pairs):
        P.bond_R0[k], P.bond_tauD[k], P.bond_icd[k] = bp["R0"], bp["tauD"], bp["icd"]
        P.bond_donor[k], P.bond_acceptor[k], P.bond_intra[k] = bp["donor"], bp["acceptor"], int(bp["intra"])
    P.n_prox = len(pd.prox_pairs)
    for k, pp in enumerate(pd.prox_pairs):
        P.prox_radius_um[k], P.prox_khigh[k], P.prox_klow[k] = pp["radius_um"], pp["k_high"], pp["k_low"]
        P.prox_donor[k], P.prox_target[k] = pp["donor"], pp["target"]
    P.max_photons, P.est_photons = pd.max_photons, pd.est_photons
    P.Lx, P.Ly = config.membrane.size
    P.periodic_x, P.periodic_y = int(config.membrane.periodic[0]), int(config.membrane.periodic[1])
    P.seed = seed
    return P


class OracleSimulation:
    """One replica of the reference's per-BD-step loop on the CPU oracle.

    state: a ParticleState-like object (positions, species_id, is_alive,
    bond_partner, has_dye, dye_type_id, ctmc_state, is_bleached); its arrays
    are copied in and the oracle keeps its own.
    """

    def __init__(self, config, state, dyn_params, phot_derived=None, scope_params=None,
                 scan_duty_fraction: float = 1.0, seed=None):
        L = lib()
        self.config = config
        self.seed = int(config.random_seed if seed is None else seed)
        self.dp = dyn_params
        self.N = int(state.positions.shape[0])
        self.dyn = OrcDyn()
        if L.orc_dyn_alloc(C.byref(self.dyn), C.byref(self.dp), self.N) != 0:
            raise MemoryError("oracle allocation failed")
        N = self.N
        # the oracle works on numpy views of its own buffers
        self.pos = np.ctypeslib.as_array(C.cast(self.dyn.pos, C.POINTER(C.c_double)), shape=(N, 2))
        self.species = np.ctypeslib.as_array(C.cast(self.dyn.species, C.POINTER(C.c_int32)), shape=(N,))
        self.alive = np.ctypeslib.as_array(C.cast(self.dyn.alive, C.POINTER(C.c_uint8)), shape=(N,))
        self.bond = np.ctypeslib.as_array(C.cast(self.dyn.bond, C.POINTER(C.c_int32)), shape=(N,))
        self.pos[:] = state.positions
        self.species[:] = state.species_id
        self.alive[:] = state.is_alive
        self.bond[:] = state.bond_partner
        self.has_dye = np.ascontiguousarray(state.has_dye, dtype=np.uint8).copy()
        self.dye_type = np.ascontiguousarray(state.dye_type_id, dtype=np.int32).copy()
        self.ctmc = np.ascontiguousarray(state.ctmc_state, dtype=np.int8).copy()
        self.bleached = np.ascontiguousarray(state.is_bleached, dtype=np.uint8).copy()
        self.step_index = 0
        self.frame_index = 0
        self.phot = None
        if phot_derived is not None and phot_derived.active:
            self.pp = orc_phot_params(phot_derived, config, self.seed)
            cap = int(self.pp.max_photons)
            self.k_fret = np.zeros(N)
            self.acc_idx = np.full(N, -1, dtype=np.int32)
            self.ph_particle = np.zeros(cap, dtype=np.int32)
            self.ph_time = np.zeros(cap)
            self.ph_channel = np.zeros(cap, dtype=np.int8)
            self.ph_is_fret = np.zeros(cap, dtype=np.uint8)
            self.phot = OrcPhot(N, _p(self.pos), _p(self.species), _p(self.alive), _p(self.bond),
                                _p(self.has_dye), _p(self.dye_type), _p(self.ctmc), _p(self.bleached),
                                _p(self.k_fret), _p(self.acc_idx), _p(self.ph_particle), _p(self.ph_time),
                                _p(self.ph_channel), _p(self.ph_is_fret), 0)
            self.total_photons = 0
        self.sp = scope_params
        if scope_params is not None:
            shape = (scope_params.n_channels, scope_params.nx, scope_params.ny, scope_params.n_bins)
            self.flim = np.zeros(shape, dtype=np.uint32)
            self.scope_stats = OrcScopeStats(0, 0)

    def __del__(self):
        try:
            lib().orc_dyn_free(C.byref(self.dyn))
        except Exception:
            pass

    @property
    def counters(self) -> np.ndarray:
        return np.array(self.dyn.counters[:], dtype=np.int64)

    def pairs(self) -> np.ndarray:
        n = int(self.dyn.n_pairs)
        arr = np.ctypeslib.as_array(C.cast(self.dyn.pairs, C.POINTER(C.c_int32)), shape=(max(n, 1), 2))
        return arr[:n].copy()

    def dynamics_step(self) -> None:
        lib().orc_dyn_step(C.byref(self.dp), C.byref(self.dyn), self.step_index)

    def photon_step(self):
        """PhotonSimulator.evolve_one_bd_step() for the current state."""
        lib().orc_photon_step(C.byref(self.pp), C.byref(self.phot), self.step_index)
        n = int(self.phot.n_photons)
        self.total_photons += n
        return (self.ph_particle[:n].copy(), self.ph_time[:n].copy(),
                self.ph_channel[:n].copy(), self.ph_is_fret[:n].astype(bool))

    def process_photons(self, batch) -> None:
        pid, t, ch, _ = batch
        n = pid.size
        pid = np.ascontiguousarray(pid, dtype=np.int32)
        t = np.ascontiguousarray(t, dtype=np.float64)
        ch = np.ascontiguousarray(ch, dtype=np.int8)
        lib().orc_process_photons(C.byref(self.sp), self.seed, self.step_index, _p(self.pos), self.N,
                                  _p(pid), _p(t), _p(ch), n, _p(self.flim), C.byref(self.scope_stats))

    def bd_step(self, with_photons: bool = True):
        """One pass of the pipeline loop body; returns the photon batch."""
        self.dynamics_step()
        batch = None
        if with_photons and self.phot is not None:
            batch = self.photon_step()
            if self.sp is not None:
                self.process_photons(batch)
        self.step_index += 1
        return batch

    def finalize_frame(self) -> np.ndarray:
        nd = C.c_int64(0)
        na = C.c_int64(0)
        lib().orc_finalize_frame(C.byref(self.sp), self.seed, self.frame_index, _p(self.flim),
                                 C.byref(nd), C.byref(na))
        self.frame_index += 1
        out = self.flim.copy()
        self.flim[:] = 0
        self.last_dark, self.last_ap = int(nd.value), int(na.value)
        return out
