"""The reference's public per-timestep API, backed by the GPU engine.

Same class names, constructor arguments, methods, attributes and in-place
state semantics as the reference's hot-path objects:

* DynamicsEngine(config, state).step() / .run(n)      (ed_mrdt/dynamics.py:1710-2487)
* PhotonSimulator(config, state, scan_duty_fraction)  (ed_mrdt/photophysics.py:690-1208)
  .evolve_one_bd_step() -> PhotonBatch, .update_fret_rates()
* VirtualMicroscope(config, state).process_photons(batch) / .finalize_frame()
                                                      (ed_mrdt/microscope.py:1021-1233)
* SimulationPipeline(config, ...).run() -> SimulationResult
                                                      (ed_mrdt/pipeline.py:236-738)

Each component works on the ParticleState arrays in place, as the reference
does.  Standalone calls upload the host arrays when they changed and download
the results before returning; SimulationPipeline.run keeps the state on the
GPU for a whole frame (captured into CUDA graphs) and downloads it only for
the per-frame ground truth.

Extra keyword arguments (ignored by the reference): `precision` (64: plain
float64 path, 32: float32 cell-relative path) and `device`.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import params as PR
from .config import ConfigError, SimulationConfig
from .engine import DeviceSystem
from .particles import ParticleState

__all__ = ["DynamicsEngine", "PhotonSimulator", "PhotonBatch", "VirtualMicroscope", "FLIMFrame",
           "SimulationPipeline", "SimulationResult", "FrameResult", "GroundTruth", "SubFrameData", "CellList"]


def _system(config, state, duty: Optional[float], precision: int, device: int) -> DeviceSystem:
    """The state's device system; rebuilt when photophysics (with this duty
    fraction) or another precision is needed."""
    sys = getattr(state, "_device_owner", None)
    need_phot = duty is not None
    if sys is not None and sys.precision == precision and (not need_phot or
                                                          (sys.duty is not None and sys.duty == duty)):
        return sys
    if sys is not None:
        sys.sync_host()
        if duty is None and sys.duty is not None and sys.precision == precision:
            return sys
    return DeviceSystem(config, state, duty, precision, device)


class CellList:
    """Geometry of the reference cell list (dynamics.py:71-173)."""

    def __init__(self, Lx: float, Ly: float, cutoff: float, periodic=(True, True)):
        if cutoff <= 0:
            raise ValueError(f"cutoff must be positive, got {cutoff}")
        self.Lx, self.Ly, self.cutoff = Lx, Ly, cutoff
        self.periodic_x, self.periodic_y = periodic
        self.nx = max(3, int(math.floor(Lx / cutoff)))
        self.ny = max(3, int(math.floor(Ly / cutoff)))
        self.cell_sx = Lx / self.nx
        self.cell_sy = Ly / self.ny


# =============================================================================
# Dynamics
# =============================================================================
class DynamicsEngine:
    def __init__(self, config: SimulationConfig, state: ParticleState, precision: int = 64, device: int = 0):
        self.config = config
        self.state = state
        self.precision = precision
        self.device = device
        sys = _system(config, state, getattr(getattr(state, "_device_owner", None), "duty", None), precision, device)
        d = sys.derived
        self.Lx, self.Ly = config.membrane.size
        self.periodic_x, self.periodic_y = config.membrane.periodic
        self.dt = config.bd_timestep
        self.cutoff_um = d.cutoff_um
        self.cell_list = CellList(self.Lx, self.Ly, self.cutoff_um, (self.periodic_x, self.periodic_y))
        self.sigma_matrix, self.epsilon_matrix, self.harmonic_matrix = d.sigma_matrix, d.epsilon_matrix, d.harmonic_matrix
        self._use_wca, self._use_harmonic = d.use_wca, d.use_harmonic
        self.max_displacement = d.max_displacement
        self._reactions = d.reactions
        self._catalytic_reactions = d.catalytic
        self._compartment_exchanges = d.exchanges
        self._unimolecular_conversions = d.conversions
        self.n_bindings = self.n_dissociations = 0
        self.n_catalytic = self.n_recruited = self.n_detached = self.n_converted = 0
        self._base = None

    @property
    def _sys(self) -> DeviceSystem:
        return _system(self.config, self.state, getattr(getattr(self.state, "_device_owner", None), "duty", None),
                       self.precision, self.device)

    @property
    def forces(self):
        raise AttributeError("per-particle forces are not materialised by the GPU engine")

    def _pull_counters(self, sys):
        c = sys.engine.counters()[0]
        if self._base is None or self._base[0] is not sys:
            self._base = (sys, np.zeros_like(c), (self.n_bindings, self.n_dissociations, self.n_catalytic,
                                                  self.n_recruited, self.n_detached, self.n_converted))
        _, c0, (b, d, ca, r, de, co) = self._base
        dc = c - c0
        self.n_bindings = b + int(dc[PR.C_BINDINGS])
        self.n_dissociations = d + int(dc[PR.C_DISSOC])
        self.n_catalytic = ca + int(dc[PR.C_CATALYTIC])
        self.n_recruited = r + int(dc[PR.C_RECRUITED])
        self.n_detached = de + int(dc[PR.C_DETACHED])
        self.n_converted = co + int(dc[PR.C_CONVERTED])

    def step(self) -> None:
        """One BD timestep (dynamics.py:2150-2465)."""
        self.run(1)

    def run(self, n_steps: int, report_every: int = 0) -> None:
        sys = self._sys
        if self._base is None or self._base[0] is not sys:
            self._base = None
            self._pull_counters(sys)
        sys.ensure_device()
        done = 0
        while done < n_steps:
            chunk = n_steps - done if report_every <= 0 else min(report_every, n_steps - done)
            sys.engine.dynamics_step(chunk)
            sys.mark_device_newer()
            done += chunk
            if report_every > 0 and done % report_every == 0:
                sys.sync_host()
                self._pull_counters(sys)
                n_prod = int(np.sum(self.state.species_id == self._reactions[0]["product"])) if self._reactions else 0
                print(f"  t={done * self.dt:.4f}s | bound={n_prod} "
                      f"| Σbind={self.n_bindings} Σdissoc={self.n_dissociations}")
        sys.sync_host()
        self._pull_counters(sys)


# =============================================================================
# Photophysics
# =============================================================================
@dataclass
class PhotonBatch:
    """Photons of one BD step (photophysics.py:184-211)."""
    particle_idx: np.ndarray
    arrival_time: np.ndarray
    channel: np.ndarray
    pulse_index: np.ndarray
    is_fret: np.ndarray
    n_photons: int = 0

    @staticmethod
    def empty() -> "PhotonBatch":
        return PhotonBatch(np.empty(0, np.int32), np.empty(0, np.float64), np.empty(0, np.int8),
                           np.empty(0, np.int32), np.empty(0, np.bool_), 0)

    def __repr__(self) -> str:
        if self.n_photons > 0:
            u, c = np.unique(self.channel, return_counts=True)
            s = ", ".join(f"ch{a}={b}" for a, b in zip(u, c))
        else:
            s = "empty"
        return f"PhotonBatch(n={self.n_photons}, {s})"


class _DeviceBatch(PhotonBatch):
    """A batch that lives on the GPU; arrays are copied to the host on first
    access.  VirtualMicroscope.process_photons consumes it without a copy."""

    def __init__(self, sys: DeviceSystem, token: int, n: int):
        object.__setattr__(self, "_sys", sys)
        object.__setattr__(self, "_token", token)
        object.__setattr__(self, "_arrays", None)
        object.__setattr__(self, "n_photons", n)

    def _fetch(self):
        if self._arrays is None:
            pid, t, ch, fr = self._sys.engine.photons(0)
            object.__setattr__(self, "_arrays", (pid, t, ch, np.zeros(pid.size, np.int32), fr))
        return self._arrays

    particle_idx = property(lambda s: s._fetch()[0])
    arrival_time = property(lambda s: s._fetch()[1])
    channel = property(lambda s: s._fetch()[2])
    pulse_index = property(lambda s: s._fetch()[3])
    is_fret = property(lambda s: s._fetch()[4])


class PhotonSimulator:
    def __init__(self, config: SimulationConfig, state: ParticleState, scan_duty_fraction: float = 1.0,
                 precision: int = 64, device: int = 0):
        self.config = config
        self.state = state
        self.precision = precision
        self.device = device
        self.scan_duty_fraction = max(0.0, min(1.0, scan_duty_fraction))
        self._active = len(config.fluorophores) > 0
        self.n_fluoro_types = len(config.fluorophores)
        self.total_donor_photons = self.total_acceptor_photons = 0
        self.total_fret_events = self.total_bleached = 0
        if not self._active:
            return
        sys = _system(config, state, self.scan_duty_fraction, precision, device)
        pd = sys.pd
        self._pd = pd
        self.rate_matrices = pd.rates
        self.laser_period = pd.laser_period
        self.n_pulses_per_step = pd.n_pulses
        self._p_excitation = pd.p_exc
        self._T_step_all, self._T_step_fret_all = pd.T_step, pd.T_step_fret
        self._mean_ph_all, self._mean_ph_fret_all = pd.mean_ph, pd.mean_ph_fret
        self._mean_fret_all, self._mean_fret_fret_all = pd.mean_fret, pd.mean_fret_fret
        self._tau_all, self._tau_fret_all = pd.tau_all, pd.tau_fret_all
        self._k_fret_bound_all = pd.k_fret_bound
        self._max_photons = pd.max_photons
        self.donor_channel, self.acceptor_channel = pd.donor_channel, pd.acceptor_channel
        self._k_fret = np.zeros(state.N)
        self._fret_acceptor_idx = np.full(state.N, -1, dtype=np.int32)
        self._token = 0
        self._base = None

    @property
    def _sys(self) -> DeviceSystem:
        return _system(self.config, self.state, self.scan_duty_fraction, self.precision, self.device)

    def update_fret_rates(self) -> None:
        """k_FRET per particle (photophysics.py:1021-1114), on the host mirror
        of the current state (used for ground truth; the GPU kernels evaluate
        the same rule per emitter on the device)."""
        self._sys.sync_host()
        k, acc = host_fret_rates(self._pd, self.config, self.state)
        self._k_fret[:] = k
        self._fret_acceptor_idx[:] = acc

    def evolve_one_bd_step(self) -> PhotonBatch:
        if not self._active:
            return PhotonBatch.empty()
        sys = self._sys
        sys.ensure_device()
        if self._base is None:
            self._base = sys.engine.counters()[0].copy()
        sys.engine.photon_step()
        sys.mark_device_newer()
        n = int(sys.engine.photon_counts()[0])
        self._token += 1
        sys.batch_token = self._token
        batch = _DeviceBatch(sys, self._token, n)
        c = sys.engine.counters()[0] - self._base
        self.total_donor_photons = int(c[PR.C_DONOR_PH])
        self.total_acceptor_photons = int(c[PR.C_ACCEPTOR_PH])
        self.total_fret_events = int(c[PR.C_FRET_PH])
        sys.sync_host()
        self.total_bleached = int(np.sum(self.state.is_bleached))
        return batch

    def get_donor_lifetime_histogram(self, photon_batch: PhotonBatch, n_bins: int = 256,
                                     time_range: float = 25e-9) -> Tuple[np.ndarray, np.ndarray]:
        edges = np.linspace(0, time_range, n_bins + 1)
        t = photon_batch.arrival_time[photon_batch.channel == self.donor_channel]
        counts, _ = np.histogram(t, bins=edges)
        return counts, edges


def host_fret_rates(pd, config, state) -> Tuple[np.ndarray, np.ndarray]:
    """k_FRET and acceptor index per particle as update_fret_rates computes
    them (photophysics.py:528-683, 1021-1114)."""
    N = state.N
    k = np.zeros(N)
    acc = np.full(N, -1, dtype=np.int32)
    if pd is None:
        return k, acc
    for bp in pd.bond_pairs:
        sel = state.has_dye & ~state.is_bleached & (state.dye_type_id == bp["donor"]) & (state.bond_partner >= 0)
        for i in np.flatnonzero(sel):
            partner = state.bond_partner[i]
            if bp["intra"]:
                k[i] = bp["k"]
                acc[i] = -1
            elif state.has_dye[partner] and state.dye_type_id[partner] == bp["acceptor"]:
                k[i] = bp["k"]
                acc[i] = partner
    Lx, Ly = config.membrane.size
    px, py = config.membrane.periodic
    for pp in pd.prox_pairs:
        donors = np.flatnonzero(state.has_dye & state.is_alive & ~state.is_bleached
                                & (state.dye_type_id == pp["donor"]))
        targets = np.flatnonzero(state.is_alive & (state.species_id == pp["target"]))
        r2 = pp["radius_um"] * pp["radius_um"]
        for i in donors:
            tj = targets[targets != i]
            dx = state.positions[tj, 0] - state.positions[i, 0]
            dy = state.positions[tj, 1] - state.positions[i, 1]
            if px:
                dx = np.where(dx > Lx / 2.0, dx - Lx, np.where(dx < -Lx / 2.0, dx + Lx, dx))
            if py:
                dy = np.where(dy > Ly / 2.0, dy - Ly, np.where(dy < -Ly / 2.0, dy + Ly, dy))
            found = bool(np.any(dx * dx + dy * dy < r2))
            k[i] = pp["k_high"] if found else pp["k_low"]
            acc[i] = -1
    return k, acc


# =============================================================================
# Microscope
# =============================================================================
@dataclass
class FLIMFrame:
    """One FLIM frame (microscope.py:973-1012)."""
    flim_stack: np.ndarray
    intensity: np.ndarray
    frame_index: int = 0
    n_signal_photons: int = 0
    n_dark_counts: int = 0
    n_afterpulses: int = 0

    @staticmethod
    def from_stack(flim_stack: np.ndarray, frame_index: int = 0, n_signal: int = 0, n_dark: int = 0,
                   n_ap: int = 0) -> "FLIMFrame":
        return FLIMFrame(flim_stack.copy(), flim_stack.sum(axis=-1).astype(np.float64), frame_index, n_signal,
                         n_dark, n_ap)

    @property
    def total_counts(self) -> int:
        return int(self.flim_stack.sum())

    @property
    def shape(self) -> Tuple[int, ...]:
        return self.flim_stack.shape


class VirtualMicroscope:
    def __init__(self, config: SimulationConfig, state: ParticleState, precision: int = 64, device: int = 0):
        self.config = config
        self.state = state
        self.precision = precision
        self.device = device
        sp, sd = PR.build_scope_params(config)
        self._sd = sd
        self.psf_sigma_um = dict(sd.sigma_um)
        self._frame_index = 0
        self._n_signal = 0
        self._n_bd_steps_in_frame = 0
        self.total_photons_received = 0
        self.total_photons_detected = 0
        self.total_dark_counts = 0
        self.total_afterpulses = 0
        self._host_key = 0

    @property
    def _sys(self) -> DeviceSystem:
        sys = getattr(self.state, "_device_owner", None)
        duty = sys.duty if sys is not None and sys.duty is not None else 1.0
        return _system(self.config, self.state, duty, self.precision, self.device)

    @property
    def frame_shape(self) -> Tuple[int, int, int, int]:
        return self._sd.frame_shape

    def process_photons(self, photon_batch) -> int:
        """Detect one BD step's photons into the TCSPC stacks (microscope.py:1069-1157)."""
        n = int(photon_batch.n_photons)
        if n == 0:
            return 0
        sys = self._sys
        sys.ensure_device()
        eng = sys.engine
        if not (isinstance(photon_batch, _DeviceBatch) and photon_batch._sys is sys
                and photon_batch._token == getattr(sys, "batch_token", None)):
            eng.set_photons(0, photon_batch.particle_idx, photon_batch.arrival_time, photon_batch.channel,
                            photon_batch.is_fret, self._host_key)
            self._host_key += 1
        c0 = eng.counters()[0]
        eng.scope_process()
        c1 = eng.counters()[0]
        nd = int(c1[PR.C_DETECTED] - c0[PR.C_DETECTED])
        self.total_photons_received += n
        self.total_photons_detected += nd
        self._n_signal += nd
        self._n_bd_steps_in_frame += 1
        return nd

    def finalize_frame(self) -> FLIMFrame:
        """Dark counts, afterpulsing, frame extraction (microscope.py:1159-1203)."""
        eng = self._sys.engine
        c0 = eng.counters()[0]
        eng.finalize(self._frame_index)
        stack = eng.flim(0)
        c1 = eng.counters()[0]
        n_dark = int(c1[PR.C_DARK] - c0[PR.C_DARK])
        n_ap = int(c1[PR.C_AFTERPULSE] - c0[PR.C_AFTERPULSE])
        self.total_dark_counts += n_dark
        self.total_afterpulses += n_ap
        frame = FLIMFrame.from_stack(stack, self._frame_index, self._n_signal, n_dark, n_ap)
        eng.reset_flim()
        self._frame_index += 1
        self._n_signal = 0
        self._n_bd_steps_in_frame = 0
        return frame


# =============================================================================
# Pipeline
# =============================================================================
@dataclass
class GroundTruth:
    positions: np.ndarray
    species_id: np.ndarray
    bond_partner: np.ndarray
    is_alive: np.ndarray
    has_dye: np.ndarray
    dye_type_id: np.ndarray
    is_bleached: np.ndarray
    fret_efficiency_exact: np.ndarray
    donor_lifetime_exact: np.ndarray
    n_complexes: int = 0
    n_bleached: int = 0
    n_free_donors: int = 0
    species_counts: Optional[Dict[str, int]] = None


@dataclass
class SubFrameData:
    n_complexes: np.ndarray
    n_bindings: np.ndarray
    n_dissociations: np.ndarray
    n_bleached: np.ndarray
    total_photons: np.ndarray
    mean_fret_E: np.ndarray
    dt_s: float
    steps_per_frame: int
    species_counts: Optional[Dict[str, np.ndarray]] = None
    n_catalytic: Optional[np.ndarray] = None
    n_recruited: Optional[np.ndarray] = None
    n_detached: Optional[np.ndarray] = None
    n_converted: Optional[np.ndarray] = None


@dataclass
class FrameResult:
    frame_index: int
    bio_time: float
    flim_frame: FLIMFrame
    ground_truth: GroundTruth
    n_photons_emitted: int = 0
    n_photons_detected: int = 0
    wall_time_s: float = 0.0

    @property
    def total_counts(self) -> int:
        return self.flim_frame.total_counts


@dataclass
class SimulationResult:
    config: SimulationConfig
    frames: List[FrameResult]
    total_wall_time_s: float = 0.0
    peak_ram_mb: float = 0.0
    total_photons_emitted: int = 0
    total_photons_detected: int = 0
    total_bindings: int = 0
    total_dissociations: int = 0
    total_bleached: int = 0
    subframe_data: Optional[SubFrameData] = None

    @property
    def n_frames(self) -> int:
        return len(self.frames)

    def get_flim_stack(self, frame_idx: int) -> np.ndarray:
        return self.frames[frame_idx].flim_frame.flim_stack

    def get_intensity_series(self) -> np.ndarray:
        return np.array([f.total_counts for f in self.frames])

    def get_complex_count_series(self) -> np.ndarray:
        return np.array([f.ground_truth.n_complexes for f in self.frames])

    def get_bleaching_series(self) -> np.ndarray:
        return np.array([f.ground_truth.n_bleached for f in self.frames])

    def summary(self) -> str:
        return "\n".join([
            "ED-MRDT Simulation Result",
            f"  Config: {self.config.name}",
            f"  Frames: {self.n_frames}",
            f"  Wall time: {self.total_wall_time_s:.1f} s",
            f"  Photons emitted: {self.total_photons_emitted:,}",
            f"  Photons detected: {self.total_photons_detected:,}",
            f"  Bindings: {self.total_bindings:,}",
            f"  Dissociations: {self.total_dissociations:,}",
            f"  Final bleached: {self.total_bleached}",
        ])


def subframe_series(rows: np.ndarray, prev_counters: np.ndarray, config: SimulationConfig,
                    fret_E_cls: np.ndarray) -> dict:
    """The reference's per-step sub-frame series (pipeline.py:567-642) from
    census rows recorded on the device, one row per BD step ([n][fields], one
    replica): event and photon counts are differences of the cumulative
    counters (prev_counters = the 7 counters before the first row), complexes
    are alive bonded particles / 2, and the mean FRET efficiency is taken
    over the alive unbleached carriers of dye 0 -- per donor
    k tau_D / (1 + k tau_D) by FRET class (fret_E_cls, dye 0's row of the
    exact table) in proximity mode, E(r/R0) times bound / donors in bond
    mode."""
    cum = rows[:, PR.CEN_COUNTERS:PR.CEN_COUNTERS + 7]
    d = np.diff(np.vstack([np.asarray(prev_counters, dtype=np.int64)[None, :7], cum]), axis=0)
    n_bound = rows[:, PR.CEN_BOND_ALIVE] // 2
    out = {"n_complexes": n_bound, "n_bleached": rows[:, PR.CEN_BLEACHED].copy()}
    for k, name in enumerate(("n_bindings", "n_dissociations", "n_catalytic", "n_recruited", "n_detached",
                              "n_converted", "total_photons")):
        out[name] = d[:, k]
    out["species"] = {sp.name: rows[:, PR.CEN_SPECIES + si].copy() for si, sp in enumerate(config.species)}
    mean = np.zeros(rows.shape[0])
    if config.fret_pairs:
        fp = config.fret_pairs[0]
        n_don = rows[:, PR.CEN_DONORS]
        has = n_don > 0
        if getattr(fp, "fret_mode", "bond") == "proximity":
            cls = rows[:, PR.CEN_DONOR_CLS:PR.CEN_DONOR_CLS + PR.MAX_FCLASS]
            tot = (cls * np.asarray(fret_E_cls, dtype=np.float64)[None, :PR.MAX_FCLASS]).sum(axis=1)
            mean[has] = tot[has] / n_don[has]
        else:
            e_const = 1.0 / (1.0 + (fp.intra_complex_distance / fp.R0) ** 6)
            for k in np.nonzero(has)[0]:
                nb, nd = int(n_bound[k]), int(n_don[k])
                mean[k] = e_const * nb / (nb + (nd - nb))
    out["mean_fret_E"] = mean
    return out


class SimulationPipeline:
    """BD -> photophysics -> microscope -> FLIM frames (pipeline.py:236-738),
    device-resident within each frame."""

    def __init__(self, config: SimulationConfig, progress_callback: Optional[Callable] = None,
                 record_subframe: bool = False, precision: int = 64, device: int = 0, graph_chunk: int = 100,
                 h5_path: Optional[str] = None):
        """h5_path: stream every frame to an HDF5 file in the reference's
        layout (ed_mrdt/io.py) from a host thread while the next frame runs."""
        self.config = config
        self.h5_path = h5_path
        self.record_subframe = record_subframe
        self.precision = precision
        self.device = device
        self.graph_chunk = graph_chunk
        dt = config.bd_timestep
        fi = config.scan.frame_interval
        n_frames = getattr(config, "n_frames", config.scan.n_frames)
        if fi <= 0:
            raise ConfigError("frame_interval must be positive")
        if dt <= 0:
            raise ConfigError("bd_timestep must be positive")
        self.n_bd_per_frame = int(round(fi / dt))
        if self.n_bd_per_frame < 1:
            raise ConfigError(f"frame_interval ({fi}s) < bd_timestep ({dt}s)")
        if abs(self.n_bd_per_frame * dt - fi) / fi > 0.01:
            raise ConfigError(f"frame_interval ({fi}s) is not an integer multiple of bd_timestep ({dt}s)")
        self.n_frames = n_frames
        self.dt = dt
        self.frame_interval = self.n_bd_per_frame * dt
        self._progress = progress_callback if progress_callback is not None else self._default_progress
        self._state = self._dynamics = self._photon_sim = self._microscope = None

    @staticmethod
    def _default_progress(frame_idx: int, n_frames: int, msg: str) -> None:
        print(f"  [{frame_idx + 1}/{n_frames}] {msg}")

    def _init_components(self) -> None:
        cfg = self.config
        self._state = ParticleState(cfg)
        duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
        self._photon_sim = PhotonSimulator(cfg, self._state, scan_duty_fraction=duty, precision=self.precision,
                                           device=self.device)
        self._dynamics = DynamicsEngine(cfg, self._state, precision=self.precision, device=self.device)
        self._microscope = VirtualMicroscope(cfg, self._state, precision=self.precision, device=self.device)

    def _extract_ground_truth(self) -> GroundTruth:
        """Exact per-frame state (pipeline.py:357-455).  FRET classes, E and
        tau_DA of every donor, and the bond / bleaching / species / free-donor
        counts are evaluated on the device (edm_ground_truth); the state
        arrays are the host copies the frame loop has just synced."""
        st = self._state
        cfg = self.config
        eng = st._device_owner.engine
        fret_E, tau_DA, census = eng.ground_truth()
        c = census[0]
        n_free = 0
        for fp in cfg.fret_pairs:
            for fi, f in enumerate(cfg.fluorophores):
                if f.name == fp.donor_type and fi < PR.MAX_FLUO:
                    n_free += int(c[PR.CEN_FREE_DYE + fi])
        counts = {sp.name: int(c[PR.CEN_SPECIES + i]) for i, sp in enumerate(cfg.species)}
        return GroundTruth(st.positions.copy(), st.species_id.copy(), st.bond_partner.copy(), st.is_alive.copy(),
                           st.has_dye.copy(), st.dye_type_id.copy(), st.is_bleached.copy(), fret_E, tau_DA,
                           int(c[PR.CEN_BOND_ALL]) // 2, int(c[PR.CEN_BLEACHED]), n_free, counts)

    def run(self) -> SimulationResult:
        t_all = time.perf_counter()
        self._init_components()
        sys = self._state._device_owner
        eng = sys.engine
        self._progress(-1, self.n_frames, f"Initialized: {self._state.N} particles, {self.n_bd_per_frame} BD "
                                          f"steps/frame, {self.n_frames} frames.")
        import torch
        stream = torch.cuda.Stream(device=self.device)
        frames: List[FrameResult] = []
        tot_em = tot_det = 0
        sub = None
        c_prev = eng.counters()[0].copy()
        sys.ensure_device()
        if self.record_subframe:
            sub = self._subframe_alloc()
            eng.record_enable(self.n_bd_per_frame)
            sub["prev"] = c_prev[:7].copy()
        step0 = eng.get_step()
        writer = None
        if self.h5_path is not None:
            from .io import StreamingHDF5Writer
            writer = StreamingHDF5Writer(self.h5_path, self.config, self._state.N).open()
        for fidx in range(self.n_frames):
            tf = time.perf_counter()
            eng.pipeline_steps(self.n_bd_per_frame, True, self.graph_chunk, stream=stream)
            if self.record_subframe:
                rows = eng.record_read(step0 + fidx * self.n_bd_per_frame, self.n_bd_per_frame, stream=stream)
                self._decode_subframe(sub, rows[:, 0, :])
            stream.synchronize()
            sys.mark_device_newer()
            c_now = eng.counters()[0].copy()
            em = int(c_now[PR.C_PHOTONS] - c_prev[PR.C_PHOTONS])
            det = int(c_now[PR.C_DETECTED] - c_prev[PR.C_DETECTED])
            self._microscope._n_signal = det
            frame = self._microscope.finalize_frame()
            c_prev = eng.counters()[0].copy()
            sys.sync_host()
            gt = self._extract_ground_truth()
            bio = (fidx + 1) * self.frame_interval
            wall = time.perf_counter() - tf
            frames.append(FrameResult(fidx, bio, frame, gt, em, det, wall))
            if writer is not None:
                writer.write_frame(frames[-1])
            tot_em += em
            tot_det += det
            self._progress(fidx, self.n_frames, f"t={bio:.3f}s | photons={det:,} | counts={frame.total_counts:,} "
                                                f"| complexes={gt.n_complexes} | bleached={gt.n_bleached} "
                                                f"| wall={wall:.2f}s")
        if self.record_subframe:
            eng.record_enable(0)
        # the reference leaves PhotonSimulator._k_fret at the last frame's update_fret_rates
        self._photon_sim.update_fret_rates()
        c = eng.counters()[0]
        res = SimulationResult(self.config, frames, time.perf_counter() - t_all, 0.0, tot_em, tot_det,
                               int(c[PR.C_BINDINGS]), int(c[PR.C_DISSOC]), int(np.sum(self._state.is_bleached)),
                               self._subframe_result(sub) if sub is not None else None)
        if writer is not None:
            writer.finalize(total_wall_time=res.total_wall_time_s, peak_ram_mb=res.peak_ram_mb,
                            total_bindings=res.total_bindings, total_dissociations=res.total_dissociations)
            writer.close()
        self._dynamics._pull_counters(sys)
        self._progress(self.n_frames - 1, self.n_frames, f"DONE. {res.summary()}")
        return res

    # ---- per-step recording (pipeline.py:567-642) ---------------------------
    def _subframe_alloc(self):
        n = self.n_frames * self.n_bd_per_frame
        z = lambda: np.zeros(n, dtype=np.int32)
        return dict(i=0, n_complexes=z(), n_bindings=z(), n_dissociations=z(), n_bleached=z(), total_photons=z(),
                    mean_fret_E=np.zeros(n), species={sp.name: z() for sp in self.config.species},
                    n_catalytic=z(), n_recruited=z(), n_detached=z(), n_converted=z())

    def _decode_subframe(self, sub, rows: np.ndarray) -> None:
        """Append one frame of census rows to the sub-frame series."""
        e_cls = np.array(self._state._device_owner.engine._phot[0].fret_E[0][:PR.MAX_FCLASS])
        series = subframe_series(rows, sub["prev"], self.config, e_cls)
        sub["prev"] = rows[-1, PR.CEN_COUNTERS:PR.CEN_COUNTERS + 7].copy()
        sl = slice(sub["i"], sub["i"] + rows.shape[0])
        for k, v in series.items():
            if k == "species":
                for name, arr in v.items():
                    sub["species"][name][sl] = arr
            else:
                sub[k][sl] = v
        sub["i"] = sl.stop

    def _subframe_result(self, sub) -> SubFrameData:
        return SubFrameData(
            n_complexes=sub["n_complexes"], n_bindings=sub["n_bindings"], n_dissociations=sub["n_dissociations"],
            n_bleached=sub["n_bleached"], total_photons=sub["total_photons"], mean_fret_E=sub["mean_fret_E"],
            dt_s=self._dynamics.dt, steps_per_frame=self.n_bd_per_frame, species_counts=sub["species"],
            n_catalytic=sub["n_catalytic"], n_recruited=sub["n_recruited"], n_detached=sub["n_detached"],
            n_converted=sub["n_converted"])
