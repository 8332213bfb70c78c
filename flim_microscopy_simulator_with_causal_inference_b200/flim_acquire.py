"""Batched FLIM acquisition from expected intensities (the "config 4" workload).

R replicas of a 256 x 256-pixel field of view, each holding n_emitters donors
at uniform pixels, bound (FRET-quenched) with a per-replica fraction.  One
acquisition produces a uint32 TCSPC histogram [R][256][256][n_bins]:
emitter maps -> PSF projection on tcgen05 tensor cores -> Poisson histogram
writer (csrc/edm_flim.cu).

The reference forms FLIM stacks photon by photon (VirtualMicroscope,
ed_mrdt/microscope.py:1069-1203) and has no batched acquisition.  Every
constant of this one is derived with the reference's own formulas from the
same configuration:

* PSF sigma per channel: 0.21 lambda / NA for illumination and detection,
  combined confocally (microscope.py:97-151); the window half-width
  R = ceil(4 sigma_max / pixel) (microscope.py:281-282); weights renormalised
  over the in-field pixels (microscope.py:522-631);
* IRF sigma sqrt((FWHM_laser / 2.3548)^2 + jitter^2) (microscope.py:674-677);
  bins of time_range / n_bins, negative times in bin 0, late times lost
  (microscope.py:778-803);
* lifetimes 1/k_S1 and 1/(k_S1 + k_FRET) and the ratio of photon yields
  bound/free from the per-pulse chain with the FRET-bound rate
  (photophysics.py:218-331, 911-951), at the scan duty fraction
  dwell / frame_interval (pipeline.py:343-344).

The photon budget fixes the absolute yield: an all-free field of view would
collect `photon_budget` photons per pixel on average.
"""
from __future__ import annotations

import copy
import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import engine as E
from . import params as PR
from . import workloads as W
from .config import SimulationConfig, config_from_dict

NPIX = 256

# Donor photophysics of the workload: S1 -> S0 3.58e8 /s, ISC 1e6 /s,
# T1 -> S0 1e5 /s, bleaching 1e-6 per excitation (~1e-6 k_S1 = 359 /s).
DONOR_RATES = {"S1": {"S0": 3.58e8, "T1": 1.0e6, "bleached": 359.0}, "T1": {"S0": 1.0e5}}
# 27.6 nm pixels: the donor PSF sigma is 100 nm and the widest channel's
# sigma (103 nm) gives R = 15, a 31-tap window.
PIXEL_SIZE_NM = 27.6


def flim_config(pixels: int = NPIX, pixel_size_nm: float = PIXEL_SIZE_NM, seed: int = 42) -> dict:
    """The workload's configuration as a YAML-equivalent dict: the PIP3/PTEN
    membrane configuration with the donor rates above and a 256 x 256 scan."""
    d = W.membrane_pip3_pten(pixels=pixels, pixel_size_nm=pixel_size_nm, seed=seed)
    d["fluorophores"][0]["thermal_rates"] = copy.deepcopy(DONOR_RATES)
    return d


@dataclass
class FlimDerived:
    sigma_psf_um: float
    pixel_size_um: float
    sigma_psf_px: float
    half_taps: int
    n_bins: int
    bin_width_ns: float
    sigma_irf_ns: float
    tau_free_ns: float
    tau_bound_ns: float
    mean_ph_free: float    # per BD step, per-pulse chain (no FRET)
    mean_ph_bound: float   # per BD step, per-pulse chain at the FRET-bound rate
    yield_free: float      # detected photons per free emitter per acquisition
    yield_bound: float
    scan_duty: float


def derive_flim(config: SimulationConfig, n_emitters: int, photon_budget: float = 1000.0) -> FlimDerived:
    """Constants of the acquisition from the reference's formulas (module doc)."""
    scope_p, scope = PR.build_scope_params(config)
    duty = config.scan.dwell_time / config.scan.frame_interval if config.scan.frame_interval > 0 else 1.0
    n_lab = 1
    phot = PR.derive_photophysics(config, n_lab, n_lab, duty)
    donor = phot.donor_channel
    mean_free = float(phot.mean_ph[donor, 0])
    mean_bound = float(phot.mean_ph_fret[donor, 0])
    npx = config.scan.pixels_x * config.scan.pixels_y
    y_free = photon_budget * npx / max(1, n_emitters)
    y_bound = y_free * (mean_bound / mean_free if mean_free > 0 else 0.0)
    sig = scope.sigma_um[donor]
    return FlimDerived(
        sigma_psf_um=sig, pixel_size_um=scope.pixel_size_um, sigma_psf_px=sig / scope.pixel_size_um,
        half_taps=scope.psf_range_px, n_bins=config.tcspc.n_bins,
        bin_width_ns=config.tcspc.bin_width * 1e9, sigma_irf_ns=scope.sigma_irf * 1e9,
        tau_free_ns=float(phot.tau_all[donor]) * 1e9, tau_bound_ns=float(phot.tau_fret_all[donor]) * 1e9,
        mean_ph_free=mean_free, mean_ph_bound=mean_bound, yield_free=y_free, yield_bound=y_bound,
        scan_duty=duty)


def build_flim_params(config: SimulationConfig, n_replicas: int, n_emitters: int = 50_000,
                      photon_budget: float = 1000.0, seed: int = 0):
    d = derive_flim(config, n_emitters, photon_budget)
    p = PR.EdmFlimParams()
    p.nx, p.ny = config.scan.pixels_x, config.scan.pixels_y
    p.n_replicas, p.n_emitters, p.n_bins, p.half_taps = n_replicas, n_emitters, d.n_bins, d.half_taps
    p.seed = seed & 0xFFFFFFFFFFFFFFFF
    p.bin_width_ns, p.sigma_irf_ns, p.sigma_psf_px = d.bin_width_ns, d.sigma_irf_ns, d.sigma_psf_px
    p.tau_free_ns, p.tau_bound_ns = d.tau_free_ns, d.tau_bound_ns
    p.yield_free, p.yield_bound = d.yield_free, d.yield_bound
    return p, d


def replica_seed(seed: int, r: int) -> int:
    """edm_flim_replica_seed of include/edm_b200.h."""
    return (seed ^ ((0x9E3779B97F4A7C15 * (r + 1)) & 0xFFFFFFFFFFFFFFFF)) & 0xFFFFFFFFFFFFFFFF


def bound_fractions(n_replicas: int, seed: int) -> np.ndarray:
    """Per-replica bound fraction ~ U(0, 1)."""
    return np.random.default_rng(seed).random(n_replicas)


HIST, INTENSITY, COUNTS, TAU, BINS, ERROR = range(6)


class FlimAcquisition:
    """Device-resident batched acquisition (C ABI: edm_flim_*).

    Raises when the CUDA library or the GPU is missing: there is no CPU
    fallback.
    """

    def __init__(self, config: SimulationConfig | dict, n_replicas: int, n_emitters: int = 50_000,
                 photon_budget: float = 1000.0, seed: int = 0, bound_fraction: Optional[np.ndarray] = None,
                 device: int = 0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("FlimAcquisition needs a CUDA device (no CPU fallback)")
        if isinstance(config, dict):
            config = config_from_dict(config)
        self.config = config
        self.lib = E.load_library()
        self.params, self.derived = build_flim_params(config, n_replicas, n_emitters, photon_budget, seed)
        self.n_replicas, self.n_bins = n_replicas, self.params.n_bins
        self.device = device
        self._h = C.c_void_p()
        self._check(self.lib.edm_flim_create(C.byref(self.params), device, C.byref(self._h)))
        bf = bound_fractions(n_replicas, seed) if bound_fraction is None else np.asarray(bound_fraction)
        self.set_inputs(bf, seed)

    def _check(self, rc: int):
        if rc != 0:
            raise RuntimeError(f"edm_flim: {self.lib.edm_last_error().decode()} (code {rc})")

    def set_inputs(self, bound_fraction: np.ndarray, seed: int, stream: Optional[int] = None) -> None:
        bf = np.ascontiguousarray(bound_fraction, dtype=np.float64)
        if bf.shape != (self.n_replicas,):
            raise ValueError(f"bound_fraction must have shape ({self.n_replicas},)")
        self.bound_fraction = bf
        self.seed = seed
        self._check(self.lib.edm_flim_set_inputs(self._h, bf.ctypes.data_as(C.c_void_p), seed & (2**64 - 1),
                                                 stream))
        if stream is None:
            import torch
            torch.cuda.synchronize(self.device)

    def project(self, stream: Optional[int] = None) -> None:
        self._check(self.lib.edm_flim_project(self._h, stream))

    def histograms(self, with_tau: bool = True, stream: Optional[int] = None) -> None:
        self._check(self.lib.edm_flim_histograms(self._h, int(with_tau), stream))

    def acquire(self, stream: Optional[int] = None) -> None:
        self._check(self.lib.edm_flim_acquire(self._h, stream))

    def device_ptr(self, what: int):
        ptr, nbytes = C.c_void_p(), C.c_int64()
        self._check(self.lib.edm_flim_device_ptr(self._h, what, C.byref(ptr), C.byref(nbytes)))
        return ptr.value, nbytes.value

    def read(self, what: int, replica: int = -1, out: Optional[np.ndarray] = None) -> np.ndarray:
        shapes = {HIST: ((NPIX, NPIX, self.n_bins), np.uint32), INTENSITY: ((2, NPIX, NPIX), np.float32),
                  COUNTS: ((2, NPIX, NPIX), np.int32), TAU: ((NPIX, NPIX), np.float64),
                  BINS: ((2, self.n_bins), np.float64), ERROR: ((), np.uint32)}
        shape, dt = shapes[what]
        per_rep = what in (HIST, INTENSITY, COUNTS, TAU)
        if per_rep and replica < 0:
            shape = (self.n_replicas,) + shape
        if out is None:
            out = np.empty(shape, dtype=dt)
        self._check(self.lib.edm_flim_read(self._h, what, replica, out.ctypes.data_as(C.c_void_p), out.nbytes,
                                           None))
        return out

    def read_hist_narrow(self, bits: int = 8, replica: int = -1, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The histograms as `bits`-bit counts (8 or 16), narrowed on the
        device (edm_flim_read_hist_narrow): lossless, or OverflowError when a
        count does not fit (read wider then)."""
        dt = {8: np.uint8, 16: np.uint16}[bits]
        shape = (NPIX, NPIX, self.n_bins) if replica >= 0 else (self.n_replicas, NPIX, NPIX, self.n_bins)
        if out is None:
            out = np.empty(shape, dtype=dt)
        if out.dtype != dt or out.size != int(np.prod(shape)) or not out.flags.c_contiguous:
            raise ValueError(f"read_hist_narrow: out must be a contiguous {np.dtype(dt).name} array of {shape}")
        rc = self.lib.edm_flim_read_hist_narrow(self._h, int(replica), int(bits), out.ctypes.data_as(C.c_void_p),
                                                out.nbytes, None)
        if rc == -5:  # EDM_ERANGE
            raise OverflowError(self.lib.edm_last_error().decode())
        self._check(rc)
        return out

    def read_hist_narrow_async(self, out: np.ndarray, bits: int = 8, stream: Optional[int] = None) -> None:
        """edm_flim_read_hist_narrow_async: every replica's histograms as
        `bits`-bit counts into `out` (pinned, (R, 256, 256, n_bins) of
        uint8 / uint16), the copy overlapping what `stream` does next; read
        `out` after read_wait().  OverflowError (before any copy) when a count
        does not fit."""
        dt = {8: np.uint8, 16: np.uint16}[bits]
        if out.dtype != dt or out.size != self.n_replicas * NPIX * NPIX * self.n_bins or not out.flags.c_contiguous:
            raise ValueError("read_hist_narrow_async: out must be a contiguous array of every bin")
        self._pending_out = out
        rc = self.lib.edm_flim_read_hist_narrow_async(self._h, int(bits), out.ctypes.data_as(C.c_void_p),
                                                      out.nbytes, stream)
        if rc == -5:  # EDM_ERANGE
            raise OverflowError(self.lib.edm_last_error().decode())
        self._check(rc)

    def read_wait(self) -> None:
        """Wait for the last overlapped histogram read (edm_flim_read_wait)."""
        self._check(self.lib.edm_flim_read_wait(self._h))
        self._pending_out = None

    def error_word(self) -> int:
        w = C.c_uint32()
        self._check(self.lib.edm_flim_get_error(self._h, C.byref(w)))
        return int(w.value)

    def close(self) -> None:
        if self._h:
            self.lib.edm_flim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mean_arrival_time(stack: np.ndarray, time_range_s: float, min_counts: int = 10):
    """Per-pixel mean arrival time in ns of a [nx, ny, n_bins] histogram stack
    and its intensity; NaN below min_counts (analysis.py:87-150)."""
    data = stack.astype(np.float64)
    n_bins = data.shape[-1]
    t_ns = (np.arange(n_bins) + 0.5) * (time_range_s / n_bins) * 1e9
    intensity = data.sum(axis=-1)
    weighted = np.tensordot(data, t_ns, axes=([-1], [0]))
    tau = np.full_like(intensity, np.nan)
    m = intensity >= min_counts
    tau[m] = weighted[m] / intensity[m]
    return tau, intensity
