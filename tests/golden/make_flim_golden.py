"""Generate tests/golden/flim_acquire.npz from the reference itself.

Run where the reference source tree is present, with EDM_REFERENCE_ROOT set to
it (the directory holding ed_mrdt/):

    python tests/golden/make_flim_golden.py

The batched FLIM acquisition has no reference function; this pins the pieces
it is built from, on the acquisition's own configuration:

* constants: the reference's PSF sigmas (PSF), window half-width, pixel size
  and pixel centres (ConfocalScanner), IRF sigma and bin width
  (TCSPCAccumulator), lifetimes and per-pulse-chain photon means
  (PhotonSimulator);
* PSF weights: the reference's emitter-centric assignment kernel
  (microscope.py:523-631) run for an emitter at the centre of a pixel with
  K photons whose uniforms are the grid (k + 0.5) / K, so pixel counts equal
  K times the weights to within one photon;
* TCSPC: the reference's accumulate (microscope.py:716-803) for N
  mono-exponential arrivals t = -tau ln(u) (photophysics.py:440) at the free
  and FRET-bound lifetimes, seeded;
* readouts: the reference's mean_arrival_time and phasor_transform
  (analysis.py:87-150, 497-566) on a seeded count stack.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from flim_microscopy_simulator_with_causal_inference_b200 import flim_acquire as FA  # noqa: E402
from oracle import refshim as RS  # noqa: E402

EMITTERS = [(100, 120), (0, 0), (3, 250), (255, 128), (17, 240)]
K = 1 << 20
N_TCSPC = 2_000_000


def generate() -> dict:
    RS.import_reference()
    from ed_mrdt.microscope import PSF, ConfocalScanner, TCSPCAccumulator, _assign_photons_emitter_centric
    from ed_mrdt.particles import ParticleState
    from ed_mrdt.photophysics import PhotonSimulator

    cfg = RS.ref_config_from_dict(FA.flim_config())
    psf = PSF(cfg)
    sc = ConfocalScanner(cfg, psf)
    tc = TCSPCAccumulator(cfg)
    st = ParticleState(cfg)
    duty = cfg.scan.dwell_time / cfg.scan.frame_interval
    ps = PhotonSimulator(cfg, st, scan_duty_fraction=duty)
    out = {
        "sigma_um": np.array([psf.sigma_um[c] for c in sorted(psf.sigma_um)]),
        "psf_range_px": sc.psf_range_px, "pixel_size_um": sc.pixel_size_um,
        "pixel_cx": sc.pixel_cx, "pixel_cy": sc.pixel_cy,
        "sigma_irf": tc.sigma_irf, "bin_width": tc.bin_width, "n_bins": tc.n_bins,
        "tau_all": ps._tau_all, "tau_fret_all": ps._tau_fret_all,
        "mean_ph": ps._mean_ph_all, "mean_ph_fret": ps._mean_ph_fret_all, "duty": duty,
    }

    R = sc.psf_range_px
    W = 2 * R + 1
    n_ch = max(psf.sigma_um.keys()) + 1
    sigma_per_ch = np.zeros(max(n_ch, 2))
    for ch, s in psf.sigma_um.items():
        sigma_per_ch[ch] = s
    u = (np.arange(K, dtype=np.float64) + 0.5) / K
    counts = []
    for (i0, j0) in EMITTERS:
        px = np.empty(K, np.int32)
        py = np.empty(K, np.int32)
        det = np.zeros(K, np.bool_)
        n = _assign_photons_emitter_centric(
            np.zeros(K, np.int32), np.zeros(K, np.int8),
            np.array([sc.pixel_cx[i0]]), np.array([sc.pixel_cy[j0]]), K,
            sc.pixel_cx, sc.pixel_cy, sc.nx, sc.ny, sc.pixel_size_um, sc.offset_x, sc.offset_y,
            R, sigma_per_ch, u, px, py, det)
        c = np.zeros((W, W), np.int64)
        np.add.at(c, (px[:n] - i0 + R, py[:n] - j0 + R), 1)
        counts.append(c)
    out["psf_emitters"] = np.array(EMITTERS)
    out["psf_counts"] = np.stack(counts)
    out["psf_K"] = K

    for name, tau, s1, s2 in (("free", ps._tau_all[0], 7, 11), ("bound", ps._tau_fret_all[0], 8, 12)):
        rng = np.random.default_rng(s1)
        t = -tau * np.log(np.maximum(rng.random(N_TCSPC), 1e-30))
        tc.reset()
        z = np.zeros(N_TCSPC, np.int32)
        tc.accumulate(z, z, t, np.zeros(N_TCSPC, np.int8), N_TCSPC, np.random.default_rng(s2))
        out[f"tcspc_{name}"] = tc.flim_stack[0, 0, 0].copy()
    out["tcspc_n"] = N_TCSPC

    # lifetime readouts (analysis.py:87-150, 497-566) of a seeded count stack
    # [2 ch][12][12][256]: exponential decays of mixed lifetimes and brightness,
    # some pixels below the readouts' count thresholds
    from ed_mrdt.analysis import mean_arrival_time, phasor_transform
    rng = np.random.default_rng(5)
    t = (np.arange(256) + 0.5) * 25.0 / 256
    tau = rng.uniform(0.8, 4.0, size=(2, 12, 12, 1))
    bright = rng.choice([0.0, 0.05, 3.0, 40.0], size=(2, 12, 12, 1))
    stack = rng.poisson(bright * np.exp(-t / tau)).astype(np.uint32)
    out["readout_stack"] = stack
    for ch in range(2):
        tau_map, inten = mean_arrival_time(stack, time_range=25e-9, channel=ch, min_counts=10)
        out[f"readout_tau_ch{ch}"] = tau_map
        out[f"readout_intensity_ch{ch}"] = inten
        for h in (1, 2):
            ph = phasor_transform(stack, time_range=25e-9, channel=ch, harmonic=h, min_counts=20)
            for k in ("g", "s", "tau_phi", "tau_mod"):
                out[f"readout_{k}_ch{ch}_h{h}"] = getattr(ph, k)
    return out


def main():
    dest = Path(__file__).resolve().parent / "flim_acquire.npz"
    np.savez_compressed(dest, **generate())
    print("wrote", dest)


if __name__ == "__main__":
    main()
