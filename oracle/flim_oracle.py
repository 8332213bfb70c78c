"""Float64 numpy restatement of the batched FLIM acquisition.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference arm, never by the product package.

The acquisition has no reference function; each piece restates the
reference formula it is built from:

* emitter_counts  -- keyed uniform emitter pixels (the engine's Philox
  stream 200/201 draws, via the oracle library);
* band            -- the emitter-centric Gaussian PSF of
  ed_mrdt/microscope.py:522-631 for an emitter at a pixel centre: square
  window |d| <= R, weights renormalised over the in-field pixels; separable,
  so one 1-D factor per axis;
* bin_probs       -- P(bin b) of t = Exp(tau) + N(0, sigma_irf^2) binned by
  b = int(max(t, 0) / width), b >= n_bins lost (microscope.py:716-803);
* tau_expected    -- the mean-arrival-time readout (analysis.py:87-150) of
  the expected histogram;
* readouts        -- mean_arrival_time and phasor_transform (analysis.py:87-150,
  497-566) of count stacks.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc

from . import oracle as O

NPIX = 256


def replica_seed(seed: int, r: int) -> int:
    return (seed ^ ((0x9E3779B97F4A7C15 * (r + 1)) & 0xFFFFFFFFFFFFFFFF)) & 0xFFFFFFFFFFFFFFFF


def emitter_counts(seed: int, r: int, n_emitters: int, bound_fraction: float) -> np.ndarray:
    """int64 [free, bound][x][y] emitter counts of replica r."""
    s = replica_seed(seed, r)
    e = np.arange(n_emitters, dtype=np.int64)
    u = O.uniforms(s, 0, 200, e, None, two=True)
    v = O.uniforms(s, 0, 201, e, None, two=True)
    x = np.minimum(NPIX - 1, (u[:, 0] * NPIX).astype(np.int64))
    y = np.minimum(NPIX - 1, (u[:, 1] * NPIX).astype(np.int64))
    bound = (v[:, 0] < bound_fraction).astype(np.int64)
    out = np.zeros((2, NPIX, NPIX), dtype=np.int64)
    np.add.at(out, (bound, x, y), 1)
    return out


def band(sigma_px: float, R: int, n: int = NPIX) -> np.ndarray:
    """G[i][j]: weight of an emitter in pixel j seen in pixel i."""
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    d = (i - j).astype(np.float64)
    g = np.where(np.abs(d) <= R, np.exp(-0.5 * (d / sigma_px) ** 2), 0.0)
    return g / g.sum(axis=0, keepdims=True)


def intensity(counts: np.ndarray, G: np.ndarray) -> np.ndarray:
    """[free, bound][x][y] = G . counts . G^T."""
    return np.stack([G @ counts[k].astype(np.float64) @ G.T for k in range(counts.shape[0])])


def _sf(t: np.ndarray, tau: float, s: float) -> np.ndarray:
    a = t / s
    g = a - s / tau
    return 0.5 * erfc(a / math.sqrt(2.0)) + np.exp(-t / tau + 0.5 * (s / tau) ** 2) * 0.5 * erfc(-g / math.sqrt(2.0))


def bin_probs(tau_ns: float, sigma_ns: float, width_ns: float, n_bins: int) -> np.ndarray:
    b = np.arange(n_bins, dtype=np.float64)
    lo = np.where(b == 0, 1.0, _sf(b * width_ns, tau_ns, sigma_ns))
    return lo - _sf((b + 1) * width_ns, tau_ns, sigma_ns)


def expected_hist(I: np.ndarray, h_free: np.ndarray, h_bound: np.ndarray, y_free: float,
                  y_bound: float) -> np.ndarray:
    """Poisson means [x][y][bin]."""
    return I[0][..., None] * (h_free * y_free) + I[1][..., None] * (h_bound * y_bound)


def tau_expected(mu: np.ndarray, width_ns: float) -> np.ndarray:
    t = (np.arange(mu.shape[-1]) + 0.5) * width_ns
    den = mu.sum(axis=-1)
    return np.where(den > 0, (mu @ t) / np.where(den > 0, den, 1.0), 0.0)


def acquire_expected(params, bound_fraction: np.ndarray, replica: int):
    """Float64 expected acquisition of one replica: counts, intensity maps,
    bin probabilities, Poisson means and expected mean arrival times."""
    p = params
    counts = emitter_counts(int(p.seed), replica, int(p.n_emitters), float(bound_fraction[replica]))
    G = band(p.sigma_psf_px, int(p.half_taps))
    I = intensity(counts, G)
    hf = bin_probs(p.tau_free_ns, p.sigma_irf_ns, p.bin_width_ns, int(p.n_bins))
    hb = bin_probs(p.tau_bound_ns, p.sigma_irf_ns, p.bin_width_ns, int(p.n_bins))
    mu = expected_hist(I, hf, hb, p.yield_free, p.yield_bound)
    return dict(counts=counts, G=G, I=I, h=np.stack([hf, hb]), mu=mu, tau=tau_expected(mu, p.bin_width_ns))


def poisson_histograms(mu: np.ndarray, seed: int) -> np.ndarray:
    """A CPU sample of the histograms (numpy's Poisson generator): the timed
    baseline of the acquisition, not a bit-level model of the GPU draws."""
    return np.random.default_rng(seed).poisson(mu).astype(np.uint32)


def readouts(stack: np.ndarray, time_range_s: float, harmonic: int = 1, min_counts_mean: int = 10,
             min_counts_phasor: int = 20) -> dict:
    """mean_arrival_time (ed_mrdt/analysis.py:87-150) and phasor_transform
    (:497-566) of a [..., n_bins] count stack, restated in float64 numpy."""
    data = stack.astype(np.float64)
    n_bins = data.shape[-1]
    t_ns = (np.arange(n_bins) + 0.5) * ((time_range_s / n_bins) * 1e9)
    intensity = data.sum(axis=-1)
    weighted = np.tensordot(data, t_ns, axes=([-1], [0]))
    tau = np.full_like(intensity, np.nan)
    m = intensity >= min_counts_mean
    tau[m] = weighted[m] / intensity[m]
    omega = 2.0 * np.pi * harmonic / time_range_s
    phi = 2.0 * np.pi * harmonic * (np.arange(n_bins) + 0.5) / n_bins
    g_num = np.tensordot(data, np.cos(phi), axes=([-1], [0]))
    s_num = np.tensordot(data, np.sin(phi), axes=([-1], [0]))
    mask = intensity >= min_counts_phasor
    g = np.zeros_like(intensity)
    s = np.zeros_like(intensity)
    g[mask] = g_num[mask] / intensity[mask]
    s[mask] = s_num[mask] / intensity[mask]
    omega_ns = omega * 1e-9
    tau_phi = np.full_like(g, np.nan)
    tau_mod = np.full_like(g, np.nan)
    valid = mask & (g > 1e-10)
    tau_phi[valid] = (s[valid] / g[valid]) / omega_ns
    m_sq = g ** 2 + s ** 2
    mod_valid = valid & (m_sq > 1e-10) & (m_sq < 1.0 - 1e-10)
    tau_mod[mod_valid] = np.sqrt(1.0 / m_sq[mod_valid] - 1.0) / omega_ns
    return dict(intensity=intensity, tau_mean_ns=tau, g=g, s=s, tau_phi_ns=tau_phi, tau_mod_ns=tau_mod)
