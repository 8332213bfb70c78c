"""The float64 oracle of the batched FLIM acquisition, pinned against the
reference (tests/golden/flim_acquire.npz, written by make_flim_golden.py):
host-derived constants, PSF weights of the emitter-centric assignment kernel,
and TCSPC histograms of the reference's accumulator."""
import math
from pathlib import Path

import numpy as np
import pytest

from flim_microscopy_simulator_with_causal_inference_b200 import flim_acquire as FA
from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
from oracle import flim_oracle as FO

GOLDEN = Path(__file__).resolve().parent / "golden" / "flim_acquire.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def derived():
    return FA.derive_flim(config_from_dict(FA.flim_config()), 50_000, 1000.0)


def test_host_constants_equal_the_reference(gold, derived):
    d = derived
    assert d.sigma_psf_um == pytest.approx(float(gold["sigma_um"][0]), rel=1e-15)
    assert d.half_taps == int(gold["psf_range_px"]) == 15  # 31-tap window
    assert d.pixel_size_um == pytest.approx(float(gold["pixel_size_um"]), rel=1e-15)
    assert d.sigma_irf_ns == pytest.approx(float(gold["sigma_irf"]) * 1e9, rel=1e-14)
    assert d.bin_width_ns == pytest.approx(float(gold["bin_width"]) * 1e9, rel=1e-14)
    assert d.n_bins == int(gold["n_bins"]) == 256
    assert d.tau_free_ns == pytest.approx(float(gold["tau_all"][0]) * 1e9, rel=1e-14)
    assert d.tau_bound_ns == pytest.approx(float(gold["tau_fret_all"][0]) * 1e9, rel=1e-14)
    assert d.mean_ph_free == pytest.approx(float(gold["mean_ph"][0, 0]), rel=1e-12)
    assert d.mean_ph_bound == pytest.approx(float(gold["mean_ph_fret"][0, 0]), rel=1e-12)
    assert d.scan_duty == pytest.approx(float(gold["duty"]), rel=1e-15)
    # the donor PSF sigma is 100 nm and the yield ratio is the FRET-quenched one
    assert abs(d.sigma_psf_um - 0.1) < 1e-4
    assert d.yield_bound / d.yield_free == pytest.approx(d.mean_ph_bound / d.mean_ph_free, rel=1e-15)


def test_band_columns_are_normalised_over_the_field(derived):
    G = FO.band(derived.sigma_psf_px, derived.half_taps)
    np.testing.assert_allclose(G.sum(axis=0), 1.0, rtol=0, atol=1e-14)
    assert np.count_nonzero(G[:, 128]) == 2 * derived.half_taps + 1
    assert np.count_nonzero(G[:, 0]) == derived.half_taps + 1


def test_band_weights_equal_the_reference_assignment_kernel(gold, derived):
    """Pixel counts of K grid photons through the reference kernel equal K
    times the separable band weights to within the grid quantum."""
    G = FO.band(derived.sigma_psf_px, derived.half_taps)
    R = derived.half_taps
    K = int(gold["psf_K"])
    for (i0, j0), counts in zip(gold["psf_emitters"], gold["psf_counts"]):
        w = np.zeros((2 * R + 1, 2 * R + 1))
        for a in range(-R, R + 1):
            for b in range(-R, R + 1):
                i, j = i0 + a, j0 + b
                if 0 <= i < 256 and 0 <= j < 256:
                    w[a + R, b + R] = G[i, i0] * G[j, j0]
        assert counts.sum() == K
        assert np.abs(counts - K * w).max() <= 1.01, (i0, j0)


@pytest.mark.parametrize("which", ["free", "bound"])
def test_bin_probabilities_match_the_reference_tcspc(gold, derived, which):
    tau = derived.tau_free_ns if which == "free" else derived.tau_bound_ns
    h = FO.bin_probs(tau, derived.sigma_irf_ns, derived.bin_width_ns, derived.n_bins)
    obs = gold[f"tcspc_{which}"].astype(np.float64)
    N = int(gold["tcspc_n"])
    exp = N * h
    m = exp >= 5.0
    chi2 = float((((obs - exp) ** 2) / exp)[m].sum())
    dof = int(m.sum())
    assert abs(chi2 - dof) < 6.0 * math.sqrt(2.0 * dof), (chi2, dof)
    # photons past the 25 ns window are lost, as in the reference
    lost = N - obs.sum()
    assert abs(lost - N * (1.0 - h.sum())) < 6.0 * math.sqrt(max(1.0, N * (1.0 - h.sum()))) + 1


def test_bin_probabilities_fold_negative_times_into_bin_zero(derived):
    h = FO.bin_probs(derived.tau_free_ns, derived.sigma_irf_ns, derived.bin_width_ns, derived.n_bins)
    tail = FO._sf(np.array([25.0]), derived.tau_free_ns, derived.sigma_irf_ns)[0]
    assert h.sum() + tail == pytest.approx(1.0, abs=1e-15)
    assert h[0] > 0.5 * derived.bin_width_ns / derived.tau_free_ns  # half the IRF mass lands in bin 0


def test_emitter_counts_and_expected_photons(derived):
    p, _ = FA.build_flim_params(config_from_dict(FA.flim_config()), 2, 50_000, 1000.0, seed=99)
    bf = np.array([0.0, 1.0])
    e0 = FO.acquire_expected(p, bf, 0)
    e1 = FO.acquire_expected(p, bf, 1)
    assert e0["counts"].sum() == 50_000 and e0["counts"][1].sum() == 0
    assert e1["counts"][0].sum() == 0
    # emitters near the edge keep their photons (renormalised window)
    assert e0["I"].sum() == pytest.approx(50_000, rel=1e-12)
    # an all-free field collects the budget minus the photons past the window
    h = e0["h"][0]
    assert e0["mu"].sum() / 65536 == pytest.approx(1000.0 * h.sum(), rel=1e-12)
    # the expected lifetime readout of a pure population is its truncated mean
    m = e0["mu"].sum(axis=-1) > 1
    t = (np.arange(256) + 0.5) * derived.bin_width_ns
    np.testing.assert_allclose(e0["tau"][m], (h @ t) / h.sum(), rtol=1e-12)


def test_mean_arrival_time_readout_matches_the_formula():
    rng = np.random.default_rng(1)
    stack = rng.integers(0, 5, size=(4, 4, 256)).astype(np.uint32)
    stack[0, 0] = 0
    tau, inten = FA.mean_arrival_time(stack, 25e-9, min_counts=10)
    t = (np.arange(256) + 0.5) * (25.0 / 256)
    assert math.isnan(tau[0, 0]) and inten[0, 0] == 0
    assert tau[1, 1] == pytest.approx((stack[1, 1] * t).sum() / stack[1, 1].sum(), rel=1e-14)


@pytest.mark.parametrize("ch", [0, 1])
@pytest.mark.parametrize("h", [1, 2])
def test_readouts_equal_the_reference_analysis_functions(gold, ch, h):
    stack = gold["readout_stack"][ch]
    r = FO.readouts(stack, 25e-9, harmonic=h, min_counts_mean=10, min_counts_phasor=20)
    np.testing.assert_allclose(r["intensity"], gold[f"readout_intensity_ch{ch}"], rtol=0, atol=0)
    np.testing.assert_allclose(r["tau_mean_ns"], gold[f"readout_tau_ch{ch}"], rtol=1e-14, equal_nan=True)
    for k, name in (("g", "g"), ("s", "s"), ("tau_phi_ns", "tau_phi"), ("tau_mod_ns", "tau_mod")):
        np.testing.assert_allclose(r[k], gold[f"readout_{name}_ch{ch}_h{h}"], rtol=1e-13, atol=1e-15,
                                   equal_nan=True, err_msg=k)
    assert np.isnan(r["tau_mean_ns"]).any() and (~np.isnan(r["tau_mean_ns"])).any()
