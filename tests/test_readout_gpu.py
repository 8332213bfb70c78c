"""Device lifetime readouts (edm_readout_lifetimes): mean arrival time and
phasor coordinates of count stacks against the reference's own
analysis.mean_arrival_time / phasor_transform outputs (golden) and against
the float64 restatement on engine and acquisition stacks.  Tolerance: rtol
1e-12 (float64 sums in another order), NaN where the reference has NaN."""
from pathlib import Path

import numpy as np
import pytest
import torch

from flim_microscopy_simulator_with_causal_inference_b200 import flim_acquire as FA
from flim_microscopy_simulator_with_causal_inference_b200 import readouts as RD
from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
from oracle import flim_oracle as FO

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "flim_acquire.npz"


def _close(dev: np.ndarray, ref: dict, shape):
    for i, k in enumerate(RD.FIELDS):
        np.testing.assert_allclose(dev[i].reshape(shape), ref[k], rtol=1e-12, atol=1e-14, equal_nan=True,
                                   err_msg=k)


@pytest.mark.parametrize("h", [1, 2])
def test_device_readouts_equal_the_reference_functions(h):
    gold = np.load(GOLDEN)
    stack = np.ascontiguousarray(gold["readout_stack"])  # [2][12][12][256]
    dev_stack = torch.from_numpy(stack.view(np.int32)).cuda()
    out = RD.lifetimes_device(dev_stack.data_ptr(), 2 * 12 * 12, 256, 25e-9, harmonic=h).cpu().numpy()
    for ch in range(2):
        sl = out[:, ch * 144:(ch + 1) * 144]
        np.testing.assert_array_equal(sl[0].reshape(12, 12), gold[f"readout_intensity_ch{ch}"])
        np.testing.assert_allclose(sl[1].reshape(12, 12), gold[f"readout_tau_ch{ch}"], rtol=1e-12, equal_nan=True)
        for i, name in ((2, "g"), (3, "s"), (4, "tau_phi"), (5, "tau_mod")):
            np.testing.assert_allclose(sl[i].reshape(12, 12), gold[f"readout_{name}_ch{ch}_h{h}"], rtol=1e-12,
                                       atol=1e-14, equal_nan=True, err_msg=name)


def test_readouts_of_acquisition_histograms():
    acq = FA.FlimAcquisition(FA.flim_config(), 2, n_emitters=50_000, seed=77)
    acq.acquire()
    ptr, nbytes = acq.device_ptr(FA.HIST)
    n_px = 2 * 256 * 256
    out = RD.lifetimes_device(ptr, n_px, 256, 25e-9).cpu().numpy()
    hist = acq.read(FA.HIST)
    _close(out, FO.readouts(hist.reshape(n_px, 256), 25e-9), (n_px,))
    acq.close()


def test_readouts_of_engine_stacks():
    ens = Ensemble(W.ensemble_replicas(2, seed=9, n_min=2000, n_max=3000), precision=32, photons=True, device=0)
    eng = ens.engine
    eng.pipeline_steps(100, True, 100)
    eng.finalize(0)
    torch.cuda.synchronize()
    for r in range(ens.R):
        got = RD.engine_readouts(eng, r, 25e-9, min_counts_mean=1, min_counts_phasor=1)
        ref = FO.readouts(eng.flim(r), 25e-9, min_counts_mean=1, min_counts_phasor=1)
        for k in RD.FIELDS:
            np.testing.assert_allclose(got[k], ref[k], rtol=1e-12, atol=1e-14, equal_nan=True, err_msg=k)
        assert got["intensity"].sum() > 0
