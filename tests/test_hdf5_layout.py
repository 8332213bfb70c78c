"""HDF5 output in the reference's layout (ed_mrdt/io.py:107-485), on CPU.

h5py is not installed here; tests/fake_h5py.py stands in for it.  The golden
fixture tests/golden/h5_layout.json is the layout the reference's own
HDF5Writer produced for the seeded two-frame result of tests/h5_case.py
(tests/golden/make_h5_layout.py): every dataset's path, shape, dtype,
chunking, compression and a digest of its contents.  This package's
HDF5Writer, its streaming (host-thread) variant and write_results must
produce the same, and the readers must read it back.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from tests import fake_h5py
from tests import h5_case as HC

GOLDEN = Path(__file__).resolve().parent / "golden" / "h5_layout.json"


@pytest.fixture()
def h5io(monkeypatch):
    from flim_microscopy_simulator_with_causal_inference_b200 import io as h5io
    monkeypatch.setattr(h5io, "h5py", fake_h5py)
    monkeypatch.setattr(h5io, "HAS_H5PY", True)
    return h5io


def _inputs():
    from flim_microscopy_simulator_with_causal_inference_b200.api import FLIMFrame, FrameResult, GroundTruth
    from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
    from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
    cfg = config_from_dict(HC.raw_config())
    n = ParticleState(cfg).N
    arrays = HC.frame_arrays(n, len(cfg.species), cfg.scan.pixels_x, cfg.scan.pixels_y, cfg.tcspc.n_bins)
    return cfg, n, HC.build_frames(arrays, FLIMFrame, GroundTruth, FrameResult)


@pytest.mark.parametrize("writer", ["plain", "streaming"])
def test_writer_layout_equals_reference_layout(h5io, writer):
    golden = json.loads(GOLDEN.read_text())
    cfg, n, frames = _inputs()
    assert n == golden["n_particles"]
    path = f"/virtual/{writer}.h5"
    cls = h5io.HDF5Writer if writer == "plain" else h5io.StreamingHDF5Writer
    with cls(path, cfg, n) as w:
        for fr in frames:
            w.write_frame(fr)
        w.finalize(**HC.TOTALS)
    got = fake_h5py.describe(fake_h5py._FILES[path])
    assert sorted(got) == sorted(golden["datasets"])
    for k, want in golden["datasets"].items():
        assert got[k] == want, k


def test_write_results_and_readers(h5io):
    from flim_microscopy_simulator_with_causal_inference_b200.api import SimulationResult
    cfg, n, frames = _inputs()
    res = SimulationResult(cfg, frames, total_wall_time_s=HC.TOTALS["total_wall_time"],
                           peak_ram_mb=HC.TOTALS["peak_ram_mb"], total_bindings=HC.TOTALS["total_bindings"],
                           total_dissociations=HC.TOTALS["total_dissociations"])
    path = "/virtual/results.h5"
    h5io.write_results(res, path)
    got = fake_h5py.describe(fake_h5py._FILES[path])
    golden = json.loads(GOLDEN.read_text())["datasets"]
    assert got == golden
    meta = h5io.read_metadata(path)
    assert meta["n_particles"] == n and meta["frames_written"] == len(frames)
    assert meta["species_names"] == [s.name for s in cfg.species]
    assert meta["total_bindings"] == HC.TOTALS["total_bindings"]
    assert np.array_equal(h5io.read_flim_stack(path, 1), frames[1].flim_frame.flim_stack)
    gt = h5io.read_ground_truth_frame(path, 0)
    assert np.array_equal(gt["positions"], frames[0].ground_truth.positions)
    assert gt["n_free_donors"] == frames[0].ground_truth.n_free_donors
    st = h5io.read_statistics(path)
    assert st["photons_emitted"].tolist() == [f.n_photons_emitted for f in frames]
    assert np.allclose(h5io.read_intensity_series(path), [f.flim_frame.intensity.sum() for f in frames])


def test_streaming_writer_reports_thread_errors(h5io):
    cfg, n, frames = _inputs()
    w = h5io.StreamingHDF5Writer("/virtual/err.h5", cfg, n).open()
    bad = frames[0]
    bad.ground_truth.positions = np.zeros((n + 1, 2))  # wrong shape: the thread's write fails
    w.write_frame(bad)
    with pytest.raises(RuntimeError, match="writer thread failed"):
        w.close()


def test_writer_needs_h5py(monkeypatch):
    from flim_microscopy_simulator_with_causal_inference_b200 import io as h5io
    monkeypatch.setattr(h5io, "h5py", None)
    cfg, n, _ = _inputs()
    with pytest.raises(ImportError, match="h5py"):
        h5io.HDF5Writer("/virtual/x.h5", cfg, n)
