"""Generate tests/golden/h5_layout.json from the reference's own HDF5 writer.

Run where the reference source tree is present, with EDM_REFERENCE_ROOT set to
it (the directory holding ed_mrdt/):

    python tests/golden/make_h5_layout.py

h5py is not installed here, so the in-memory stand-in tests/fake_h5py.py
takes its place under the name h5py before the reference is imported.  The
reference's HDF5Writer (ed_mrdt/io.py:107-485) writes the seeded two-frame
result of tests/h5_case.py; the fixture keeps every dataset's path, shape,
dtype, chunking, compression settings and a digest of its contents.
"""
from __future__ import annotations

import json
import sys
import warnings
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from tests import fake_h5py  # noqa: E402

sys.modules["h5py"] = fake_h5py

from oracle import refshim as RS  # noqa: E402
from tests import h5_case as HC  # noqa: E402


def main():
    warnings.filterwarnings("ignore")
    RS.import_reference()
    from ed_mrdt import io as rio
    from ed_mrdt.microscope import FLIMFrame
    from ed_mrdt.pipeline import FrameResult, GroundTruth
    assert rio.HAS_H5PY and rio.h5py is fake_h5py
    cfg = RS.ref_config_from_dict(HC.raw_config())
    from ed_mrdt.particles import ParticleState
    n = ParticleState(cfg).N
    arrays = HC.frame_arrays(n, len(cfg.species), cfg.scan.pixels_x, cfg.scan.pixels_y, cfg.tcspc.n_bins)
    frames = HC.build_frames(arrays, FLIMFrame, GroundTruth, FrameResult)
    path = "/virtual/reference_layout.h5"
    w = rio.HDF5Writer(path, cfg, n)
    with w:
        for fr in frames:
            w.write_frame(fr)
        w.finalize(**HC.TOTALS)
    layout = fake_h5py.describe(fake_h5py._FILES[path])
    out = Path(__file__).resolve().parent / "h5_layout.json"
    out.write_text(json.dumps({"n_particles": n, "datasets": layout}, indent=1, sort_keys=True) + "\n")
    print(f"{len(layout)} datasets -> {out}")


if __name__ == "__main__":
    main()
