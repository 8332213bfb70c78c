"""HDF5 output in the reference's file layout (ed_mrdt/io.py:107-485).

The layout is the interface: a file written here opens with the reference's
readers (read_metadata, read_flim_stack, read_ground_truth_frame) and with any
tool written against ed_mrdt's output.  Groups /metadata, /microscopy,
/ground_truth and /statistics; per-frame datasets of F frames with one frame
per chunk; gzip level 4 on the TCSPC stacks and level 1 on the float
per-particle arrays; the same dataset names, shapes, dtypes and scalar
metadata (ed_mrdt/io.py:12-66 lists them).

h5py does the file I/O; without it the writer raises ImportError, as the
reference's does.  What is new here is `StreamingHDF5Writer`: frames are
handed to a host thread that writes (and gzip-compresses) them while the GPU
simulates the next frame, so the output stays off the per-step path.
`SimulationPipeline.run(h5_path=...)` uses it.
"""
from __future__ import annotations

import queue
import threading
from pathlib import Path
from typing import Optional, Union

import numpy as np
import yaml

try:
    import h5py
    HAS_H5PY = True
except ImportError:  # pragma: no cover - depends on the environment
    h5py = None
    HAS_H5PY = False

__all__ = ["HDF5Writer", "StreamingHDF5Writer", "write_results", "read_metadata", "read_flim_stack",
           "read_ground_truth_frame", "read_intensity_series", "read_statistics"]

_N_CHANNELS = 2  # donor + acceptor (ed_mrdt/io.py:299)


def _need_h5py():
    if h5py is None:
        raise ImportError("h5py is required for HDF5 output. Install with: pip install h5py")


def config_to_dict(cfg) -> dict:
    """The configuration fields the reference serialises into
    /metadata/config_yaml (ed_mrdt/io.py:233-287), in its key order."""
    s, la, det = cfg.scan, cfg.laser, cfg.detector
    return {
        "name": cfg.name,
        "version": cfg.version,
        "membrane": {"size": list(cfg.membrane.size), "periodic": list(cfg.membrane.periodic),
                     "geometry_type": cfg.membrane.geometry_type},
        "simulation_time": cfg.simulation_time,
        "bd_timestep": cfg.bd_timestep,
        "random_seed": cfg.random_seed,
        "n_threads": cfg.n_threads,
        "ram_limit_gb": cfg.ram_limit_gb,
        "initial_populations": dict(cfg.initial_populations),
        "scan": {"mode": s.mode, "pixel_size": s.pixel_size, "pixels_x": s.pixels_x, "pixels_y": s.pixels_y,
                 "dwell_time": s.dwell_time, "n_frames": s.n_frames, "frame_interval": s.frame_interval},
        "tcspc": {"n_bins": cfg.tcspc.n_bins, "time_range": cfg.tcspc.time_range},
        "laser": {"wavelength": la.wavelength, "repetition_rate": la.repetition_rate, "power": la.power},
        "detector": {"type": det.type, "detection_efficiency": det.detection_efficiency,
                     "dark_count_rate": det.dark_count_rate},
    }


class HDF5Writer:
    """Frame-by-frame writer of one simulation (the reference's HDF5Writer
    interface: open / write_frame / finalize / close, usable as a context
    manager)."""

    def __init__(self, path: Union[str, Path], config, n_particles: int, compression: Optional[str] = "gzip",
                 compression_level: int = 4):
        _need_h5py()
        self.path = Path(path)
        self.config = config
        self.n_particles = int(n_particles)
        self.compression = compression
        self.compression_level = compression_level
        self._file = None
        self._frame_idx = 0
        self._is_open = False

    # ---- open / close ----------------------------------------------------
    def open(self) -> "HDF5Writer":
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self._file = h5py.File(str(self.path), "w")
        self._is_open = True
        self._write_metadata()
        self._create_datasets()
        return self

    def close(self) -> None:
        if self._file is not None:
            self._file.close()
            self._file = None
        self._is_open = False

    def __enter__(self) -> "HDF5Writer":
        return self.open()

    def __exit__(self, *args) -> None:
        self.close()

    @property
    def frames_written(self) -> int:
        return self._frame_idx

    # ---- layout ----------------------------------------------------------
    def _write_metadata(self) -> None:
        cfg = self.config
        meta = self._file.create_group("metadata")
        text = h5py.string_dtype()
        meta.create_dataset("config_yaml", data=yaml.dump(config_to_dict(cfg), default_flow_style=False,
                                                          allow_unicode=True), dtype=text)
        meta.create_dataset("random_seed", data=cfg.random_seed)
        meta.create_dataset("version", data=cfg.version, dtype=text)
        meta.create_dataset("sim_name", data=cfg.name, dtype=text)
        meta.create_dataset("n_particles", data=self.n_particles)
        meta.create_dataset("n_frames", data=cfg.scan.n_frames)
        meta.create_dataset("bd_timestep", data=cfg.bd_timestep)
        meta.create_dataset("frame_interval", data=cfg.scan.frame_interval)
        meta.create_dataset("membrane_size", data=np.array(cfg.membrane.size, dtype=np.float64))
        for key, names in (("species_names", [s.name for s in cfg.species]),
                           ("fluorophore_names", [f.name for f in cfg.fluorophores])):
            ds = meta.create_dataset(key, shape=(len(names),), dtype=text)
            for i, name in enumerate(names):
                ds[i] = name

    def _create_datasets(self) -> None:
        f = self._file
        cfg = self.config
        F, N, C = cfg.scan.n_frames, self.n_particles, _N_CHANNELS
        px, py, nb = cfg.scan.pixels_x, cfg.scan.pixels_y, cfg.tcspc.n_bins
        heavy = dict(compression=self.compression, compression_opts=self.compression_level) if self.compression else {}
        light = dict(compression=self.compression, compression_opts=1) if self.compression else {}
        mic = f.create_group("microscopy")
        mic.create_dataset("flim_stack", shape=(F, C, px, py, nb), dtype=np.uint32, chunks=(1, C, px, py, nb),
                           **heavy)
        mic.create_dataset("intensity", shape=(F, C, px, py), dtype=np.float64, chunks=(1, C, px, py), **light)
        mic.create_dataset("bio_time", shape=(F,), dtype=np.float64)
        for k in ("n_signal_photons", "n_dark_counts", "n_afterpulses"):
            mic.create_dataset(k, shape=(F,), dtype=np.int32)
        gt = f.create_group("ground_truth")
        gt.create_dataset("positions", shape=(F, N, 2), dtype=np.float64, chunks=(1, N, 2), **light)
        for k, dt in (("species_id", np.int32), ("bond_partner", np.int32), ("is_alive", np.bool_),
                      ("has_dye", np.bool_), ("dye_type_id", np.int32), ("is_bleached", np.bool_)):
            gt.create_dataset(k, shape=(F, N), dtype=dt, chunks=(1, N))
        for k in ("fret_efficiency", "donor_lifetime"):
            gt.create_dataset(k, shape=(F, N), dtype=np.float64, chunks=(1, N), **light)
        for k in ("n_complexes", "n_bleached", "n_free_donors"):
            gt.create_dataset(k, shape=(F,), dtype=np.int32)
        stats = f.create_group("statistics")
        stats.create_dataset("photons_emitted", shape=(F,), dtype=np.int64)
        stats.create_dataset("photons_detected", shape=(F,), dtype=np.int64)
        stats.create_dataset("wall_time_per_frame", shape=(F,), dtype=np.float64)
        stats.create_dataset("total_wall_time", data=0.0)
        stats.create_dataset("peak_ram_mb", data=0.0)
        stats.create_dataset("total_bindings", data=np.int64(0))
        stats.create_dataset("total_dissociations", data=np.int64(0))

    # ---- frames ------------------------------------------------------------
    def write_frame(self, frame) -> None:
        """Write one FrameResult at the next frame index and flush."""
        if not self._is_open:
            raise RuntimeError("HDF5Writer is not open. Call open() first.")
        i, f = self._frame_idx, self._file
        fl, gt = frame.flim_frame, frame.ground_truth
        for path, value in (("microscopy/flim_stack", fl.flim_stack), ("microscopy/intensity", fl.intensity),
                            ("microscopy/bio_time", frame.bio_time),
                            ("microscopy/n_signal_photons", fl.n_signal_photons),
                            ("microscopy/n_dark_counts", fl.n_dark_counts),
                            ("microscopy/n_afterpulses", fl.n_afterpulses),
                            ("ground_truth/positions", gt.positions), ("ground_truth/species_id", gt.species_id),
                            ("ground_truth/bond_partner", gt.bond_partner), ("ground_truth/is_alive", gt.is_alive),
                            ("ground_truth/has_dye", gt.has_dye), ("ground_truth/dye_type_id", gt.dye_type_id),
                            ("ground_truth/is_bleached", gt.is_bleached),
                            ("ground_truth/fret_efficiency", gt.fret_efficiency_exact),
                            ("ground_truth/donor_lifetime", gt.donor_lifetime_exact),
                            ("ground_truth/n_complexes", gt.n_complexes), ("ground_truth/n_bleached", gt.n_bleached),
                            ("ground_truth/n_free_donors", gt.n_free_donors),
                            ("statistics/photons_emitted", frame.n_photons_emitted),
                            ("statistics/photons_detected", frame.n_photons_detected),
                            ("statistics/wall_time_per_frame", frame.wall_time_s)):
            f[path][i] = value
        f.flush()
        self._frame_idx += 1

    def finalize(self, total_wall_time: float = 0.0, peak_ram_mb: float = 0.0, total_bindings: int = 0,
                 total_dissociations: int = 0) -> None:
        """Summary statistics and the number of frames written."""
        if not self._is_open:
            return
        f = self._file
        f["statistics/total_wall_time"][()] = total_wall_time
        f["statistics/peak_ram_mb"][()] = peak_ram_mb
        f["statistics/total_bindings"][()] = np.int64(total_bindings)
        f["statistics/total_dissociations"][()] = np.int64(total_dissociations)
        if "frames_written" not in f["metadata"]:
            f["metadata"].create_dataset("frames_written", data=self._frame_idx)
        else:
            f["metadata/frames_written"][()] = self._frame_idx
        f.flush()


class StreamingHDF5Writer:
    """HDF5Writer on a host thread.  write_frame() queues the frame (at most
    `depth` frames wait; the caller blocks beyond that) and returns at once;
    the thread writes and compresses while the caller goes on.  The frame's
    arrays must not be modified after they are queued (the pipeline hands
    over fresh copies).  An error on the thread is raised by the next call."""

    def __init__(self, path: Union[str, Path], config, n_particles: int, compression: Optional[str] = "gzip",
                 compression_level: int = 4, depth: int = 2):
        self.writer = HDF5Writer(path, config, n_particles, compression, compression_level)
        self._q: queue.Queue = queue.Queue(maxsize=max(1, depth))
        self._err: Optional[BaseException] = None
        self._thread: Optional[threading.Thread] = None

    def _run(self):
        while True:
            item = self._q.get()
            try:
                if item is None:
                    return
                kind, payload = item
                if self._err is None:
                    if kind == "frame":
                        self.writer.write_frame(payload)
                    else:
                        self.writer.finalize(**payload)
            except BaseException as ex:  # noqa: BLE001 - reported to the caller
                self._err = ex
            finally:
                self._q.task_done()

    def _raise(self):
        if self._err is not None:
            err, self._err = self._err, None
            raise RuntimeError(f"HDF5 writer thread failed: {err}") from err

    def open(self) -> "StreamingHDF5Writer":
        self.writer.open()
        self._thread = threading.Thread(target=self._run, name="edm-hdf5-writer", daemon=True)
        self._thread.start()
        return self

    def write_frame(self, frame) -> None:
        self._raise()
        self._q.put(("frame", frame))

    def finalize(self, **totals) -> None:
        self._raise()
        self._q.put(("finalize", totals))

    def close(self) -> None:
        if self._thread is not None:
            self._q.put(None)
            self._thread.join()
            self._thread = None
        self.writer.close()
        self._raise()

    @property
    def frames_written(self) -> int:
        self._q.join()
        return self.writer.frames_written

    def __enter__(self) -> "StreamingHDF5Writer":
        return self.open()

    def __exit__(self, *args) -> None:
        self.close()


def write_results(result, path: Union[str, Path], compression: Optional[str] = "gzip",
                  compression_level: int = 4) -> Path:
    """Write a complete SimulationResult (ed_mrdt/io.py:492-541)."""
    if not result.frames:
        raise ValueError("SimulationResult has no frames to write")
    n = result.frames[0].ground_truth.positions.shape[0]
    path = Path(path)
    with HDF5Writer(path, result.config, n, compression=compression, compression_level=compression_level) as w:
        for frame in result.frames:
            w.write_frame(frame)
        w.finalize(total_wall_time=result.total_wall_time_s, peak_ram_mb=result.peak_ram_mb,
                   total_bindings=result.total_bindings, total_dissociations=result.total_dissociations)
    return path


def _text(v) -> str:
    return v.decode() if isinstance(v, bytes) else str(v)


def read_metadata(path: Union[str, Path]) -> dict:
    """Metadata and summary statistics of a file (ed_mrdt/io.py:548-586)."""
    _need_h5py()
    info = {}
    with h5py.File(str(path), "r") as f:
        m = f["metadata"]
        info["config_yaml"] = _text(m["config_yaml"][()])
        info["random_seed"] = int(m["random_seed"][()])
        info["version"] = _text(m["version"][()])
        info["sim_name"] = _text(m["sim_name"][()])
        info["n_particles"] = int(m["n_particles"][()])
        info["n_frames"] = int(m["n_frames"][()])
        info["bd_timestep"] = float(m["bd_timestep"][()])
        info["frame_interval"] = float(m["frame_interval"][()])
        info["membrane_size"] = np.asarray(m["membrane_size"][()]).tolist()
        info["species_names"] = [_text(s) for s in m["species_names"][()]]
        info["fluorophore_names"] = [_text(s) for s in m["fluorophore_names"][()]]
        if "frames_written" in m:
            info["frames_written"] = int(m["frames_written"][()])
        if "statistics" in f:
            s = f["statistics"]
            info["total_wall_time"] = float(s["total_wall_time"][()])
            info["peak_ram_mb"] = float(s["peak_ram_mb"][()])
            info["total_bindings"] = int(s["total_bindings"][()])
            info["total_dissociations"] = int(s["total_dissociations"][()])
    return info


def read_flim_stack(path: Union[str, Path], frame_idx: int) -> np.ndarray:
    """TCSPC stack [C, Px, Py, Tb] of one frame."""
    _need_h5py()
    with h5py.File(str(path), "r") as f:
        return np.asarray(f["microscopy/flim_stack"][frame_idx])


def read_ground_truth_frame(path: Union[str, Path], frame_idx: int) -> dict:
    """Per-particle ground truth and counts of one frame."""
    _need_h5py()
    with h5py.File(str(path), "r") as f:
        g = f["ground_truth"]
        out = {k: np.asarray(g[k][frame_idx]) for k in ("positions", "species_id", "bond_partner", "is_alive",
                                                         "has_dye", "dye_type_id", "is_bleached",
                                                         "fret_efficiency", "donor_lifetime")}
        for k in ("n_complexes", "n_bleached", "n_free_donors"):
            out[k] = int(g[k][frame_idx])
    return out


def read_intensity_series(path: Union[str, Path]) -> np.ndarray:
    """Total counts per frame (sum of the intensity images over channels and pixels)."""
    _need_h5py()
    with h5py.File(str(path), "r") as f:
        return np.asarray(f["microscopy/intensity"][()]).sum(axis=(1, 2, 3))


def read_statistics(path: Union[str, Path]) -> dict:
    """Per-frame photon counts and wall times, and the run totals."""
    _need_h5py()
    with h5py.File(str(path), "r") as f:
        g = f["statistics"]
        out = {k: np.array(g[k][()]) for k in ("photons_emitted", "photons_detected", "wall_time_per_frame")}
        out["total_wall_time"] = float(g["total_wall_time"][()])
        out["peak_ram_mb"] = float(g["peak_ram_mb"][()])
        out["total_bindings"] = int(g["total_bindings"][()])
        out["total_dissociations"] = int(g["total_dissociations"][()])
    return out
