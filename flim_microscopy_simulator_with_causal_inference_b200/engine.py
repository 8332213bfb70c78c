"""ctypes binding of the C ABI (include/edm_b200.h) and the device system.

`Engine` is a thin, typed wrapper over one `EdmEngine*`: R replicas of the
per-timestep path on one GPU.  `DeviceSystem` binds an Engine to one host
`ParticleState` and implements the reference API's in-place semantics: the
host arrays are uploaded before a device call when they differ from what the
device last saw, and downloaded after calls that must leave them current.

There is no CPU fallback: if the CUDA library is missing or no GPU is
visible, constructing an Engine raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

from . import params as PR

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libedm_b200.so"

_lib = None


def build_library(force: bool = False) -> Path:
    """Compile the CUDA library in-tree with nvcc (sm_100a)."""
    csrc = PKG / "csrc"
    deps = list(csrc.glob("*.cu")) + list(csrc.glob("*.cuh")) + [PKG.parent / "include" / "edm_b200.h"]
    if force or not LIB_PATH.exists() or any(d.stat().st_mtime > LIB_PATH.stat().st_mtime for d in deps):
        subprocess.run(["make", "-C", str(csrc)], check=True)
    return LIB_PATH


def load_library():
    """Load the CUDA engine library (fails loudly when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"CUDA engine library not built: {LIB_PATH} (run __graft_entry__.build())")
    L = C.CDLL(str(LIB_PATH))
    vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
    L.edm_abi_version.restype = C.c_int
    L.edm_abi_sizeof.argtypes = [C.c_int]
    L.edm_abi_sizeof.restype = i64
    L.edm_last_error.restype = C.c_char_p
    L.edm_create.argtypes = [vp, vp, vp, i32, vp, i64, i32, i32, C.POINTER(vp)]
    L.edm_destroy.argtypes = [vp]
    L.edm_set_state.argtypes = [vp, vp, vp]
    L.edm_get_state.argtypes = [vp, vp, vp]
    L.edm_set_step.argtypes = [vp, i64]
    L.edm_get_step.argtypes = [vp]
    L.edm_get_step.restype = i64
    L.edm_dynamics_step.argtypes = [vp, i32, vp]
    L.edm_photon_step.argtypes = [vp, vp]
    L.edm_get_photon_counts.argtypes = [vp, vp, vp]
    L.edm_get_photons.argtypes = [vp, i32, vp, vp, vp, vp, i64, vp]
    L.edm_scope_process.argtypes = [vp, vp]
    L.edm_set_photons.argtypes = [vp, i32, vp, vp, vp, vp, i64, i64, vp]
    L.edm_pipeline_steps.argtypes = [vp, i32, i32, i32, vp]
    L.edm_scope_finalize.argtypes = [vp, i64, vp]
    L.edm_get_flim.argtypes = [vp, i32, vp, i64, vp]
    L.edm_reset_flim.argtypes = [vp, vp]
    L.edm_get_counters.argtypes = [vp, vp, vp]
    L.edm_get_status.argtypes = [vp, vp, vp]
    L.edm_get_cells.argtypes = [vp, i32, vp, vp, i64, i64, vp]
    L.edm_profile_steps.argtypes = [vp, i32, i32, vp, vp]
    L.edm_profile_passes.argtypes = [vp, i32, vp, vp, i32, vp]
    L.edm_launches_per_step.argtypes = [vp, i32]
    L.edm_autotune.argtypes = [vp, i32, i32, vp]
    L.edm_launch_shapes.argtypes = [vp, vp, vp]
    L.edm_contact_sides.argtypes = [vp, i32]
    L.edm_set_state_async.argtypes = [vp, vp, vp]
    L.edm_get_state_async.argtypes = [vp, vp, vp]
    L.edm_state_transfers_wait.argtypes = [vp]
    L.edm_stage_state_async.argtypes = [vp, vp]
    L.edm_install_state.argtypes = [vp, vp]
    L.edm_set_launch_shapes.argtypes = [vp, vp]
    L.edm_record_enable.argtypes = [vp, i32]
    L.edm_record_read.argtypes = [vp, i64, i32, vp, vp]
    L.edm_ground_truth.argtypes = [vp, vp, vp, vp, vp]
    L.edm_cell_list_static.argtypes = [vp, i64, C.c_double, C.c_double, i32, i32, vp, vp, vp]
    L.edm_readout_lifetimes.argtypes = [vp, i64, i32, C.c_double, i32, i32, i32, vp, vp]
    L.edm_flim_stack_ptr.argtypes = [vp, i32, C.POINTER(vp), C.POINTER(i64), C.POINTER(i32)]
    L.edm_flim_elems.argtypes = [vp]
    L.edm_flim_elems.restype = i64
    L.edm_frame_out_begin.argtypes = [vp, vp, i64, vp]
    L.edm_frame_out_wait.argtypes = [vp]
    L.edm_frame_out_sparse.argtypes = [vp, vp, vp, i64, vp]
    L.edm_frame_out_sparse.restype = i64
    L.edm_flim_create.argtypes = [vp, i32, C.POINTER(vp)]
    L.edm_flim_destroy.argtypes = [vp]
    L.edm_flim_set_inputs.argtypes = [vp, vp, u64, vp]
    L.edm_flim_project.argtypes = [vp, vp]
    L.edm_flim_histograms.argtypes = [vp, i32, vp]
    L.edm_flim_acquire.argtypes = [vp, vp]
    L.edm_flim_device_ptr.argtypes = [vp, i32, C.POINTER(vp), C.POINTER(i64)]
    L.edm_flim_read.argtypes = [vp, i32, i32, vp, i64, vp]
    L.edm_flim_read_hist_narrow.argtypes = [vp, i32, i32, vp, i64, vp]
    L.edm_flim_read_hist_narrow_async.argtypes = [vp, i32, vp, i64, vp]
    L.edm_flim_read_wait.argtypes = [vp]
    L.edm_flim_get_error.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.edm_noise_normal_pairs.argtypes = [u64, i64, i32, vp, i64, vp, vp]
    L.edm_noise_uniforms.argtypes = [u64, i64, i32, vp, vp, i64, vp, vp]
    for which, cls in ((0, PR.EdmDynParams), (1, PR.EdmPhotParams), (2, PR.EdmScopeParams), (3, PR.EdmHostState),
                       (4, PR.EdmFlimParams)):
        if L.edm_abi_sizeof(which) != C.sizeof(cls):
            raise ImportError(f"ABI mismatch for {cls.__name__}: C {L.edm_abi_sizeof(which)} vs ctypes {C.sizeof(cls)}")
    _lib = L
    return L


def _check(rc: int, what: str) -> int:
    if rc < 0:
        msg = load_library().edm_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")
    return rc


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream))


class Engine:
    """R replicas of the per-timestep path on one GPU (one EdmEngine*)."""

    def __init__(self, dyn: Sequence[PR.EdmDynParams], hill: np.ndarray,
                 phot: Optional[Sequence[PR.EdmPhotParams]] = None,
                 scope: Optional[Sequence[PR.EdmScopeParams]] = None, precision: int = 64, device: int = 0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device visible: the B200 engine has no CPU fallback")
        self.L = load_library()
        self.R = len(dyn)
        self.precision = int(precision)
        self._dyn = (PR.EdmDynParams * self.R)(*dyn)
        self._phot = (PR.EdmPhotParams * self.R)(*phot) if phot is not None else None
        self._scope = (PR.EdmScopeParams * self.R)(*scope) if scope is not None else None
        self._hill = np.ascontiguousarray(hill, dtype=np.float64)
        self.N = int(sum(p.n_particles for p in dyn))
        self.handle = C.c_void_p()
        _check(self.L.edm_create(C.byref(self._dyn), C.byref(self._phot) if self._phot is not None else None,
                                 C.byref(self._scope) if self._scope is not None else None, self.R,
                                 _ptr(self._hill), self._hill.size, self.precision, device,
                                 C.byref(self.handle)), "edm_create")

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.L.edm_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state ---------------------------------------------------------------
    def set_state(self, positions, species, alive, bond, has_dye, dye_type, ctmc, bleached, stream=None):
        arrs = dict(positions=np.ascontiguousarray(positions, dtype=np.float64),
                    species=np.ascontiguousarray(species, dtype=np.int32),
                    alive=np.ascontiguousarray(alive, dtype=np.uint8),
                    bond=np.ascontiguousarray(bond, dtype=np.int32),
                    has_dye=np.ascontiguousarray(has_dye, dtype=np.uint8),
                    dye=np.ascontiguousarray(dye_type, dtype=np.int32),
                    ctmc=np.ascontiguousarray(ctmc, dtype=np.int8),
                    bleached=np.ascontiguousarray(bleached, dtype=np.uint8))
        hs = PR.EdmHostState(self.N, _ptr(arrs["positions"]), _ptr(arrs["species"]), _ptr(arrs["alive"]),
                             _ptr(arrs["bond"]), _ptr(arrs["has_dye"]), _ptr(arrs["dye"]), _ptr(arrs["ctmc"]),
                             _ptr(arrs["bleached"]))
        _check(self.L.edm_set_state(self.handle, C.byref(hs), _stream_handle(stream)), "edm_set_state")

    STATE_FIELDS = (("positions", np.float64, 2), ("species", np.int32, 1), ("alive", np.uint8, 1),
                    ("bond", np.int32, 1), ("ctmc", np.int8, 1), ("bleached", np.uint8, 1),
                    ("has_dye", np.uint8, 1))

    def get_state(self, stream=None, out: Optional[dict] = None) -> dict:
        """The particle state in id order.  `out` may hold preallocated
        (e.g. pinned) arrays of STATE_FIELDS' dtypes and shapes to fill."""
        N = self.N
        if out is None:
            out = {k: np.empty((N, w) if w > 1 else N, dtype=dt) for k, dt, w in self.STATE_FIELDS}
        for k, dt, w in self.STATE_FIELDS:
            a = out[k]
            if a.dtype != dt or a.shape != ((N, w) if w > 1 else (N,)) or not a.flags.c_contiguous:
                raise ValueError(f"get_state: out['{k}'] must be a contiguous {np.dtype(dt).name} array of N rows")
        hs = PR.EdmHostState(N, _ptr(out["positions"]), _ptr(out["species"]), _ptr(out["alive"]), _ptr(out["bond"]),
                             _ptr(out["has_dye"]), None, _ptr(out["ctmc"]), _ptr(out["bleached"]))
        _check(self.L.edm_get_state(self.handle, C.byref(hs), _stream_handle(stream)), "edm_get_state")
        return out

    # ---- transfers overlapped with computation ------------------------------
    SET_FIELDS = (("positions", np.float64, 2), ("species", np.int32, 1), ("alive", np.uint8, 1),
                  ("bond", np.int32, 1), ("has_dye", np.uint8, 1), ("dye", np.int32, 1), ("ctmc", np.int8, 1),
                  ("bleached", np.uint8, 1))

    def _require(self, arrs: dict, fields, what: str):
        N = self.N
        for k, dt, w in fields:
            a = arrs[k]
            if a.dtype != dt or a.shape != ((N, w) if w > 1 else (N,)) or not a.flags.c_contiguous:
                raise ValueError(f"{what}: '{k}' must be a contiguous {np.dtype(dt).name} array of N rows")

    def set_state_async(self, arrs: dict, stream=None):
        """edm_set_state_async: the host arrays (SET_FIELDS' dtypes, pinned)
        go up on the engine's upload stream while `stream` computes; they
        must stay unchanged until transfers_wait()."""
        self._require(arrs, self.SET_FIELDS, "set_state_async")
        hs = PR.EdmHostState(self.N, _ptr(arrs["positions"]), _ptr(arrs["species"]), _ptr(arrs["alive"]),
                             _ptr(arrs["bond"]), _ptr(arrs["has_dye"]), _ptr(arrs["dye"]), _ptr(arrs["ctmc"]),
                             _ptr(arrs["bleached"]))
        self._xfer_refs = getattr(self, "_xfer_refs", []) + [arrs]
        _check(self.L.edm_set_state_async(self.handle, C.byref(hs), _stream_handle(stream)), "edm_set_state_async")

    def stage_state_async(self, arrs: dict):
        """edm_stage_state_async: the upload half of set_state_async (the
        arrays go up on the engine's upload stream); install_state() puts the
        staged state in place on a stream."""
        self._require(arrs, self.SET_FIELDS, "stage_state_async")
        hs = PR.EdmHostState(self.N, _ptr(arrs["positions"]), _ptr(arrs["species"]), _ptr(arrs["alive"]),
                             _ptr(arrs["bond"]), _ptr(arrs["has_dye"]), _ptr(arrs["dye"]), _ptr(arrs["ctmc"]),
                             _ptr(arrs["bleached"]))
        self._xfer_refs = getattr(self, "_xfer_refs", []) + [arrs]
        _check(self.L.edm_stage_state_async(self.handle, C.byref(hs)), "edm_stage_state_async")

    def install_state(self, stream=None):
        """edm_install_state: the staged state, in order on `stream`."""
        _check(self.L.edm_install_state(self.handle, _stream_handle(stream)), "edm_install_state")

    def get_state_async(self, out: dict, stream=None) -> dict:
        """edm_get_state_async: the state (STATE_FIELDS) comes down on the
        engine's download stream while `stream` goes on; read `out` after
        transfers_wait()."""
        self._require(out, self.STATE_FIELDS, "get_state_async")
        hs = PR.EdmHostState(self.N, _ptr(out["positions"]), _ptr(out["species"]), _ptr(out["alive"]),
                             _ptr(out["bond"]), _ptr(out["has_dye"]), None, _ptr(out["ctmc"]), _ptr(out["bleached"]))
        self._xfer_refs = getattr(self, "_xfer_refs", []) + [out]
        _check(self.L.edm_get_state_async(self.handle, C.byref(hs), _stream_handle(stream)), "edm_get_state_async")
        return out

    def transfers_wait(self):
        """Wait for the asynchronous state transfers (edm_state_transfers_wait)."""
        _check(self.L.edm_state_transfers_wait(self.handle), "edm_state_transfers_wait")
        self._xfer_refs = []

    def set_step(self, k: int):
        _check(self.L.edm_set_step(self.handle, int(k)), "edm_set_step")

    def get_step(self) -> int:
        return int(self.L.edm_get_step(self.handle))

    # ---- stepping ------------------------------------------------------------
    def dynamics_step(self, n: int = 1, stream=None):
        _check(self.L.edm_dynamics_step(self.handle, int(n), _stream_handle(stream)), "edm_dynamics_step")

    def photon_step(self, stream=None):
        _check(self.L.edm_photon_step(self.handle, _stream_handle(stream)), "edm_photon_step")

    def scope_process(self, stream=None):
        _check(self.L.edm_scope_process(self.handle, _stream_handle(stream)), "edm_scope_process")

    def pipeline_steps(self, n: int, with_photons: bool = True, graph_chunk: int = 0, stream=None):
        _check(self.L.edm_pipeline_steps(self.handle, int(n), int(bool(with_photons)), int(graph_chunk),
                                         _stream_handle(stream)), "edm_pipeline_steps")

    def set_photons(self, replica: int, particle_idx, arrival_time, channel, is_fret, batch_key: int, stream=None):
        pid = np.ascontiguousarray(particle_idx, dtype=np.int32)
        t = np.ascontiguousarray(arrival_time, dtype=np.float64)
        ch = np.ascontiguousarray(channel, dtype=np.int8)
        fr = np.ascontiguousarray(is_fret, dtype=np.uint8)
        _check(self.L.edm_set_photons(self.handle, replica, _ptr(pid), _ptr(t), _ptr(ch), _ptr(fr), pid.size,
                                      int(batch_key), _stream_handle(stream)), "edm_set_photons")

    PROFILE_GROUPS = ("cell_scan", "scatter", "move", "reactions", "photophysics", "detection", "step")

    def profile_steps(self, n: int, with_photons: bool = True, stream=None) -> dict:
        """Mean device ms per step of each kernel group (CUDA events, eager)."""
        out = np.zeros(7, dtype=np.float32)
        _check(self.L.edm_profile_steps(self.handle, int(n), int(bool(with_photons)), _ptr(out),
                                        _stream_handle(stream)), "edm_profile_steps")
        return dict(zip(self.PROFILE_GROUPS, out.astype(float).tolist()))

    PASS_KINDS = ("bind_candidates", "bind_apply", "dissociation", "contacts", "catalytic", "recruit_candidates",
                  "recruit_apply", "detach", "convert", "grid_merge", "particle_passes", "pass_draws",
                  "adaptation", "local_cdf")

    def profile_passes(self, n: int, stream=None) -> list:
        """Mean device ms per dynamics step of each reaction pass, in schedule
        order: [(kind, index, ms)] (CUDA events, eager, dynamics only)."""
        cap = 256
        out = np.zeros(cap, dtype=np.float32)
        kinds = np.zeros(cap, dtype=np.int32)
        n_pass = _check(self.L.edm_profile_passes(self.handle, int(n), _ptr(out), _ptr(kinds), cap,
                                                  _stream_handle(stream)), "edm_profile_passes")
        return [(self.PASS_KINDS[kinds[k] // 100], int(kinds[k] % 100), float(out[k])) for k in range(n_pass)]

    # ---- launch-shape autotuner ---------------------------------------------
    TUNED_KERNELS = ("k_scatter", "k_move", "k_contacts")

    def autotune(self, steps_per_shape: int = 3, retune: bool = False, stream=None) -> dict:
        """Time every candidate launch shape of the tuned kernels on real
        dynamics steps and keep the fastest (edm_autotune); returns
        launch_shapes()."""
        _check(self.L.edm_autotune(self.handle, int(steps_per_shape), int(bool(retune)), _stream_handle(stream)),
               "edm_autotune")
        return self.launch_shapes()

    def launch_shapes(self) -> dict:
        """{kernel: {block, min_blocks_per_sm, candidates, default_ms, tuned_ms}}."""
        shp = np.zeros((3, 4), dtype=np.int32)
        ms = np.zeros((3, 2), dtype=np.float32)
        n = _check(self.L.edm_launch_shapes(self.handle, _ptr(shp), _ptr(ms)), "edm_launch_shapes")
        return {self.TUNED_KERNELS[k]: {"block": int(shp[k, 0]), "min_blocks_per_sm": int(shp[k, 1]),
                                        "candidates": int(shp[k, 2]), "candidate": int(shp[k, 3]),
                                        "default_ms": float(ms[k, 0]),
                                        "tuned_ms": float(ms[k, 1])} for k in range(n)}

    def set_launch_shapes(self, candidates: Sequence[int]) -> dict:
        """Sets each tuned kernel's launch shape (edm_set_launch_shapes):
        candidates[k] for TUNED_KERNELS[k], -1 keeps it; returns
        launch_shapes()."""
        c = np.full(len(self.TUNED_KERNELS), -1, dtype=np.int32)
        c[: len(candidates)] = np.asarray(candidates, dtype=np.int32)
        _check(self.L.edm_set_launch_shapes(self.handle, _ptr(c)), "edm_set_launch_shapes")
        return self.launch_shapes()

    def contact_sides(self, force_mask: Optional[int] = None) -> int:
        """Sides of the catalytic contact sweep (edm_contact_sides): bit c set
        = reaction c swept from its enzyme species, clear = from its substrate
        species.  force_mask sets them; returns the mask in use."""
        return _check(self.L.edm_contact_sides(self.handle, -1 if force_mask is None else int(force_mask)),
                      "edm_contact_sides")

    # ---- census: sub-frame recorder and per-frame ground truth --------------
    def record_enable(self, capacity_steps: int) -> None:
        """Record every later pipeline step's census rows into a device ring
        of `capacity_steps` steps (0 stops recording)."""
        _check(self.L.edm_record_enable(self.handle, int(capacity_steps)), "edm_record_enable")

    def record_read(self, first_step: int, n_steps: int, stream=None, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Census rows [n_steps][R][CENSUS_FIELDS] of steps first_step .. +n_steps."""
        shape = (int(n_steps), self.R, PR.CENSUS_FIELDS)
        if out is None:
            out = np.empty(shape, dtype=np.int64)
        elif out.shape != shape or out.dtype != np.int64 or not out.flags.c_contiguous:
            raise ValueError(f"record_read: out must be a contiguous int64 array of shape {shape}")
        _check(self.L.edm_record_read(self.handle, int(first_step), int(n_steps), _ptr(out), _stream_handle(stream)),
               "edm_record_read")
        self._sync(stream)
        return out

    def ground_truth(self, stream=None):
        """(fret_E[N], tau_DA[N], census[R][CENSUS_FIELDS]) of the current state."""
        e = np.empty(self.N, dtype=np.float64)
        tau = np.empty(self.N, dtype=np.float64)
        cen = np.empty((self.R, PR.CENSUS_FIELDS), dtype=np.int64)
        _check(self.L.edm_ground_truth(self.handle, _ptr(e), _ptr(tau), _ptr(cen), _stream_handle(stream)),
               "edm_ground_truth")
        self._sync(stream)
        return e, tau, cen

    @staticmethod
    def _sync(stream):
        import torch
        if stream is None:
            torch.cuda.synchronize()
        elif hasattr(stream, "synchronize"):
            stream.synchronize()
        else:
            torch.cuda.ExternalStream(int(stream)).synchronize()

    def launches_per_step(self, with_photons: bool = True) -> int:
        return _check(self.L.edm_launches_per_step(self.handle, int(bool(with_photons))), "edm_launches_per_step")

    def flim_elems(self) -> int:
        """uint32 elements of all replicas' FLIM stacks (edm_flim_elems)."""
        return int(self.L.edm_flim_elems(self.handle))

    def frame_out_begin(self, host_out: np.ndarray, stream=None) -> None:
        """Snapshot and clear the finalized stacks on `stream`, then read the
        snapshot into `host_out` (pinned uint32, flim_elems() long) on the
        engine's copy stream, overlapping what `stream` does next."""
        if host_out.dtype != np.uint32 or not host_out.flags.c_contiguous:
            raise ValueError("host_out must be a contiguous uint32 array")
        _check(self.L.edm_frame_out_begin(self.handle, _ptr(host_out), host_out.size, _stream_handle(stream)),
               "edm_frame_out_begin")

    def frame_out_sparse(self, idx_out: np.ndarray, count_out: np.ndarray, stream=None) -> int:
        """Every replica's finalized stacks as nonzero bins (element index into
        the concatenated stacks, count) written into idx_out (int64) and
        count_out (uint32), both of capacity len(idx_out); the emitted bins
        are cleared.  Returns the number of nonzero bins."""
        if idx_out.dtype != np.int64 or count_out.dtype != np.uint32 or idx_out.size != count_out.size:
            raise ValueError("idx_out must be int64 and count_out uint32 of the same length")
        n = self.L.edm_frame_out_sparse(self.handle, _ptr(idx_out), _ptr(count_out), idx_out.size,
                                        _stream_handle(stream))
        return _check(int(n), "edm_frame_out_sparse")

    @staticmethod
    def sparse_to_dense(idx: np.ndarray, count: np.ndarray, n: int, n_elems: int) -> np.ndarray:
        """The dense concatenated stacks (uint32, n_elems long) of a sparse readout of n bins."""
        out = np.zeros(n_elems, dtype=np.uint32)
        out[idx[:n]] = count[:n]
        return out

    def frame_out_wait(self) -> None:
        """Block until the last frame_out_begin read has landed in host memory."""
        _check(self.L.edm_frame_out_wait(self.handle), "edm_frame_out_wait")

    def finalize(self, frame_index: int, stream=None):
        _check(self.L.edm_scope_finalize(self.handle, int(frame_index), _stream_handle(stream)), "edm_scope_finalize")

    # ---- outputs -------------------------------------------------------------
    def photon_counts(self, stream=None) -> np.ndarray:
        out = np.zeros(self.R, dtype=np.int64)
        _check(self.L.edm_get_photon_counts(self.handle, _ptr(out), _stream_handle(stream)), "edm_get_photon_counts")
        return out

    def photons(self, replica: int = 0, stream=None):
        cap = int(self._phot[replica].max_photons)
        pid = np.empty(cap, np.int32)
        t = np.empty(cap, np.float64)
        ch = np.empty(cap, np.int8)
        fr = np.empty(cap, np.uint8)
        n = _check(self.L.edm_get_photons(self.handle, replica, _ptr(pid), _ptr(t), _ptr(ch), _ptr(fr), cap,
                                          _stream_handle(stream)), "edm_get_photons")
        return pid[:n].copy(), t[:n].copy(), ch[:n].copy(), fr[:n].astype(bool)

    def flim(self, replica: int = 0, stream=None) -> np.ndarray:
        sp = self._scope[replica]
        shape = (sp.n_channels, sp.nx, sp.ny, sp.n_bins)
        out = np.empty(shape, dtype=np.uint32)
        _check(self.L.edm_get_flim(self.handle, replica, _ptr(out), out.size, _stream_handle(stream)), "edm_get_flim")
        return out

    def reset_flim(self, stream=None):
        _check(self.L.edm_reset_flim(self.handle, _stream_handle(stream)), "edm_reset_flim")

    def counters(self, stream=None) -> np.ndarray:
        out = np.zeros((self.R, PR.NCOUNTERS), dtype=np.int64)
        _check(self.L.edm_get_counters(self.handle, _ptr(out), _stream_handle(stream)), "edm_get_counters")
        return out

    def status(self, stream=None) -> int:
        v = C.c_uint32(0)
        _check(self.L.edm_get_status(self.handle, C.byref(v), _stream_handle(stream)), "edm_get_status")
        return int(v.value)

    def cells(self, replica: int = 0, stream=None):
        p = self._dyn[replica]
        nc = p.nx * p.ny
        start = np.empty(nc + 1, np.int32)
        mem = np.empty(max(p.n_particles, 1), np.int32)
        _check(self.L.edm_get_cells(self.handle, replica, _ptr(start), _ptr(mem), nc + 1, mem.size,
                                    _stream_handle(stream)), "edm_get_cells")
        return start, mem[:p.n_particles]


# ---------------------------------------------------------------------------
# keyed noise of the device generator (for injection / tests)
# ---------------------------------------------------------------------------
def device_normals(seed: int, step: int, stream_id: int, keys) -> np.ndarray:
    import torch
    L = load_library()
    k = torch.as_tensor(np.asarray(keys, dtype=np.int64), device="cuda")
    out = torch.empty((k.numel(), 2), dtype=torch.float64, device="cuda")
    _check(L.edm_noise_normal_pairs(seed, step, stream_id, C.c_void_p(k.data_ptr()), k.numel(),
                                    C.c_void_p(out.data_ptr()), None), "edm_noise_normal_pairs")
    return out.cpu().numpy()


def device_uniforms(seed: int, step: int, stream_id: int, a, b=None) -> np.ndarray:
    import torch
    L = load_library()
    ka = torch.as_tensor(np.asarray(a, dtype=np.int64), device="cuda")
    kb = None if b is None else torch.as_tensor(np.asarray(b, dtype=np.int64), device="cuda")
    out = torch.empty((ka.numel(), 2), dtype=torch.float64, device="cuda")
    _check(L.edm_noise_uniforms(seed, step, stream_id, C.c_void_p(ka.data_ptr()),
                                None if kb is None else C.c_void_p(kb.data_ptr()), ka.numel(),
                                C.c_void_p(out.data_ptr()), None), "edm_noise_uniforms")
    return out.cpu().numpy()


# ---------------------------------------------------------------------------
# Device-resident system bound to one ParticleState
# ---------------------------------------------------------------------------
_SYNC_FIELDS = ("positions", "species_id", "is_alive", "bond_partner", "has_dye", "dye_type_id",
                "ctmc_state", "is_bleached")


class DeviceSystem:
    """One replica on the GPU, bound to a host ParticleState.

    Shared by the DynamicsEngine / PhotonSimulator / VirtualMicroscope of the
    same state (state._device_owner).  Host arrays are uploaded lazily when
    they changed since the last sync, and downloaded on request."""

    def __init__(self, config, state, scan_duty_fraction: Optional[float] = None, precision: int = 64,
                 device: int = 0):
        self.config = config
        self.state = state
        self.precision = precision
        self.dp, self.hill, self.derived = PR.build_dyn_params(config, state.N)
        self.duty = scan_duty_fraction
        phot = scope = None
        self.pd = self.sd = None
        if scan_duty_fraction is not None and len(config.fluorophores) > 0:
            self.pp, self.pd = PR.build_phot_params(config, state.N, int(np.count_nonzero(state.has_dye)),
                                                    scan_duty_fraction)
            self.sp, self.sd = PR.build_scope_params(config)
            phot, scope = [self.pp], [self.sp]
        self.engine = Engine([self.dp], self.hill, phot, scope, precision=precision, device=device)
        self._snapshot = None
        self._host_current = True
        self.upload()
        state._device_owner = self
        self._host_dirty = False

    @property
    def has_photophysics(self) -> bool:
        return self.pd is not None and self.pd.active

    def _host_changed(self) -> bool:
        if self._snapshot is None:
            return True
        s = self.state
        return any(not np.array_equal(getattr(s, f), self._snapshot[f]) for f in _SYNC_FIELDS)

    def upload(self):
        s = self.state
        self.engine.set_state(s.positions, s.species_id, s.is_alive, s.bond_partner, s.has_dye, s.dye_type_id,
                              s.ctmc_state, s.is_bleached)
        self._snapshot = {f: getattr(s, f).copy() for f in _SYNC_FIELDS}
        self._host_current = True

    def ensure_device(self):
        """Upload host arrays if the user changed them since the last sync."""
        if self._host_current and (self._host_dirty or self._host_changed()):
            self.upload()
            self._host_dirty = False

    def mark_device_newer(self):
        self._host_current = False

    def _download_state(self):
        if self._host_current:
            return
        st = self.engine.get_state()
        s = self.state
        s.positions[:] = st["positions"]
        s.species_id[:] = st["species"]
        s.is_alive[:] = st["alive"].astype(bool)
        s.bond_partner[:] = st["bond"]
        s.ctmc_state[:] = st["ctmc"]
        s.is_bleached[:] = st["bleached"].astype(bool)
        self._snapshot = {f: getattr(s, f).copy() for f in _SYNC_FIELDS}
        self._host_current = True

    def sync_host(self):
        self._download_state()
