"""Lifetime readouts of TCSPC stacks on the device (C ABI: edm_readout_lifetimes).

The reference computes them on the host with numpy (ed_mrdt/analysis.py):
mean_arrival_time (:87-150) and phasor_transform (:497-566).  Here they run
on the stacks where they live (the engine's FLIM stacks or the batched
acquisition's histograms), one pass over the counts, float64 sums.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import engine as E

FIELDS = ("intensity", "tau_mean_ns", "g", "s", "tau_phi_ns", "tau_mod_ns")


def lifetimes_device(stack_ptr: int, n_px: int, n_bins: int, time_range_s: float, harmonic: int = 1,
                     min_counts_mean: int = 10, min_counts_phasor: int = 20, out=None, stream=None):
    """Readouts of a device stack [n_px][n_bins] (uint32) as a float64 CUDA
    tensor [6][n_px] in FIELDS order."""
    import torch
    L = E.load_library()
    if out is None:
        out = torch.empty((6, n_px), dtype=torch.float64, device="cuda")
    if out.dtype != torch.float64 or tuple(out.shape) != (6, n_px) or not out.is_contiguous():
        raise ValueError("out must be a contiguous float64 CUDA tensor of shape (6, n_px)")
    E._check(L.edm_readout_lifetimes(C.c_void_p(stack_ptr), int(n_px), int(n_bins), float(time_range_s),
                                     int(harmonic), int(min_counts_mean), int(min_counts_phasor),
                                     C.c_void_p(out.data_ptr()), E._stream_handle(stream)), "edm_readout_lifetimes")
    return out


def engine_stack(engine: "E.Engine", replica: int = 0):
    """(device pointer, pixels (n_ch * nx * ny), n_bins) of an engine stack."""
    L = engine.L
    ptr, n_px, n_bins = C.c_void_p(), C.c_int64(), C.c_int32()
    E._check(L.edm_flim_stack_ptr(engine.handle, int(replica), C.byref(ptr), C.byref(n_px), C.byref(n_bins)),
             "edm_flim_stack_ptr")
    return ptr.value, int(n_px.value), int(n_bins.value)


def engine_readouts(engine: "E.Engine", replica: int, time_range_s: float, harmonic: int = 1,
                    min_counts_mean: int = 10, min_counts_phasor: int = 20, stream=None) -> dict:
    """Readouts of one replica's stacks, as host arrays [n_ch][nx][ny] per field."""
    ptr, n_px, n_bins = engine_stack(engine, replica)
    sp = engine._scope[replica]
    dev = lifetimes_device(ptr, n_px, n_bins, time_range_s, harmonic, min_counts_mean, min_counts_phasor,
                           stream=stream)
    host = dev.cpu().numpy()
    return {k: host[i].reshape(sp.n_channels, sp.nx, sp.ny) for i, k in enumerate(FIELDS)}
