"""End-of-run collection of a multi-GPU ensemble's results.

Replicas are independent: each rank (one process per GPU) runs its own slice
of the ensemble with no exchange while it steps.  At the end one collective
per quantity brings the per-replica results together over NVLink / NVSwitch
(NCCL; gloo on CPU):

* `gather_replicas` - arrays whose first axis is the rank's replicas
  (counters, lifetime maps, readout summaries), concatenated in rank order.
  Ranks may hold different replica counts: every rank's rows are padded to
  the largest count for one all-gather and trimmed after it;
* `reduce_sum` - arrays summed over all ranks (pooled TCSPC decays, totals).

Every rank calls the same functions in the same order with the same keys.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np


def _torch_dtype(dt: np.dtype):
    import torch
    return {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32,
            np.dtype(np.uint8): torch.uint8, np.dtype(np.int8): torch.int8}[np.dtype(dt)]


def _as_tensor(a, device):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device).contiguous()
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.copy()).to(device) if a.size else torch.zeros(a.shape, dtype=_torch_dtype(a.dtype),
                                                                            device=device)


def gather_replicas(arrays: Dict[str, "np.ndarray"], device="cpu", group=None) -> Dict[str, "np.ndarray"]:
    """{name: array [R_rank, ...]} on every rank -> {name: array [sum R, ...]}
    in rank order, on every rank (an all-gather).  Trailing shapes and dtypes
    must agree across ranks.  numpy inputs give numpy outputs; torch tensors
    (e.g. maps already on the GPU) give tensors on `device`."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    out = {}
    for name in sorted(arrays):
        is_np = not isinstance(arrays[name], torch.Tensor)
        a = _as_tensor(arrays[name], device)
        n = torch.tensor([a.shape[0]], dtype=torch.int64, device=device)
        sizes = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(sizes, n, group=group)
        counts = [int(x.item()) for x in sizes]
        buf = torch.zeros((max(counts),) + tuple(a.shape[1:]), dtype=a.dtype, device=device)
        if a.shape[0]:
            buf[: a.shape[0]] = a
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        cat = torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)
        out[name] = cat.cpu().numpy() if is_np else cat
    return out


def reduce_sum(arrays: Dict[str, np.ndarray], device="cpu", group=None) -> Dict[str, np.ndarray]:
    """{name: array} summed element-wise over all ranks (an all-reduce)."""
    import torch
    import torch.distributed as dist
    out = {}
    for name in sorted(arrays):
        is_np = not isinstance(arrays[name], torch.Tensor)
        t = _as_tensor(arrays[name], device).clone()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[name] = t.cpu().numpy() if is_np else t
    return out


class _DeviceArray:
    """A device buffer of this library exposed through the CUDA array
    interface, so torch.as_tensor wraps it without a copy."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, n: int, dtype=np.int32):
    """A CUDA tensor over n elements of `dtype` at device address ptr (no copy)."""
    import torch
    return torch.as_tensor(_DeviceArray(ptr, n, np.dtype(dtype).str), device="cuda")


def collect_ensemble(counters: np.ndarray, tau_maps: Optional[np.ndarray] = None,
                     decay: Optional[np.ndarray] = None, device="cpu", group=None) -> dict:
    """The ensemble's end-of-run results on every rank: per-replica counters
    [R_total, EDM_NCOUNTERS], per-replica lifetime maps (if given) and the
    pooled TCSPC decay summed over every rank's replicas and pixels."""
    per = {"counters": counters}
    if tau_maps is not None:
        per["tau_maps"] = tau_maps
    out = gather_replicas(per, device=device, group=group)
    if decay is not None:
        out.update(reduce_sum({"decay": decay}, device=device, group=group))
    return out
