"""Benchmark of the per-timestep hot path on B200.

Workload (headline): the batched ensemble -- 512 independent PIP3/PTEN
membrane replicas, particle count log-uniform in 1,000-50,000 per replica,
box side scaled to keep the density, k_cat and K_half jittered, float32
cell-relative path, every BD step = dynamics + reactions + PSS photophysics
+ PSF/TCSPC detection of all replicas, captured as CUDA graphs of 100 steps.

A bench "step" is one FLIM frame of 100 BD timesteps over all replicas:
pipeline steps, then finalize_frame (dark counts, afterpulsing).

* value      particle-steps/s (membrane particles x BD steps / s) with the
             state resident on the GPU, whole job over all ranks;
* e2e        the same metric through the C-ABI frame loop a caller runs with
             host buffers: per frame upload the state from pinned memory,
             100 pipeline steps, finalize, read back every FLIM stack and
             the state;
* roofline   the dominant kernel group's algorithmic bytes / CUDA-event time;
* fp64_plain the plain float64 path (same kernels, one 13,000-particle
             system, per-step launches, no graphs) for the FP32/FP64 ratio;
* large_membrane the 1.3M-particle 100x100 µm^2 harmonic membrane on the
             float32 and float64 paths (CUDA graphs of 100 steps each), with
             the float32 path's per-step position error in lockstep with the
             float64 path and its reaction-count deviation over 100 steps;
* cpu_baseline the CPU oracle (the reference algorithm restated in C) on
             this host's cores on a bounded sample of the same workload.

`--impl reference` runs the CPU oracle alone on a bounded sample of the
same workload with every host core (rank 0 only) and prints its line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s & FLIM px/s: batched FP32 vs plain FP64, 1 B200, fixed error"
UNIT = "particle-steps/s"
STEPS_PER_FRAME = 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10, help="timed frames (100 BD steps each)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--flim-replicas", type=int, default=256, help="FLIM acquisition replicas (256^2 px each)")
    ap.add_argument("--no-flim", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the 1.3M-particle float32-vs-float64 comparison")
    ap.add_argument("--no-autotune", action="store_true", help="keep the fixed default launch shapes")
    ap.add_argument("--shapes", default=None,
                    help="launch-shape candidates of k_scatter,k_move,k_contacts instead of tuning (e.g. 1,5,7: "
                         "a profiler run replays the shapes a plain run tuned)")
    return ap.parse_args()


def rank_replicas(n_replicas: int, seed: int, rank: int):
    """The replicas of one rank: each rank runs its own ensemble (weak
    scaling, no exchange between ranks), seeded per rank."""
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    return W.ensemble_replicas(n_replicas, seed=seed + 7919 * rank)


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Job time = the slowest rank's time (all-reduce MAX)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_particle_steps(n_membrane_local: int, world: int, steps: int, device=None) -> int:
    """Membrane particle-steps of the whole job (sum over ranks)."""
    if world <= 1:
        return n_membrane_local * steps
    import torch
    import torch.distributed as dist
    t = torch.tensor([n_membrane_local], dtype=torch.int64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item()) * steps


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU side: the oracle on a bounded sample
# ---------------------------------------------------------------------------
def oracle_sample(raws, steps: int, threads: int):
    """Run `steps` BD steps (full per-step path) of each replica in `raws` on
    the CPU oracle, replicas in parallel threads; returns particle-steps/s."""
    from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
    from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
    from flim_microscopy_simulator_with_causal_inference_b200.particles import ParticleState
    from oracle import oracle as O

    sims = []
    for raw in raws:
        cfg = config_from_dict(raw)
        st = ParticleState(cfg)
        dp, _, _ = PR.build_dyn_params(cfg, st.N, hill_len=2)
        duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
        _, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty)
        sp, _ = PR.build_scope_params(cfg)
        sims.append((O.OracleSimulation(cfg, st, dp, pd, sp, duty), int(sum(cfg.initial_populations.values()))))

    def run(sim):
        o, _ = sim
        for _ in range(steps):
            o.bd_step()

    O.lib()
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(run, sims))
    dt = time.perf_counter() - t0
    ps = sum(n for _, n in sims) * steps
    return ps / dt, dt, ps


def oracle_sample_sized(raws, threads: int, target_s: float = 10.0):
    """oracle_sample with the step count calibrated so the timed run takes
    about target_s seconds (10 calibration steps first, at most 2000 steps)."""
    _, dt, _ = oracle_sample(raws, 10, threads)
    steps = int(min(2000, max(10, round(10 * target_s / max(dt, 1e-3)))))
    v, dt, ps = oracle_sample(raws, steps, threads)
    return v, dt, ps, steps


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    raws = W.ensemble_replicas(args.replicas, seed=args.seed)
    cores = os.cpu_count() or 1
    # bounded sample: the 16 replicas nearest the median size, 10 BD steps each
    sizes = np.array([sum(r["initial_populations"].values()) for r in raws])
    order = np.argsort(np.abs(sizes - np.median(sizes)))[:16]
    sample = [raws[i] for i in order]
    for _ in range(max(0, args.warmup)):
        oracle_sample(sample[:2], 1, cores)
    vals = []
    steps_used = 0
    for _ in range(max(1, args.steps)):
        v, dt, ps, steps_used = oracle_sample_sized(sample, cores, target_s=10.0)
        vals.append(v)
    value = float(statistics.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"batched ensemble, {args.replicas} replicas (sample: 16 median-size replicas x "
                               f"{steps_used} BD steps per timed step, about 10 s)", "replicas": args.replicas},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"16 median-size replicas x {steps_used} full BD steps "
                                   "(dynamics+photophysics+TCSPC), about 10 s per timed step, on " + PORT_NOTE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_flim:
        fv, fdt, fr, fcores = flim_cpu_sample(16, args.seed)
        line["flim"] = {"metric": "FLIM px/s", "value": fv, "unit": "px/s",
                        "workload": FLIM_WORKLOAD.format(R=args.flim_replicas),
                        "cpu_baseline": {"value": fv, "unit": "px/s", "cores": fcores, "kind": "port",
                                         "sample": f"{fr} replicas, float64 numpy restatement + numpy Poisson "
                                                   f"({fdt:.1f} s), one replica per process; the reference has no "
                                                   "batched acquisition"}}
    print(json.dumps(line), flush=True)


FLIM_WORKLOAD = ("batched FLIM acquisition: {R} replicas x 256x256 px x 256 bins, 50,000 donors per replica "
                 "(bound fraction U(0,1)), 31-tap PSF (sigma 100 nm), 1000 photons/px budget")
FLIM_BYTES_PER_PX = 256 * 4 + 8  # histogram written + the two intensity values read
PORT_NOTE = ("the C restatement of the reference's algorithm (oracle/edm_oracle.c, pinned bit-exactly to the "
             "reference), not the reference's own Python/Numba code")


def _flim_cpu_replica(args):
    """One replica of the float64 numpy restatement (a worker process's task)."""
    n_replicas, seed, r = args
    from flim_microscopy_simulator_with_causal_inference_b200 import flim_acquire as FA
    from flim_microscopy_simulator_with_causal_inference_b200.config import config_from_dict
    from oracle import flim_oracle as FO
    if r < 0:  # warm-up task: imports only
        return 0
    p, _ = FA.build_flim_params(config_from_dict(FA.flim_config()), n_replicas, 50_000, 1000.0, seed)
    bf = FA.bound_fractions(n_replicas, seed)
    e = FO.acquire_expected(p, bf, r)
    FO.poisson_histograms(e["mu"], seed + r)
    return 65536


def flim_cpu_sample(n_replicas: int, seed: int):
    """The float64 numpy restatement (oracle/flim_oracle.py) of the acquisition
    on a bounded sample of replicas, one replica per worker process on every
    host core (spawned: the parent holds a CUDA context).  Returns FLIM px/s,
    seconds, replicas, cores."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    cores = min(os.cpu_count() or 1, n_replicas)
    with ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_flim_cpu_replica, [(n_replicas, seed, -1)] * cores))
        t0 = time.perf_counter()
        px = sum(ex.map(_flim_cpu_replica, [(n_replicas, seed, r) for r in range(n_replicas)]))
        dt = time.perf_counter() - t0
    return px / dt, dt, n_replicas, cores


def large_membrane_bench(device: int, stream) -> dict:
    """The 1.3M-particle membrane (100x100 µm^2, harmonic repulsion, 200x200
    density grid) on the float32 and float64 GPU paths: throughput of each
    (100 steps in CUDA graphs, dynamics + photons + detection), the float32
    path's position error after one step from the float64 path's state
    (5 lockstep steps), and the relative deviation of its reaction counts
    after 100 free-running steps from the same initial state."""
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    raw = W.config2(n_frames=1)
    ens = {prec: Ensemble([raw], precision=prec, photons=True, device=device) for prec in (32, 64)}
    n_mem = ens[32].total_membrane
    rates, counts = {}, {}
    shapes = {}
    for prec, e in ens.items():
        shapes[prec] = {k: v["candidate"] for k, v in e.engine.autotune(3, stream=stream).items()}
        e.engine.pipeline_steps(100, True, 100, stream=stream)  # capture + warm
        stream.synchronize()
        e.upload(stream=stream)  # back to the initial state, step 0
        e.engine.set_step(0)
        c0 = e.engine.counters(stream=stream).sum(axis=0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.engine.pipeline_steps(100, True, 100, stream=stream)
        b.record(stream)
        stream.synchronize()
        rates[prec] = n_mem * 100 / (a.elapsed_time(b) / 1e3)
        counts[prec] = e.engine.counters(stream=stream).sum(axis=0) - c0
    ev = counts[64][2:6].astype(np.float64)
    dev = float(np.abs(counts[32][2:6] - counts[64][2:6]).sum() / max(1.0, ev.sum()))
    # lockstep: the float32 path steps from the float64 path's state
    e32, e64 = ens[32].engine, ens[64].engine
    worst = 0.0
    same_events = True
    for _ in range(5):
        st = e64.get_state(stream=stream)
        e32.set_state(st["positions"], st["species"], st["alive"], st["bond"], st["has_dye"], ens[64].host["dye"],
                      st["ctmc"], st["bleached"], stream=stream)
        e32.set_step(e64.get_step())
        e64.pipeline_steps(1, True, 0, stream=stream)
        e32.pipeline_steps(1, True, 0, stream=stream)
        a64, a32 = e64.get_state(stream=stream), e32.get_state(stream=stream)
        d = np.abs(a32["positions"] - a64["positions"])
        d = np.minimum(d, np.array([100.0, 100.0]) - d)  # periodic box
        worst = max(worst, float(d.max()))
        same_events &= bool(np.array_equal(a32["species"], a64["species"]) and np.array_equal(a32["alive"], a64["alive"]))
    del ens
    torch.cuda.empty_cache()
    return {"workload": "1.3M-particle 100x100 um^2 PIP3/PTEN membrane, harmonic repulsion, 200x200 density grid, "
                        "dynamics + PSS photons + TCSPC per step, CUDA graphs of 100 steps",
            "unit": UNIT, "fp32": rates[32], "fp64": rates[64], "fp32_over_fp64": rates[32] / rates[64],
            "lockstep_max_position_error_um": worst, "lockstep_event_sets_identical": same_events,
            "reaction_count_rel_deviation_100_steps": dev,
            "reaction_counts_100_steps": {"fp32": counts[32][2:6].tolist(), "fp64": counts[64][2:6].tolist(),
                                          "fields": ["catalytic", "recruited", "detached", "converted"]},
            "launch_shapes": {"fp32": shapes[32], "fp64": shapes[64]}}


def flim_bench(args, device: int, rank: int, world: int, stream):
    """FLIM px/s of the batched acquisition (device-resident and end to end)."""
    import ctypes
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import flim_acquire as FA
    R = args.flim_replicas
    acq = FA.FlimAcquisition(FA.flim_config(), R, n_emitters=50_000, photon_budget=1000.0,
                             seed=args.seed + 7919 * rank, device=device)
    s = int(stream.cuda_stream)
    for _ in range(max(3, args.warmup)):
        acq.acquire(stream=s)
    stream.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
    with ClockSampler(device) as clk:
        for k in range(args.steps):
            ev[3 * k].record(stream)
            acq.project(stream=s)
            ev[3 * k + 1].record(stream)
            acq.histograms(True, stream=s)
            ev[3 * k + 2].record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    # lifetime readouts (mean arrival time + phasor) of all histograms: one streaming pass
    from flim_microscopy_simulator_with_causal_inference_b200 import readouts as RD
    hist_ptr, _ = acq.device_ptr(FA.HIST)
    ro_out = torch.empty((6, R * 65536), dtype=torch.float64, device="cuda")
    for _ in range(2):
        RD.lifetimes_device(hist_ptr, R * 65536, 256, 25e-9, out=ro_out, stream=s)
    rev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    for k in range(args.steps):
        rev[2 * k].record(stream)
        RD.lifetimes_device(hist_ptr, R * 65536, 256, 25e-9, out=ro_out, stream=s)
        rev[2 * k + 1].record(stream)
    stream.synchronize()
    ro_ms = statistics.mean(rev[2 * k].elapsed_time(rev[2 * k + 1]) for k in range(args.steps))
    ro_bytes = R * 65536 * (256 * 4 + 6 * 8)
    keep_tau = ro_out[1].view(R, 65536) if world > 1 else None  # mean-arrival-time maps, for the collection
    del ro_out
    proj = [ev[3 * k].elapsed_time(ev[3 * k + 1]) for k in range(args.steps)]
    hist = [ev[3 * k + 1].elapsed_time(ev[3 * k + 2]) for k in range(args.steps)]
    ms = max_over_ranks(ev[0].elapsed_time(ev[-1]), world, "cuda")
    px = R * 65536 * world * args.steps
    value = px / (ms / 1e3)
    hist_ms = statistics.mean(hist)
    proj_ms = statistics.mean(proj)
    peak, peak_kind = peaks()
    achieved = FLIM_BYTES_PER_PX * R * 65536 / (hist_ms / 1e3) / 1e9
    gemm_flops = 2 * (2 * 2 * 256 ** 3) * R  # two maps, two 256^3 products each (algorithmic)
    traffic = ro_traffic = None
    tr_file = ROOT / "profiles" / "traffic.json"
    if tr_file.exists() and R == 256:  # the committed figures are for 256 replicas
        tr = json.loads(tr_file.read_text())
        traffic, ro_traffic = tr.get("hist"), tr.get("readout")
    err = acq.error_word()

    # e2e: host bound fractions in, every histogram out to pinned host memory
    ring = [torch.empty(65536 * 256, dtype=torch.int32).pin_memory().numpy() for _ in range(4)]
    bf = FA.bound_fractions(R, args.seed + 1)
    bf_pinned = torch.from_numpy(bf).pin_memory().numpy()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    all8 = torch.empty(R * 65536 * 256, dtype=torch.uint8).pin_memory().numpy()

    def e2e_acquisitions(narrow: bool):
        """Acquisitions through the C ABI: bound fractions H2D, acquire, every
        replica's histograms D2H, as 8-bit counts narrowed on the device when
        they fit (edm_flim_read_hist_narrow_async: lossless, checked there,
        the copy overlapping the next acquisition; per replica at 16 bits,
        then uint32, when not), or as the uint32 array."""
        d2h = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.steps):
            acq.set_inputs(bf_pinned, args.seed + 1 + k, stream=s)
            acq.acquire(stream=s)
            if narrow:
                rc = acq.lib.edm_flim_read_hist_narrow_async(acq._h, 8, all8.ctypes.data_as(ctypes.c_void_p),
                                                             all8.nbytes, s)
                if rc == 0:
                    d2h += all8.nbytes
                    continue
                if rc != -5:  # not EDM_ERANGE: a real failure
                    acq._check(rc)
            for r in range(R):
                buf = ring[r % 4]
                ptr = buf.ctypes.data_as(ctypes.c_void_p)
                done = False
                for bits in ((16,) if narrow else ()):
                    rc = acq.lib.edm_flim_read_hist_narrow(acq._h, r, bits, ptr, buf.nbytes, s)
                    if rc == 0:
                        d2h += 65536 * 256 * bits // 8
                        done = True
                        break
                    if rc != -5:  # not EDM_ERANGE: a real failure
                        acq._check(rc)
                if not done:
                    acq._check(acq.lib.edm_flim_read(acq._h, FA.HIST, r, ptr, buf.nbytes, s))
                    d2h += 65536 * 256 * 4
        acq.read_wait()
        torch.cuda.synchronize()
        return max_over_ranks(time.perf_counter() - t0, world, "cuda"), d2h / args.steps

    e2e_s, d2h_narrow = e2e_acquisitions(True)
    e2e32_s, d2h_32 = e2e_acquisitions(False)
    acq.close()
    return {
        "metric": "FLIM px/s", "value": value, "unit": "px/s", "ms_per_step": ms / args.steps,
        "workload": FLIM_WORKLOAD.format(R=R), "replicas_per_gpu": R, "dtype": "bf16 GEMM / f32 accumulate, f64 bins",
        "kernel_ms": {"project": proj_ms, "histograms": hist_ms},
        "roofline": {"bound": "hbm", "kernel": "k_hist", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "alg_bytes_per_px": FLIM_BYTES_PER_PX, "alg_bytes": FLIM_BYTES_PER_PX * R * 65536},
        "tensor": {"kernel": "k_umma_gemm x2 (+ emitter maps)", "alg_tflops": gemm_flops / (proj_ms / 1e3) / 1e12,
                   "note": "algorithmic 2 x 2*256^3 FLOP per map over the whole projection time"},
        "e2e": {"value": px / e2e_s, "unit": "px/s", "h2d_bytes_per_step": int(bf.nbytes),
                "d2h_bytes_per_step": int(d2h_narrow),
                "note": "per acquisition: bound fractions H2D, acquire, every histogram D2H to pinned host memory "
                        "as 8-bit counts narrowed on the device (edm_flim_read_hist_narrow_async: lossless, the "
                        "copy overlapping the next acquisition; a count that does not fit makes the read fall "
                        "back to 16 bits, then to uint32)",
                "uint32": {"value": px / e2e32_s, "d2h_bytes_per_step": int(d2h_32),
                           "note": "the same loop reading the uint32 histograms"}},
        "readout": {"kernel": "k_readout (mean arrival time + phasor of every pixel)", "ms": ro_ms,
                    "px_per_s": R * 65536 / (ro_ms / 1e3),
                    "roofline": {"bound": "hbm", "achieved": ro_bytes / (ro_ms / 1e3) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": ro_bytes / (ro_ms / 1e3) / 1e9 / peak,
                                 "traffic": ro_traffic, "alg_bytes_per_px": 256 * 4 + 6 * 8}},
        "gpu_launches": 5 * args.steps, "error_word": err, "clocks": clk.summary(),
        "l2": "histograms 17 GB per acquisition >> 126 MB L2",
        "_tau_maps": keep_tau,
    }


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    device = local
    torch.cuda.set_device(device)
    from flim_microscopy_simulator_with_causal_inference_b200 import params as PR
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble

    raws = rank_replicas(args.replicas, args.seed, rank)
    ens = Ensemble(raws, precision=32, photons=True, device=device)
    eng = ens.engine
    stream = torch.cuda.Stream(device=device)
    frame = 0
    # launch shapes: timed on the first real steps of the run (untimed here), then fixed
    if args.shapes:
        shapes = eng.set_launch_shapes([int(x) for x in args.shapes.split(",")])
    elif not args.no_autotune:
        shapes = eng.autotune(3, stream=stream)
    else:
        shapes = eng.launch_shapes()
    stream.synchronize()
    ens.upload(stream=stream)  # the timed frames start from the initial state
    eng.set_step(0)

    def run_frame():
        nonlocal frame
        eng.pipeline_steps(STEPS_PER_FRAME, True, STEPS_PER_FRAME, stream=stream)
        eng.finalize(frame, stream=stream)
        eng.reset_flim(stream=stream)
        frame += 1

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            run_frame()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            run_frame()
        e1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    n_mem = ens.total_membrane
    job_ps = job_particle_steps(n_mem, world, STEPS_PER_FRAME * args.steps, "cuda")
    value = job_ps / (ms / 1e3)
    launches = eng.launches_per_step(True) * STEPS_PER_FRAME * args.steps + 2 * args.steps
    status = eng.status()

    # ---- e2e through the C ABI with host buffers ---------------------------
    h = ens.host
    pinned = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in h.items()}
    flim_elems = eng.flim_elems()
    flim_host = torch.empty(flim_elems, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    tdt = {np.float64: torch.float64, np.int32: torch.int32, np.uint8: torch.uint8, np.int8: torch.int8}
    state_out = {k: torch.empty((eng.N, w) if w > 1 else (eng.N,), dtype=tdt[dt]).pin_memory().numpy()
                 for k, dt, w in eng.STATE_FIELDS}
    state_bytes_in = sum(v.nbytes for v in pinned.values())
    sp_cap = max(1, flim_elems // 64)
    sp_idx = torch.empty(sp_cap, dtype=torch.int64).pin_memory().numpy()
    sp_cnt = torch.empty(sp_cap, dtype=torch.int32).pin_memory().numpy().view(np.uint32)

    state_outs = [state_out, {k: torch.empty((eng.N, w) if w > 1 else (eng.N,), dtype=tdt[dt]).pin_memory().numpy()
                              for k, dt, w in eng.STATE_FIELDS}]

    # the transfers' staging areas and the sparse output are allocated by their first use, outside the timing
    eng.set_state_async(pinned, stream=stream)
    eng.get_state_async(state_outs[0], stream=stream)
    eng.transfers_wait()
    eng.frame_out_sparse(sp_idx, sp_cnt, stream=stream)
    stream.synchronize()

    def e2e_loop(sparse: bool):
        """Frames through the C ABI with pinned host buffers, the transfers
        overlapped with the computation: every frame uploads its state
        (edm_set_state_async: the next frame's upload runs while this frame
        computes), runs 100 steps, finalizes, downloads the state
        (edm_get_state_async: while the next frame computes) and reads every
        replica's stacks (their nonzero bins with edm_frame_out_sparse, or
        dense on the copy stream)."""
        nonlocal frame
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        d2h_flim = 0
        t0 = time.perf_counter()
        eng.set_state_async(pinned, stream=stream)
        for k in range(args.steps):
            eng.pipeline_steps(STEPS_PER_FRAME, True, STEPS_PER_FRAME, stream=stream)
            eng.finalize(frame, stream=stream)
            if k + 1 < args.steps:  # the next frame's state goes up while this frame computes
                eng.stage_state_async(pinned)
            done = False
            if sparse:
                try:
                    nnz = eng.frame_out_sparse(sp_idx, sp_cnt, stream=stream)
                    d2h_flim += nnz * 12
                    done = True
                except RuntimeError:  # a frame denser than the buffer: read it dense
                    pass
            if not done:
                # snapshot + clear on the stream, D2H on the engine's copy stream, overlapping the next frame
                eng.frame_out_begin(flim_host, stream=stream)
                d2h_flim += flim_elems * 4
            # the state comes down while the next frame computes (after the stacks' small read)
            st = eng.get_state_async(state_outs[k % 2], stream=stream)
            if k + 1 < args.steps:
                eng.install_state(stream=stream)
            frame += 1
        eng.frame_out_wait()
        eng.transfers_wait()
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        state_bytes_out = sum(v.nbytes for v in st.values())
        return job_ps / e2e_s, state_bytes_in / STEPS_PER_FRAME, \
            (d2h_flim / args.steps + state_bytes_out) / STEPS_PER_FRAME

    e2e_value, h2d, d2h = e2e_loop(sparse=True)
    e2e_dense, _, d2h_dense = e2e_loop(sparse=False)

    # ---- per-kernel timing (CUDA events inside a captured graph) -------------
    prof = eng.profile_steps(20, True, stream=stream)
    passes = eng.profile_passes(10, stream=stream)  # reaction passes one by one (eager, for the breakdown)
    N = ens.total_particles
    n_buckets = int(sum(p.nx * p.ny + 1 for p in ens.dyn_params))
    groups = {k: prof[k] for k in ("cell_scan", "scatter", "move", "reactions", "photophysics", "detection")}
    # Candidate kernels with their algorithmic bytes per launch (float32 path).  Single-kernel
    # groups are timed inside the graph; the reaction passes eagerly, scaled so that they add up to
    # the reactions group's in-graph time.
    cand = {
        "k_scan (3 launches)": (groups["cell_scan"], 20 * n_buckets, "20 B per sort bucket"),
        "k_scatter": (groups["scatter"], 46 * N, "46 B per slot: 21 B slot record (offset hi 8 + lo 4, cell, flags, "
                                                 "id) read + written, 4 B inverse map"),
        "k_move": (groups["move"], 37 * N, "37 B per slot: 21 B pre-move slot read (offset hi 8 + lo 4, cell, "
                                           "flags, id), 16 B offset hi + lo and cell written"),
    }
    eager_rx = sum(pm for _, _, pm in passes)
    scale_rx = groups["reactions"] / eager_rx if eager_rx > 0 else 1.0
    for kind, idx, pm in passes:
        if kind == "contacts":
            cand["k_contacts"] = (pm * scale_rx, 22 * N, "22 B per slot: flag sweep + every slot's cell, flags, "
                                                         "pre- and post-move position read once")
        elif kind == "pass_draws":
            cand["k_pass_draws"] = (pm * scale_rx, 1 * N, "1 B per slot: flag sweep")
    dom = max(cand, key=lambda k: cand[k][0])
    dom_ms, dom_bytes, dom_def = cand[dom]
    peak, peak_kind = peaks()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tr_file = ROOT / "profiles" / "traffic.json"
    if tr_file.exists() and args.replicas == 512 and world == 1:  # the committed figures are for this workload
        traffic = json.loads(tr_file.read_text()).get(dom)
    step_ms = ms / args.steps / STEPS_PER_FRAME  # device ms per BD step, whole job
    step_roofline = {
        "alg_bytes_per_particle_step": 64,
        "definition": "16 B packed state read + written, cell-sorted copy written + read once per particle-step",
        "membrane": {"particles": n_mem, "achieved": 64 * n_mem / (step_ms / 1e3) / 1e9,
                     "frac": 64 * n_mem / (step_ms / 1e3) / 1e9 / peak},
        "all_slots": {"particles": N, "achieved": 64 * N / (step_ms / 1e3) / 1e9,
                      "frac": 64 * N / (step_ms / 1e3) / 1e9 / peak},
        "ms_per_bd_step": step_ms,
    }
    kernel_roofline = {k: {"ms": v[0], "alg_bytes": v[1], "frac": v[1] / (v[0] / 1e3) / 1e9 / peak,
                           "definition": v[2]} for k, v in cand.items()}

    # ---- plain float64 path: one 13,000-particle system, per-step launches ---
    fp64 = None
    if not args.no_fp64 and rank == 0:
        from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble as E2
        c1 = E2([W.config1(n_frames=1)], precision=64, photons=True, device=device)
        c1.engine.pipeline_steps(20, True, 0, stream=stream)
        stream.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        n64 = 200
        f0.record(stream)
        c1.engine.pipeline_steps(n64, True, 0, stream=stream)
        f1.record(stream)
        stream.synchronize()
        fp64 = c1.total_membrane * n64 / (f0.elapsed_time(f1) / 1e3)
        del c1

    large = None
    if not args.no_large and rank == 0:
        try:  # a secondary comparison: report its failure in the line rather than lose the line
            large = large_membrane_bench(device, stream)
        except Exception as ex:  # noqa: BLE001
            large = {"error": f"{type(ex).__name__}: {ex}"}

    # ---- batched FLIM acquisition -------------------------------------------
    flim = None
    if not args.no_flim:
        flim = flim_bench(args, device, rank, world, stream)

    # ---- end-of-run collection over ranks (untimed): per-replica counters, ----
    # lifetime maps and the pooled TCSPC decay of one more frame
    collect = None
    tau_maps = flim.pop("_tau_maps", None) if flim is not None else None
    if world > 1:
        from flim_microscopy_simulator_with_causal_inference_b200 import gather as G
        from flim_microscopy_simulator_with_causal_inference_b200 import readouts as RD
        eng.pipeline_steps(STEPS_PER_FRAME, True, STEPS_PER_FRAME, stream=stream)
        eng.finalize(frame, stream=stream)
        stream.synchronize()
        ptr, _, nb = RD.engine_stack(eng, 0)
        stacks = G.device_view(ptr, eng.flim_elems(), np.int32).view(-1, nb)  # counts < 2^31
        decay = torch.sum(stacks, dim=0, dtype=torch.int64)
        eng.reset_flim(stream=stream)
        torch.cuda.synchronize()
        dist.barrier()
        c0 = time.perf_counter()
        got = G.collect_ensemble(eng.counters(stream=stream), tau_maps, decay, device="cuda")
        torch.cuda.synchronize()
        collect = {"ms": 1e3 * max_over_ranks(time.perf_counter() - c0, world, "cuda"),
                   "replicas": int(got["counters"].shape[0]),
                   "tau_map_bytes": int(got["tau_maps"].numel() * 8) if "tau_maps" in got else 0,
                   "pooled_decay_counts": int(got["decay"].sum().item()),
                   "note": "NCCL all-gather of per-replica counters and lifetime maps, all-reduce of the pooled "
                           "decay; outside the timed region"}
    elif flim is not None:
        flim.pop("_tau_maps", None)

    # ---- CPU baseline (oracle) on a bounded sample ---------------------------
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        sizes = np.array([sum(r["initial_populations"].values()) for r in raws])
        order = np.argsort(np.abs(sizes - np.median(sizes)))[:16]
        cores = os.cpu_count() or 1
        v, dt, ps, nsteps = oracle_sample_sized([raws[i] for i in order], cores, target_s=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"16 median-size replicas x {nsteps} full BD steps ({ps} particle-steps, {dt:.1f} s) on "
                         + PORT_NOTE}
        if flim is not None:
            fv, fdt, fr, fcores = flim_cpu_sample(16, args.seed)
            flim["cpu_baseline"] = {"value": fv, "unit": "px/s", "cores": fcores, "kind": "port",
                                    "sample": f"{fr} replicas, float64 numpy restatement + numpy Poisson ({fdt:.1f} s), "
                                              "one replica per process; the reference has no batched acquisition"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched ensemble: {args.replicas} PIP3/PTEN replicas per GPU, N log-uniform "
                                   f"1k-50k ({n_mem} membrane + {N - n_mem} dormant particles), full BD step "
                                   "(dynamics+reactions+PSS photons+TCSPC), CUDA graphs of 100 steps; step = one "
                                   "frame of 100 BD steps",
                       "replicas": args.replicas, "particles": N, "membrane_particles": n_mem,
                       "bd_steps_per_step": STEPS_PER_FRAME, "precision": "f32 cell-relative positions",
                       "l2": "working set > 126 MB L2 (resident state ~37 B/particle)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "note": "per frame: state H2D from pinned host (edm_set_state_async: uploaded while the "
                            "previous frame computes), 100 BD steps, finalize, state D2H (edm_get_state_async: "
                            "downloaded while the next frame computes), every replica's FLIM stacks D2H as their "
                            "nonzero bins (edm_frame_out_sparse: element index + count, lossless); bytes are per "
                            "BD step",
                    "dense_stacks": {"value": e2e_dense, "d2h_bytes_per_step": int(d2h_dense),
                                     "note": "the same loop reading the stacks dense (edm_frame_out_begin on a "
                                             "copy stream, overlapping the next frame)"}},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "alg_bytes": dom_bytes, "alg_bytes_definition": dom_def, "kernel_ms": dom_ms,
                         "step": step_roofline, "kernels": kernel_roofline},
            "kernel_ms_per_step": groups,
            "launch_shapes": shapes,
            "kernel_ms_sum_vs_step": {"sum_of_groups": sum(groups.values()), "graph_ms_per_bd_step": step_ms,
                                      "profiled_step_ms": prof["step"]},
            "reaction_passes_eager_ms": [[k, i, m] for k, i, m in passes],
            "large_membrane": large,
            "fp64_plain": None if fp64 is None else {"value": fp64, "unit": UNIT,
                                                     "workload": "13,000-particle system with sine D(x), float64, "
                                                                 "per-step launches, full BD step"},
            "fp32_over_fp64": None if fp64 is None else value / world / fp64,
            "cpu_baseline": cpu,
            "flim": flim,
            "gpu_launches": launches,
            "status_word": status,
            "collect": collect,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
