"""Ensemble statistics of the float32 path against the float64 path.

The 13,000-particle membrane with the sine D(x) field runs free on both
paths from the same initial state with the same keyed noise, for 300 BD steps
with photons and detection.  The paths follow the same trajectories until two
particles meet closer than float32 offsets resolve (~1e-8 µm): their WCA
force, capped at the displacement limit, can then point another way, and the
difference spreads through collisions (about 1,000 of 13,000 particles by
step 100).  So the early displacements are compared tightly and the rest as
statistics of two ensembles, with error bars taken from the data:

* mean squared displacement of the particles alive at every step on both
  paths (a detached and recruited particle is placed anew, which is not
  diffusion): relative difference <= 1e-3 at lags of 1 and 10 steps; within
  4 standard errors at 100 and 300 steps;
* pair correlation g(r) of the alive particles on 0.02-0.5 µm in 24 bins:
  every bin within 4 Poisson standard errors + 0.005;
* reaction counts (catalytic, recruited, detached, converted): within
  4 sqrt(n) + 2 of the float64 count;
* TCSPC lifetime histogram summed over pixels and channels: mean arrival
  time within 4 standard errors, total counts within 4 sqrt(n) + 0.5 %.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L_BOX = 10.0


def _min_image(d):
    return d - L_BOX * np.round(d / L_BOX)


def _g_of_r(pos, r_min=0.02, r_max=0.5, nbins=24):
    """g(r) and the pair count of each bin."""
    from scipy.spatial import cKDTree
    tree = cKDTree(np.mod(pos, L_BOX), boxsize=L_BOX)
    edges = np.linspace(r_min, r_max, nbins + 1)
    cum = tree.count_neighbors(tree, edges)  # ordered pairs within each edge
    counts = np.diff(cum).astype(np.float64)
    n = len(pos)
    shell = np.pi * (edges[1:] ** 2 - edges[:-1] ** 2)
    return counts / (n * (n / L_BOX ** 2) * shell), counts


def _arrivals(stack, time_range_ns=25.0):
    """Mean arrival time (ns), its standard error and the photon count of the
    histogram summed over channels and pixels."""
    h = stack.astype(np.float64).sum(axis=(0, 1, 2))
    t = (np.arange(h.size) + 0.5) * time_range_ns / h.size
    n = h.sum()
    mean = (h * t).sum() / n
    var = (h * (t - mean) ** 2).sum() / n
    return float(mean), float(np.sqrt(var / n)), float(n)


def test_fp32_ensemble_statistics_match_fp64():
    import torch
    from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
    from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble
    raw = W.config1(n_frames=1)
    s = torch.cuda.Stream()
    runs = {}
    for prec in (32, 64):
        ens = Ensemble([raw], precision=prec, photons=True, device=0)
        eng = ens.engine
        st = eng.get_state(stream=s)
        prev = st["positions"].copy()
        unwrapped = prev.copy()
        always = st["alive"].astype(bool)
        snaps = {}
        for t in range(1, 301):
            eng.pipeline_steps(1, True, 0, stream=s)
            cur = eng.get_state(stream=s)
            p = cur["positions"]
            always &= cur["alive"].astype(bool)
            unwrapped += _min_image(p - prev)
            prev = p.copy()
            if t in (1, 10, 100, 300):
                snaps[t] = unwrapped.copy()
        final = eng.get_state(stream=s)
        runs[prec] = dict(start=st["positions"].copy(), snaps=snaps, always=always, final=final,
                          counters=eng.counters(stream=s)[0], flim=eng.flim(0, stream=s))
        del ens
    a, b = runs[32], runs[64]
    keep = a["always"] & b["always"]
    assert keep.sum() > 10000
    for t in (1, 10, 100, 300):
        r32 = np.sum((a["snaps"][t][keep] - a["start"][keep]) ** 2, axis=1)
        r64 = np.sum((b["snaps"][t][keep] - b["start"][keep]) ** 2, axis=1)
        m32, m64 = r32.mean(), r64.mean()
        if t <= 10:
            assert abs(m32 - m64) <= 1e-3 * m64, (t, m32, m64)
        else:
            se = np.sqrt((r32.var() + r64.var()) / keep.sum())
            assert abs(m32 - m64) <= 4 * se, (t, m32, m64, se)
    g32, n32 = _g_of_r(a["final"]["positions"][a["final"]["alive"].astype(bool)])
    g64, n64 = _g_of_r(b["final"]["positions"][b["final"]["alive"].astype(bool)])
    tol = 4 * g64 * np.sqrt(1.0 / np.maximum(n32, 1) + 1.0 / np.maximum(n64, 1)) + 0.005
    assert (np.abs(g32 - g64) <= tol).all(), (g32 - g64, tol)
    c32, c64 = a["counters"][2:6], b["counters"][2:6]
    assert c64.sum() > 0
    for x, y in zip(c32, c64):
        assert abs(int(x) - int(y)) <= 4 * np.sqrt(y) + 2, (c32, c64)
    t32, e32, p32 = _arrivals(a["flim"])
    t64, e64, p64 = _arrivals(b["flim"])
    assert p64 > 1000
    assert abs(t32 - t64) <= 4 * np.hypot(e32, e64), (t32, t64, e32, e64)
    assert abs(p32 - p64) <= 4 * np.sqrt(p64) + 0.005 * p64, (p32, p64)
