"""Keyed-noise injection into the reference implementation itself.

TEST INFRASTRUCTURE ONLY.  Runs only where the reference source tree is
present (this build container); on other machines the committed golden
fixtures under tests/golden/ stand in for it.

The reference draws every random number on the host with numpy Generators and
passes the arrays into its Numba kernels (e.g. ed_mrdt/dynamics.py:2194,
ed_mrdt/photophysics.py:1136-1145, ed_mrdt/microscope.py:322,743,848).  A
`KeyedRNG` object replaces each engine's `_rng` and returns, call by call, the
keyed Philox draws of the matching stream.  Which stream a call belongs to is
known from the engine's configuration and the call order of
DynamicsEngine.step (dynamics.py:2150-2465); per-pair draws are keyed by the
pair's particle indices, learned by wrapping CellList.get_neighbor_pairs; per
photon draws by the photon's index in the PhotonBatch, learned by observing
VirtualMicroscope.process_photons.  No reference source is modified: the
wrappers only observe arguments and return values.
"""
from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np
import yaml

from . import oracle as O

_ROOT_ENV = os.environ.get("EDM_REFERENCE_ROOT")
REF_ROOT = Path(_ROOT_ENV) if _ROOT_ENV else None

S_BD_NORMAL, S_BIND, S_DISSOC, S_CAT = 1, 16, 17, 32
S_EX_ACCEPT, S_EX_POS, S_EX_LOC, S_EX_DETACH, S_EX_OFFSET, S_CONV = 48, 49, 50, 51, 96, 80
S_PH_POISSON, S_PH_TRANS, S_PH_ARRIVAL = 112, 113, 114
S_SC_QE, S_SC_ASSIGN, S_SC_JITTER = 120, 121, 122
S_SC_DARK, S_SC_DARK_BIN, S_SC_AP, S_SC_AP_BIN = 123, 124, 125, 126


def available() -> bool:
    return REF_ROOT is not None and (REF_ROOT / "ed_mrdt" / "__init__.py").exists()


def import_reference():
    """Import the reference package (Numba cache kept outside its tree)."""
    if REF_ROOT is None:
        raise RuntimeError("set EDM_REFERENCE_ROOT to the reference source tree (the directory holding ed_mrdt/)")
    if not available():
        raise RuntimeError(f"EDM_REFERENCE_ROOT={REF_ROOT} does not hold the reference package ed_mrdt/")
    os.environ.setdefault("NUMBA_CACHE_DIR", str(Path(tempfile.gettempdir()) / "edm_numba_cache"))
    if str(REF_ROOT) not in sys.path:
        sys.path.insert(0, str(REF_ROOT))
    import ed_mrdt  # noqa: F401
    import ed_mrdt.dynamics  # noqa: F401
    return ed_mrdt


def ref_config_from_dict(raw: dict, overrides: dict | None = None):
    """Load a YAML dict through the reference's own loader."""
    ed = import_reference()
    from ed_mrdt.config import load_config
    raw = dict(raw)
    overrides = {**raw.pop("_script_attributes", {}), **(overrides or {})}
    with tempfile.NamedTemporaryFile("w", suffix=".yaml", delete=False) as fh:
        yaml.safe_dump(raw, fh)
        path = fh.name
    try:
        cfg = load_config(path)
    finally:
        os.unlink(path)
    for k, v in (overrides or {}).items():
        setattr(cfg, k, v)
    return cfg


class KeyedRNG:
    """Duck-typed numpy Generator returning queued keyed draws."""

    def __init__(self, seed: int, name: str):
        self.seed = int(seed)
        self.name = name
        self.queue: list = []

    def _pop(self, kind: str, shape):
        if not self.queue:
            raise AssertionError(f"{self.name}: unexpected rng.{kind}{shape}")
        k, arr_fn = self.queue.pop(0)
        if k != kind:
            raise AssertionError(f"{self.name}: expected rng.{k}, got rng.{kind}{shape}")
        arr = arr_fn(shape) if callable(arr_fn) else arr_fn
        return arr

    def random(self, size=None):
        return self._pop("random", size)

    def standard_normal(self, size=None):
        return self._pop("standard_normal", size)

    def normal(self, loc=0.0, scale=1.0, size=None):
        z = self._pop("normal", size)
        return loc + scale * z

    def poisson(self, lam=1.0, size=None):
        return self._pop("poisson", lam)

    def integers(self, low, high=None, size=None):
        return self._pop("integers", (low, high, size))

    def binomial(self, n, p, size=None):
        return self._pop("binomial", (n, p))


class ShimmedDynamics:
    """Installs keyed draws into a reference DynamicsEngine.

    step_index is the 0-based BD step; it keys every draw of that step."""

    def __init__(self, engine, seed: int, sine_field: tuple | None = None):
        self.engine = engine
        self.seed = int(seed)
        self.step_index = 0
        self.rng = KeyedRNG(seed, "dynamics")
        engine._rng = self.rng
        self._pairs = None
        cl = engine.cell_list
        orig_pairs = cl.get_neighbor_pairs

        def pairs_wrapper(pos, N):
            p = orig_pairs(pos, N)
            self._pairs = p
            return p
        cl.get_neighbor_pairs = pairs_wrapper
        self._sine = sine_field
        if sine_field is not None:
            import math
            import ed_mrdt.dynamics as dyn
            amp, wl = sine_field

            def sine_dfield(D_out, gD, D_base, species_id, positions, N, *rest):
                w = 2.0 * math.pi / wl
                for i in range(N):
                    x = positions[i, 0]
                    base = D_base[species_id[i]]
                    ph = w * x
                    D_out[i] = base * (1.0 + amp * math.sin(ph))
                    gD[i, 0] = base * amp * w * math.cos(ph)
                    gD[i, 1] = 0.0
            self._orig_dfield = dyn.apply_diffusion_field_regions_smooth
            dyn.apply_diffusion_field_regions_smooth = sine_dfield

    def restore(self):
        if self._sine is not None:
            import ed_mrdt.dynamics as dyn
            dyn.apply_diffusion_field_regions_smooth = self._orig_dfield

    def _plan(self):
        e, s, t, q = self.engine, self.seed, self.step_index, []
        N = e.state.N
        ids = np.arange(N, dtype=np.int64)

        def pair_u(stream):
            def f(shape):
                p = self._pairs
                assert shape == p.shape[0], (shape, p.shape)
                return O.uniforms(s, t, stream, p[:, 0], p[:, 1])
            return f

        q.append(("standard_normal", lambda shape: O.normals(s, t, S_BD_NORMAL, ids)))
        for r, _ in enumerate(e._reactions):
            q.append(("random", pair_u(S_BIND + 2 * r)))
            q.append(("random", O.uniforms(s, t, S_DISSOC + 2 * r, ids)))
        for c, _ in enumerate(e._catalytic_reactions):
            q.append(("random", pair_u(S_CAT + c)))
        for x, ex in enumerate(e._compartment_exchanges):
            q.append(("random", O.uniforms(s, t, S_EX_ACCEPT + 4 * x, ids)))
            q.append(("random", O.uniforms(s, t, S_EX_POS + 4 * x, ids, two=True)))
            # local recruitment draws its location and offsets next (dynamics.py:2354-2373)
            if (getattr(e, "_use_local_recruitment", False) and ex.get("use_local", False)
                    and ex["feedback"] is not None and ex["feedback_2"] is None):
                q.append(("random", O.uniforms(s, t, S_EX_LOC + 4 * x, ids)))
                q.append(("standard_normal", lambda shape, x=x: O.normals(s, t, S_EX_OFFSET + x, ids)))
            q.append(("random", O.uniforms(s, t, S_EX_DETACH + 4 * x, ids)))
        for v, _ in enumerate(e._unimolecular_conversions):
            q.append(("random", O.uniforms(s, t, S_CONV + v, ids)))
        return q

    def step(self):
        self.rng.queue = self._plan()
        self.engine.step()
        assert not self.rng.queue, f"unused draws {[k for k, _ in self.rng.queue]}"
        self.step_index += 1


class ShimmedPhotons:
    """Keyed draws for PhotonSimulator.evolve_one_bd_step (photophysics.py:1136-1145)."""

    def __init__(self, sim, seed: int):
        self.sim = sim
        self.seed = int(seed)
        self.rng = KeyedRNG(seed, "photophysics")
        sim._rng = self.rng

    def evolve(self, step_index: int):
        s, t = self.seed, step_index
        N = self.sim.state.N
        ids = np.arange(N, dtype=np.int64)
        self.rng.queue = [
            ("random", O.uniforms(s, t, S_PH_POISSON, ids)),
            ("random", O.uniforms(s, t, S_PH_TRANS, ids)),
            ("random", lambda n: O.uniforms(s, t, S_PH_ARRIVAL, np.arange(n, dtype=np.int64))),
        ]
        batch = self.sim.evolve_one_bd_step()
        assert not self.rng.queue
        return batch


class ShimmedMicroscope:
    """Keyed draws for VirtualMicroscope.process_photons / finalize_frame."""

    def __init__(self, scope, seed: int):
        self.scope = scope
        self.seed = int(seed)
        self.rng = KeyedRNG(seed, "microscope")
        scope._rng = self.rng
        self.frame_index = 0
        self._sorted_orig = None
        sc = scope.scanner
        orig_assign = sc.assign_photons_emitter_centric
        shim = self

        def assign_wrapper(particle_idx, px, py, ch, n, rng):
            out = orig_assign(particle_idx, px, py, ch, n, rng)
            shim._assigned = out[2]
            return out
        sc.assign_photons_emitter_centric = assign_wrapper
        det = scope.detector
        orig_ap = det.add_afterpulsing

        def ap_wrapper(flim_stack, rng):
            tot = flim_stack.reshape(-1, flim_stack.shape[-1]).sum(axis=1)
            shim._ap_pixels = list(np.flatnonzero(tot > 0))
            return orig_ap(flim_stack, rng)
        det.add_afterpulsing = ap_wrapper

    def process(self, batch, step_index: int) -> int:
        s, t = self.seed, step_index
        n = batch.n_photons
        if n == 0:
            return self.scope.process_photons(batch)
        k_all = np.arange(n, dtype=np.int64)
        qe = O.uniforms(s, t, S_SC_QE, k_all)
        det_idx = np.where(qe < self.scope.detector.det_efficiency)[0]
        pid = batch.particle_idx[det_idx]
        valid = (pid >= 0) & (pid < self.scope.state.positions.shape[0])
        det_idx, pid = det_idx[valid], pid[valid]
        order = np.argsort(pid, kind="mergesort")
        sorted_orig = det_idx[order]

        def jitter(size):
            assigned = sorted_orig[np.where(self._assigned)[0]]
            assert assigned.size == size
            return O.normals(s, t, S_SC_JITTER, assigned, two=False)
        self.rng.queue = [
            ("random", qe),
            ("random", O.uniforms(s, t, S_SC_ASSIGN, sorted_orig)),
            ("normal", jitter),
        ]
        nd = self.scope.process_photons(batch)
        # queue may keep unused entries when nothing survived / was assigned
        self.rng.queue = []
        return nd

    def finalize(self):
        s, f = self.seed, self.frame_index
        sp = self.scope
        n_ch, nx, ny, nb = sp.tcspc.flim_stack.shape
        lam = sp.detector.dark_count_rate * sp.detector.dwell_time * max(1, 1)
        L = float(np.exp(-lam)) if lam >= 1e-10 else 1.0
        import math
        L = math.exp(-lam)
        state = {"q": -1, "apq": -1}
        rng = self.rng

        def pois(lam_):
            state["q"] += 1
            return O.poisson_knuth(s, f, S_SC_DARK, state["q"], L)

        def ints(args):
            lo, hi, size = args
            src = S_SC_DARK_BIN if state["apq"] < 0 else S_SC_AP_BIN
            q = state["q"] if state["apq"] < 0 else int(self._ap_pixels[state["apq"]])
            m = np.arange(size, dtype=np.int64)
            u = O.uniforms(s, f, src, np.full(size, q, dtype=np.int64), m)
            return (u * float(hi)).astype(np.int64)

        def binom(args):
            n, p = args
            state["apq"] += 1
            q = int(self._ap_pixels[state["apq"]])
            u = O.uniforms(s, f, S_SC_AP, np.full(int(n), q, dtype=np.int64), np.arange(int(n), dtype=np.int64))
            return int(np.count_nonzero(u < p))

        class Dispatch:
            def random(self, size=None): raise AssertionError("unexpected random")
            def poisson(self, lam=1.0, size=None): return pois(lam)
            def integers(self, low, high=None, size=None): return ints((low, high, size))
            def binomial(self, n, p, size=None): return binom((n, p))
        sp._rng = Dispatch()
        try:
            frame = sp.finalize_frame()
        finally:
            sp._rng = rng
        self.frame_index += 1
        return frame
