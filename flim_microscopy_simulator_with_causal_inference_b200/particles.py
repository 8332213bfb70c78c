"""Particle state, structure of arrays.

Same layout, dtypes and initial placement as the reference's ParticleState
(ed_mrdt/particles.py:36-368): species blocks in config order, dormant
cytosolic pools appended per compartment exchange, positions drawn with
`numpy.random.default_rng(random_seed)` in the same call order, dyes assigned
by Bernoulli labelling of every particle of the labelled species.  Identical
seeds therefore give bit-identical initial states in both implementations.

When an engine of this package owns the state on the GPU, the arrays below
are host mirrors: the engine uploads them before it runs and downloads them
afterwards (see `sync_from_device` / `mark_host_modified`).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import numpy as np

from .config import ConfigError, SimulationConfig

__all__ = ["ParticleState"]


class ParticleState:
    def __init__(self, config: SimulationConfig, rng: Optional[np.random.Generator] = None):
        if rng is None:
            rng = np.random.default_rng(config.random_seed)
        self._rng = rng
        self._config = config
        self.species_names: List[str] = [s.name for s in config.species]
        self._species_name_to_id: Dict[str, int] = {n: i for i, n in enumerate(self.species_names)}

        counts = [(i, int(config.initial_populations.get(s.name, 0))) for i, s in enumerate(config.species)]
        n_total = sum(c for _, c in counts)
        self._dormant_pools: List[Tuple[int, int, int]] = []
        for ex in config.compartment_exchanges:
            if ex.cytosol_pool > 0:
                sid = self._species_name_to_id.get(ex.species, -1)
                if sid >= 0:
                    self._dormant_pools.append((sid, n_total, int(ex.cytosol_pool)))
                    n_total += int(ex.cytosol_pool)
        if n_total == 0:
            raise ConfigError("Total particle count is 0. Check initial_populations in config.")
        self.N: int = n_total

        N = n_total
        self.positions = np.zeros((N, 2), dtype=np.float64)
        self.species_id = np.zeros(N, dtype=np.int32)
        self.state_id = np.zeros(N, dtype=np.int32)
        self.bond_partner = np.full(N, -1, dtype=np.int32)
        self.has_dye = np.zeros(N, dtype=np.bool_)
        self.dye_type_id = np.full(N, -1, dtype=np.int32)
        self.ctmc_state = np.zeros(N, dtype=np.int8)
        self.is_bleached = np.zeros(N, dtype=np.bool_)
        self.is_alive = np.ones(N, dtype=np.bool_)

        Lx, Ly = config.membrane.size
        self.species_ranges: Dict[str, Tuple[int, int]] = {}
        start = 0
        for sid, cnt in counts:
            stop = start + cnt
            self.species_id[start:stop] = sid
            # x then y, one uniform batch each (particles.py:157-159)
            self.positions[start:stop, 0] = rng.uniform(0.0, Lx, size=cnt)
            self.positions[start:stop, 1] = rng.uniform(0.0, Ly, size=cnt)
            self.species_ranges[self.species_names[sid]] = (start, stop)
            start = stop
        for sid, first, cnt in self._dormant_pools:
            stop = first + cnt
            self.species_id[first:stop] = sid
            self.positions[first:stop, 0] = rng.uniform(0.0, Lx, size=cnt)
            self.positions[first:stop, 1] = rng.uniform(0.0, Ly, size=cnt)
            self.is_alive[first:stop] = False

        self._assign_dyes(config)
        self._D_array = np.array([s.diffusion_coefficient for s in config.species], dtype=np.float64)
        self._device_owner = None

    def _assign_dyes(self, config: SimulationConfig) -> None:
        """Bernoulli labelling of all particles of each labelled species
        (particles.py:191-243), dormant pools included."""
        fmap = {f.name: i for i, f in enumerate(config.fluorophores)}
        for att in config.dye_attachments:
            sid = self._species_name_to_id.get(att.species, -1)
            if sid < 0:
                continue
            fid = fmap.get(att.fluorophore)
            if fid is None:
                raise ConfigError(f"DyeAttachment references fluorophore '{att.fluorophore}' "
                                  f"not found in config.fluorophores")
            idx = np.flatnonzero(self.species_id == sid)
            if idx.size == 0:
                continue
            sel = idx[self._rng.random(idx.size) < att.labeling_efficiency]
            self.has_dye[sel] = True
            self.dye_type_id[sel] = fid
            self.ctmc_state[sel] = 0

    # ---- device ownership -------------------------------------------------
    def sync_from_device(self) -> None:
        """Pull the latest state from the GPU engine that owns it, if any."""
        if self._device_owner is not None:
            self._device_owner._download_state()

    def mark_host_modified(self) -> None:
        """Declare that host arrays were edited; the owning engine re-uploads
        them before its next device call."""
        if self._device_owner is not None:
            self._device_owner._host_dirty = True

    # ---- queries (particles.py:247-337) ----------------------------------
    def get_positions_of(self, species_name: str) -> np.ndarray:
        sid = self._species_name_to_id.get(species_name)
        if sid is None:
            raise ConfigError(f"Species '{species_name}' not found")
        return self.positions[self.species_id == sid]

    def get_alive_mask(self) -> np.ndarray:
        return self.is_alive

    def get_labeled_mask(self, fluorophore_name: Optional[str] = None) -> np.ndarray:
        if fluorophore_name is None:
            return self.has_dye.copy()
        for i, f in enumerate(self._config.fluorophores):
            if f.name == fluorophore_name:
                return self.has_dye & (self.dye_type_id == i)
        raise ConfigError(f"Fluorophore '{fluorophore_name}' not found")

    def get_free_mask(self) -> np.ndarray:
        return self.bond_partner == -1

    def get_bound_mask(self) -> np.ndarray:
        return self.bond_partner >= 0

    def count_species(self, species_name: str) -> int:
        sid = self._species_name_to_id.get(species_name)
        if sid is None:
            raise ConfigError(f"Species '{species_name}' not found")
        return int(np.count_nonzero((self.species_id == sid) & self.is_alive))

    def get_D(self, idx: int) -> float:
        return float(self._D_array[self.species_id[idx]])

    def get_D_array(self) -> np.ndarray:
        return self._D_array[self.species_id]

    def get_numba_arrays(self) -> dict:
        return {
            "positions": self.positions, "species_id": self.species_id,
            "state_id": self.state_id, "bond_partner": self.bond_partner,
            "has_dye": self.has_dye, "dye_type_id": self.dye_type_id,
            "ctmc_state": self.ctmc_state, "is_bleached": self.is_bleached,
            "is_alive": self.is_alive, "D_per_species": self._D_array,
        }

    @property
    def ram_bytes(self) -> int:
        return sum(a.nbytes for a in (self.positions, self.species_id, self.state_id,
                                      self.bond_partner, self.has_dye, self.dye_type_id,
                                      self.ctmc_state, self.is_bleached, self.is_alive))

    def __repr__(self) -> str:
        out = [f"ParticleState(N={self.N})"]
        for name, (a, b) in self.species_ranges.items():
            out.append(f"  {name}: {b - a} particles, {int(self.has_dye[a:b].sum())} labeled")
        for sid, first, cnt in self._dormant_pools:
            out.append(f"  {self.species_names[sid]} (dormant cytosol): {cnt} particles")
        return "\n".join(out)
