"""Batched ensembles: many independent replicas in one engine.

Replica r of an ensemble has its own configuration (particle count, box,
rates, seed) but the same reaction structure; its particles, cells, density
grids, Hill tables, photon buffer and FLIM stack are contiguous slices of the
engine's arrays, located by the offsets written into its parameter blocks
(replica-offset CSR layout).  Every kernel launch covers all replicas.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from . import params as PR
from .config import SimulationConfig, config_from_dict
from .engine import Engine
from .particles import ParticleState


class Ensemble:
    def __init__(self, raws: Sequence[dict], precision: int = 32, photons: bool = True,
                 hill_len: int = 1024, device: int = 0, seeds: Optional[Sequence[int]] = None):
        self.configs: List[SimulationConfig] = [config_from_dict(r) for r in raws]
        self.states: List[ParticleState] = [ParticleState(c) for c in self.configs]
        self.R = len(self.configs)
        self.precision = precision
        dps, pps, sps, hills = [], [], [], []
        self.pds, self.sds = [], []
        poff = coff = goff = hoff = phoff = foff = 0
        for r, (cfg, st) in enumerate(zip(self.configs, self.states)):
            seed = None if seeds is None else seeds[r]
            dp, hill, d = PR.build_dyn_params(cfg, st.N, seed=seed, hill_len=min(st.N + 1, hill_len),
                                              particle_offset=poff, cell_offset=coff, grid_offset=goff,
                                              hill_offset=hoff)
            dps.append(dp)
            hills.append(hill)
            poff += st.N
            coff += PR.n_buckets(d)
            goff += dp.grid_cells
            hoff += hill.size
            if photons:
                duty = min(1.0, cfg.scan.dwell_time / cfg.scan.frame_interval)
                pp, pd = PR.build_phot_params(cfg, st.N, int(st.has_dye.sum()), duty, photon_offset=phoff)
                sp, sd = PR.build_scope_params(cfg, flim_offset=foff)
                pps.append(pp)
                sps.append(sp)
                self.pds.append(pd)
                self.sds.append(sd)
                phoff += pp.max_photons
                foff += sp.n_channels * sp.nx * sp.ny * sp.n_bins
        self.dyn_params = dps
        self.n_particles = np.array([st.N for st in self.states], dtype=np.int64)
        self.n_membrane = np.array([int(sum(c.initial_populations.values())) for c in self.configs], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.n_particles)])
        self.engine = Engine(dps, np.concatenate(hills) if hills else np.zeros(0),
                             pps if photons else None, sps if photons else None, precision=precision,
                             device=device)
        self.host = self._concat_state()
        self.upload()

    def _concat_state(self) -> dict:
        cat = lambda f, dt: np.ascontiguousarray(np.concatenate([getattr(s, f) for s in self.states]).astype(dt))
        return dict(positions=np.ascontiguousarray(np.concatenate([s.positions for s in self.states])),
                    species=cat("species_id", np.int32), alive=cat("is_alive", np.uint8),
                    bond=cat("bond_partner", np.int32), has_dye=cat("has_dye", np.uint8),
                    dye=cat("dye_type_id", np.int32), ctmc=cat("ctmc_state", np.int8),
                    bleached=cat("is_bleached", np.uint8))

    def upload(self, stream=None):
        h = self.host
        self.engine.set_state(h["positions"], h["species"], h["alive"], h["bond"], h["has_dye"], h["dye"],
                              h["ctmc"], h["bleached"], stream=stream)

    def replica_slice(self, r: int) -> slice:
        return slice(int(self.offsets[r]), int(self.offsets[r + 1]))

    @property
    def total_membrane(self) -> int:
        return int(self.n_membrane.sum())

    @property
    def total_particles(self) -> int:
        return int(self.n_particles.sum())
