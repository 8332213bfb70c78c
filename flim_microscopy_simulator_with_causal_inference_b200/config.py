"""Simulation configuration: YAML -> dataclasses, validation.

Mirrors the configuration surface of the reference (ed_mrdt/config.py:57-1094):
the same dataclass names, field names, defaults and `ConfigError` behaviour, so
a YAML file or a programmatically built config written for the reference loads
unchanged.  Fields the reference's loader does not read from YAML
(`displacement_cap_fraction`, `region_smoothing_width`, config.py:1061-1089)
keep their dataclass defaults here too.

Extra optional attributes understood by the B200 engine (ignored by the
reference): `diffusion_field.type == "sine_x"` with `amplitude` and
`wavelength` (µm) -- D(x) = D0 (1 + amplitude sin(2 pi x / wavelength)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Dict, List, Optional, Tuple, Union

import yaml

__all__ = [
    "ConfigError", "Species", "Reaction", "PairPotential", "DiffusionField",
    "CatalyticReaction", "CompartmentExchange", "UnimolecularConversion",
    "FeedbackRule", "MembraneGeometry", "PhotoState", "FluorophoreType",
    "FRETpair", "DyeAttachment", "ObjectiveLens", "PSFmodel", "Detector",
    "LaserSource", "ScanParameters", "TCSPCsettings", "SimulationConfig",
    "load_config",
]


class ConfigError(Exception):
    """Invalid configuration (reference: ed_mrdt/config.py:57-59)."""


# --------------------------------------------------------------------------
# Layer 1: reaction-diffusion system
# --------------------------------------------------------------------------
@dataclass
class Species:
    name: str
    diffusion_coefficient: float
    radius: float
    color: str = "#FFFFFF"
    states: List[str] = field(default_factory=lambda: ["default"])
    state_transitions: Dict[str, Dict[str, float]] = field(default_factory=dict)
    D_per_state: Optional[Dict[str, float]] = None

    def get_D(self, state: str = "default") -> float:
        if self.D_per_state and state in self.D_per_state:
            return self.D_per_state[state]
        return self.diffusion_coefficient


@dataclass
class Reaction:
    name: str
    reactants: List[str]
    products: List[str]
    kon: float = 0.0
    koff: float = 0.0
    contact_radius: float = 5.0
    Keq: Optional[float] = None
    f_bound: Optional[float] = None
    required_state: Optional[Dict[str, str]] = None
    product_state: Optional[Dict[str, str]] = None

    @property
    def is_bimolecular(self) -> bool:
        return len(self.reactants) == 2

    @property
    def is_reversible(self) -> bool:
        return self.koff > 0.0


@dataclass
class PairPotential:
    species_a: str
    species_b: str
    potential_type: str
    parameters: Dict[str, float] = field(default_factory=dict)

    def get_cutoff(self) -> float:
        """Interaction range in nm (reference config.py:136-147)."""
        kind = self.potential_type
        if kind == "wca":
            return self.parameters.get("sigma", 5.0) * 2.0 ** (1.0 / 6.0)
        if kind == "lennard_jones":
            return self.parameters.get("sigma", 5.0) * 2.5
        if kind == "harmonic_repulsion":
            return self.parameters.get("interaction_distance", 5.0)
        return 10.0


@dataclass
class DiffusionField:
    type: str = "uniform"
    default_D_factor: float = 1.0
    regions: List[Dict[str, Any]] = field(default_factory=list)
    amplitude: float = 0.0
    wavelength: float = 0.0

    def get_D_factor(self, x: float, y: float) -> float:
        if self.type == "uniform":
            return self.default_D_factor
        for reg in self.regions:
            shape = reg.get("shape")
            if shape == "circle":
                cx, cy = reg["center"]
                if (x - cx) ** 2 + (y - cy) ** 2 <= reg["radius"] ** 2:
                    return reg.get("D_factor", self.default_D_factor)
            elif shape == "rectangle":
                x0, y0 = reg["origin"]
                w, h = reg["size"]
                if x0 <= x <= x0 + w and y0 <= y <= y0 + h:
                    return reg.get("D_factor", self.default_D_factor)
        return self.default_D_factor


@dataclass
class CatalyticReaction:
    name: str
    enzyme: str
    substrate: str
    product: str
    k_cat: float = 1.0
    contact_radius: float = 5.0
    feedback_rule: Optional[str] = None


@dataclass
class CompartmentExchange:
    name: str
    species: str
    k_on: float = 0.01
    k_off: float = 0.01
    cytosol_pool: int = 100
    max_recruits_per_step: int = 10
    feedback_rule: Optional[str] = None
    secondary_feedback_rule: Optional[str] = None
    detachment_feedback_rule: Optional[str] = None


@dataclass
class UnimolecularConversion:
    name: str
    from_species: str
    to_species: str
    rate: float = 0.1
    feedback_rule: Optional[str] = None


@dataclass
class FeedbackRule:
    name: str
    sensor_species: str
    function_type: str = "hill_inhibition"
    K_half: float = 100.0
    n_hill: float = 3.0
    grid_resolution: float = 0.2
    basal_fraction: float = 0.0


@dataclass
class MembraneGeometry:
    size: Tuple[float, float] = (2.0, 2.0)
    periodic: Tuple[bool, bool] = (True, True)
    geometry_type: str = "planar"

    @property
    def area(self) -> float:
        return self.size[0] * self.size[1]


# --------------------------------------------------------------------------
# Layer 2: photophysics
# --------------------------------------------------------------------------
@dataclass
class PhotoState:
    name: str
    is_fluorescent: bool = False
    is_absorbing: bool = True
    is_terminal: bool = False
    quantum_yield: float = 1.0
    emission_wavelength: float = 0.0


@dataclass
class FluorophoreType:
    name: str
    states: List[PhotoState] = field(default_factory=list)
    thermal_rates: Dict[str, Dict[str, float]] = field(default_factory=dict)
    photo_yields: Dict[str, Dict[str, float]] = field(default_factory=dict)
    absorption_cross_section: float = 0.0
    excitation_wavelength: float = 0.0
    extinction_coeff: float = 0.0
    tau_rad: float = 4.0e-9
    tau_nr_base: float = 1.0e-8
    environment_sensitivity: str = "none"

    def get_state_index(self, state_name: str) -> int:
        for idx, st in enumerate(self.states):
            if st.name == state_name:
                return idx
        raise ConfigError(f"State '{state_name}' not found in fluorophore '{self.name}'")

    @property
    def n_states(self) -> int:
        return len(self.states)

    @property
    def fluorescent_states(self) -> List[int]:
        return [i for i, s in enumerate(self.states) if s.is_fluorescent]

    @property
    def terminal_states(self) -> List[int]:
        return [i for i, s in enumerate(self.states) if s.is_terminal]


@dataclass
class FRETpair:
    donor_type: str
    acceptor_type: str
    R0: float
    kappa2: float = 2.0 / 3.0
    intra_complex_distance: float = 5.0
    fret_mode: str = "bond"
    intramolecular: bool = False
    proximity_radius: float = 10.0
    proximity_E_high: float = 0.5
    proximity_E_low: float = 0.02
    proximity_target_species: str = ""

    def efficiency(self, r_nm: float) -> float:
        if r_nm <= 0:
            return 1.0
        return 1.0 / (1.0 + (r_nm / self.R0) ** 6)


@dataclass
class DyeAttachment:
    species: str
    fluorophore: str
    labeling_efficiency: float = 1.0
    linker_length: float = 1.0
    position_on_species: str = "N-term"


# --------------------------------------------------------------------------
# Layer 3: virtual microscope
# --------------------------------------------------------------------------
@dataclass
class ObjectiveLens:
    NA: float = 1.4
    magnification: float = 100.0
    immersion: str = "oil"
    n_immersion: float = 1.515

    def airy_radius(self, wavelength_nm: float) -> float:
        return 0.61 * wavelength_nm / self.NA


@dataclass
class PSFmodel:
    type: str = "gibson_lanni"
    emission_wavelength: float = 520.0
    sigma_xy: float = 0.0
    sigma_z: float = 0.0

    def get_sigma_xy(self, NA: float) -> float:
        if self.sigma_xy > 0:
            return self.sigma_xy
        return 0.21 * self.emission_wavelength / NA


@dataclass
class Detector:
    type: str = "SPAD"
    dark_count_rate: float = 100.0
    detection_efficiency: float = 0.2
    timing_jitter: float = 50e-12
    dead_time: float = 100e-9
    afterpulsing_prob: float = 0.005


@dataclass
class LaserSource:
    wavelength: float = 488.0
    repetition_rate: float = 40e6
    pulse_width: float = 100e-12
    power: float = 1e-6
    beam_profile: str = "gaussian"
    beam_waist: float = 250.0

    @property
    def period(self) -> float:
        return 1.0 / self.repetition_rate


@dataclass
class ScanParameters:
    mode: str = "confocal"
    pixel_size: float = 50.0
    pixels_x: int = 256
    pixels_y: int = 256
    dwell_time: float = 10e-6
    n_frames: int = 1
    frame_interval: float = 1.0
    pinhole_diameter: float = 1.0

    @property
    def fov_x(self) -> float:
        return self.pixels_x * self.pixel_size / 1000.0

    @property
    def fov_y(self) -> float:
        return self.pixels_y * self.pixel_size / 1000.0

    @property
    def frame_time(self) -> float:
        return self.pixels_x * self.pixels_y * self.dwell_time


@dataclass
class TCSPCsettings:
    n_bins: int = 256
    time_range: float = 25e-9

    @property
    def bin_width(self) -> float:
        return self.time_range / self.n_bins


# --------------------------------------------------------------------------
# Top level
# --------------------------------------------------------------------------
@dataclass
class SimulationConfig:
    name: str = "Unnamed simulation"
    version: str = "1.1.0"
    membrane: MembraneGeometry = field(default_factory=lambda: MembraneGeometry(size=(2.0, 2.0)))
    diffusion_field: DiffusionField = field(default_factory=DiffusionField)
    species: List[Species] = field(default_factory=list)
    reactions: List[Reaction] = field(default_factory=list)
    potentials: List[PairPotential] = field(default_factory=list)
    initial_populations: Dict[str, int] = field(default_factory=dict)
    catalytic_reactions: List[CatalyticReaction] = field(default_factory=list)
    compartment_exchanges: List[CompartmentExchange] = field(default_factory=list)
    unimolecular_conversions: List[UnimolecularConversion] = field(default_factory=list)
    feedback_rules: List[FeedbackRule] = field(default_factory=list)
    fluorophores: List[FluorophoreType] = field(default_factory=list)
    fret_pairs: List[FRETpair] = field(default_factory=list)
    dye_attachments: List[DyeAttachment] = field(default_factory=list)
    objective: ObjectiveLens = field(default_factory=ObjectiveLens)
    laser: LaserSource = field(default_factory=LaserSource)
    detector: Detector = field(default_factory=Detector)
    scan: ScanParameters = field(default_factory=ScanParameters)
    tcspc: TCSPCsettings = field(default_factory=TCSPCsettings)
    psf: PSFmodel = field(default_factory=PSFmodel)
    simulation_time: float = 60.0
    bd_timestep: float = 1e-5
    random_seed: int = 42
    pss_mode: bool = True
    n_threads: int = 8
    ram_limit_gb: float = 12.0
    displacement_cap_fraction: float = 0.5
    region_smoothing_width: float = 0.05
    # engine switches that the reference's scripts set on the config object
    # (read with getattr in dynamics.py:2078-2120; not YAML keys there)
    use_adaptation: bool = False
    adaptation_tau_w: float = 60.0
    adaptation_K_w: float = 10.0
    adaptation_n_w: float = 2.0
    use_local_pi3k_recruitment: bool = False
    recruit_sigma: float = 0.5
    _species_map: Dict[str, int] = field(default_factory=dict, repr=False)
    _fluoro_map: Dict[str, int] = field(default_factory=dict, repr=False)

    def species_by_name(self, name: str) -> Species:
        idx = self._species_map.get(name)
        if idx is None:
            raise ConfigError(f"Species '{name}' not found")
        return self.species[idx]

    def fluorophore_by_name(self, name: str) -> FluorophoreType:
        idx = self._fluoro_map.get(name)
        if idx is None:
            raise ConfigError(f"Fluorophore '{name}' not found")
        return self.fluorophores[idx]

    @property
    def total_particles(self) -> int:
        return sum(self.initial_populations.values())

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def max_potential_cutoff(self) -> float:
        if not self.potentials:
            return 0.0
        return max(p.get_cutoff() for p in self.potentials)

    def validate(self) -> List[str]:
        """Consistency checks (reference config.py:579-766); raises ConfigError."""
        warn: List[str] = []
        errs: List[str] = []
        self._species_map = {s.name: i for i, s in enumerate(self.species)}
        self._fluoro_map = {f.name: i for i, f in enumerate(self.fluorophores)}
        sp = self._species_map
        fl = self._fluoro_map
        fbn = {fb.name for fb in self.feedback_rules}

        if len(sp) != len(self.species):
            errs.append("Duplicate species names detected")
        for rx in self.reactions:
            errs += [f"Reaction '{rx.name}': reactant '{r}' not in species list"
                     for r in rx.reactants if r not in sp]
            errs += [f"Reaction '{rx.name}': product '{q}' not in species list"
                     for q in rx.products if q not in sp]
        for pot in self.potentials:
            if pot.species_a not in sp:
                errs.append(f"Potential: species_a '{pot.species_a}' not in species list")
            if pot.species_b not in sp:
                errs.append(f"Potential: species_b '{pot.species_b}' not in species list")
        errs += [f"initial_populations: species '{n}' not in species list"
                 for n in self.initial_populations if n not in sp]
        for att in self.dye_attachments:
            if att.species not in sp:
                errs.append(f"DyeAttachment: species '{att.species}' not in species list")
            if att.fluorophore not in fl:
                errs.append(f"DyeAttachment: fluorophore '{att.fluorophore}' not in fluorophores")
        for fp in self.fret_pairs:
            if fp.donor_type not in fl:
                errs.append(f"FRETpair: donor '{fp.donor_type}' not in fluorophores")
            if fp.acceptor_type not in fl:
                errs.append(f"FRETpair: acceptor '{fp.acceptor_type}' not in fluorophores")
        for fluo in self.fluorophores:
            names = {s.name for s in fluo.states}
            for src, dsts in fluo.thermal_rates.items():
                if src not in names:
                    errs.append(f"Fluorophore '{fluo.name}': thermal_rate from state '{src}' not in states")
                errs += [f"Fluorophore '{fluo.name}': thermal_rate to state '{d}' not in states"
                         for d in dsts if d not in names]
        if self.tcspc.time_range > self.laser.period * 1.01:
            errs.append(f"TCSPC time_range ({self.tcspc.time_range:.2e}s) > laser period ({self.laser.period:.2e}s)")
        if self.scan.fov_x > self.membrane.size[0] * 1.01 or self.scan.fov_y > self.membrane.size[1] * 1.01:
            warn.append("Scan FOV exceeds membrane")
        for s in self.species:
            if s.diffusion_coefficient < 0:
                errs.append(f"Species '{s.name}': negative D")
            if s.radius <= 0:
                errs.append(f"Species '{s.name}': non-positive radius")
        if self.bd_timestep <= 0:
            errs.append("bd_timestep must be positive")
        if self.simulation_time <= 0:
            errs.append("simulation_time must be positive")
        n = self.total_particles
        px, py, nb = self.scan.pixels_x, self.scan.pixels_y, self.tcspc.n_bins
        ram_gb = (n * 50 + n * 32 + px * py * nb * 4 + px * py * 4 + n * 50) / 1e9
        if ram_gb > self.ram_limit_gb:
            errs.append(f"Estimated RAM ({ram_gb:.1f} GB) exceeds limit ({self.ram_limit_gb} GB)")
        for c in self.catalytic_reactions:
            for role in ("enzyme", "substrate", "product"):
                if getattr(c, role) not in sp:
                    errs.append(f"CatalyticReaction '{c.name}': {role} '{getattr(c, role)}' not in species")
            if c.feedback_rule and c.feedback_rule not in fbn:
                errs.append(f"CatalyticReaction '{c.name}': feedback_rule '{c.feedback_rule}' not found")
        for e in self.compartment_exchanges:
            if e.species not in sp:
                errs.append(f"CompartmentExchange '{e.name}': species '{e.species}' not in species")
            for attr in ("feedback_rule", "secondary_feedback_rule", "detachment_feedback_rule"):
                v = getattr(e, attr)
                if v and v not in fbn:
                    errs.append(f"CompartmentExchange '{e.name}': {attr} '{v}' not found")
        for v in self.unimolecular_conversions:
            if v.from_species not in sp:
                errs.append(f"UnimolecularConversion '{v.name}': from '{v.from_species}' not in species")
            if v.to_species not in sp:
                errs.append(f"UnimolecularConversion '{v.name}': to '{v.to_species}' not in species")
            if v.feedback_rule and v.feedback_rule not in fbn:
                errs.append(f"UnimolecularConversion '{v.name}': feedback_rule '{v.feedback_rule}' not found")
        for fb in self.feedback_rules:
            if fb.sensor_species not in sp:
                errs.append(f"FeedbackRule '{fb.name}': sensor_species '{fb.sensor_species}' not in species")
            if fb.function_type not in ("hill_inhibition", "hill_activation"):
                errs.append(f"FeedbackRule '{fb.name}': function_type must be 'hill_inhibition' or 'hill_activation'")
            if not 0.0 <= fb.basal_fraction <= 1.0:
                errs.append(f"FeedbackRule '{fb.name}': basal_fraction must be in [0, 1], got {fb.basal_fraction}")
        for fp in self.fret_pairs:
            if fp.fret_mode == "proximity":
                if not fp.proximity_target_species:
                    errs.append("FRETpair: proximity mode requires proximity_target_species")
                elif fp.proximity_target_species not in sp:
                    errs.append(f"FRETpair: proximity_target_species '{fp.proximity_target_species}' not in species")
        if not 0.001 <= self.region_smoothing_width <= 0.5:
            errs.append(f"region_smoothing_width ({self.region_smoothing_width}) must be in [0.001, 0.5] µm")
        if errs:
            raise ConfigError(f"Configuration has {len(errs)} error(s):\n" + "\n".join(f"  • {e}" for e in errs))
        return warn


# --------------------------------------------------------------------------
# YAML loading (reference config.py:773-1094)
# --------------------------------------------------------------------------
def _take(d: Dict[str, Any], cls, required: Tuple[str, ...], **defaults):
    """Build `cls` from dict `d`: required keys must exist, others default."""
    kw = {k: d[k] for k in required}
    for k, v in defaults.items():
        kw[k] = d.get(k, v)
    return cls(**kw)


def _reaction(d: Dict[str, Any]) -> Reaction:
    kon = d.get("kon", 0.0)
    koff = d.get("koff", 0.0)
    keq = d.get("Keq", None)
    fb = d.get("f_bound", None)
    if fb is not None and keq is None and kon == 0.0:
        if not 0.0 < fb < 1.0:
            raise ConfigError(f"Reaction '{d['name']}': f_bound must be in (0,1), got {fb}")
        lig = d.get("ligand_density", None)
        if lig is None:
            raise ConfigError(f"Reaction '{d['name']}': f_bound mode requires 'ligand_density'")
        keq = 1.0 / (lig * (1.0 - fb) / fb)
    if keq is not None and kon == 0.0:
        if koff <= 0.0:
            raise ConfigError(f"Reaction '{d['name']}': Keq mode requires koff > 0")
        kon = keq * koff
    return Reaction(name=d["name"], reactants=d["reactants"], products=d["products"],
                    kon=kon, koff=koff, contact_radius=d.get("contact_radius", 5.0),
                    Keq=keq, f_bound=fb, required_state=d.get("required_state"),
                    product_state=d.get("product_state"))


def _fluorophore(d: Dict[str, Any]) -> FluorophoreType:
    states = [_take(s, PhotoState, ("name",), is_fluorescent=False, is_absorbing=True,
                    is_terminal=False, quantum_yield=1.0, emission_wavelength=0.0)
              for s in d.get("states", [])]
    f = _take(d, FluorophoreType, ("name",), thermal_rates={}, photo_yields={},
              absorption_cross_section=0.0, excitation_wavelength=0.0, extinction_coeff=0.0,
              tau_rad=4.0e-9, tau_nr_base=1.0e-8, environment_sensitivity="none")
    f.states = states
    return f


SCRIPT_ATTRIBUTES = ("use_adaptation", "adaptation_tau_w", "adaptation_K_w", "adaptation_n_w",
                     "use_local_pi3k_recruitment", "recruit_sigma")


def config_from_dict(raw: Dict[str, Any]) -> SimulationConfig:
    """Build and validate a SimulationConfig from an already-parsed YAML dict."""
    if not isinstance(raw, dict):
        raise ConfigError(f"YAML root must be a dict, got {type(raw).__name__}")
    m = raw.get("membrane", {})
    membrane = MembraneGeometry(size=tuple(m.get("size", [2.0, 2.0])),
                                periodic=tuple(m.get("periodic", [True, True])),
                                geometry_type=m.get("geometry_type", "planar"))
    df = raw.get("diffusion_field", {})
    dfield = DiffusionField(type=df.get("type", "uniform"),
                            default_D_factor=df.get("default_D_factor", 1.0),
                            regions=df.get("regions", []),
                            amplitude=df.get("amplitude", 0.0),
                            wavelength=df.get("wavelength", 0.0))
    species = [_take(s, Species, ("name", "diffusion_coefficient", "radius"), color="#FFFFFF",
                     states=["default"], state_transitions={}, D_per_state=None)
               for s in raw.get("species", [])]
    cats = [_take(c, CatalyticReaction, ("name", "enzyme", "substrate", "product"), k_cat=1.0,
                  contact_radius=5.0, feedback_rule=None) for c in raw.get("catalytic_reactions", [])]
    exch = [_take(e, CompartmentExchange, ("name", "species"), k_on=0.01, k_off=0.01,
                  cytosol_pool=100, max_recruits_per_step=10, feedback_rule=None,
                  secondary_feedback_rule=None, detachment_feedback_rule=None)
            for e in raw.get("compartment_exchanges", [])]
    convs = [_take(u, UnimolecularConversion, ("name", "from_species", "to_species"), rate=0.1,
                   feedback_rule=None) for u in raw.get("unimolecular_conversions", [])]
    fbs = [_take(f, FeedbackRule, ("name", "sensor_species"), function_type="hill_inhibition",
                 K_half=100.0, n_hill=3.0, grid_resolution=0.2, basal_fraction=0.0)
           for f in raw.get("feedback_rules", [])]
    pots = [_take(p, PairPotential, ("species_a", "species_b", "potential_type"), parameters={})
            for p in raw.get("potentials", [])]
    frets = [_take(f, FRETpair, ("donor_type", "acceptor_type", "R0"), kappa2=2.0 / 3.0,
                   intra_complex_distance=5.0, fret_mode="bond", intramolecular=False,
                   proximity_radius=10.0, proximity_E_high=0.5, proximity_E_low=0.02,
                   proximity_target_species="") for f in raw.get("fret_pairs", [])]
    dyes = [_take(a, DyeAttachment, ("species", "fluorophore"), labeling_efficiency=1.0,
                  linker_length=1.0, position_on_species="N-term")
            for a in raw.get("dye_attachments", [])]
    cfg = SimulationConfig(
        name=raw.get("name", "Unnamed simulation"),
        version=raw.get("version", "1.1.0"),
        membrane=membrane, diffusion_field=dfield, species=species,
        reactions=[_reaction(r) for r in raw.get("reactions", [])],
        potentials=pots, initial_populations=raw.get("initial_populations", {}),
        catalytic_reactions=cats, compartment_exchanges=exch,
        unimolecular_conversions=convs, feedback_rules=fbs,
        fluorophores=[_fluorophore(f) for f in raw.get("fluorophores", [])],
        fret_pairs=frets, dye_attachments=dyes,
        objective=_take(raw.get("objective", {}), ObjectiveLens, (), NA=1.4, magnification=100.0,
                        immersion="oil", n_immersion=1.515),
        laser=_take(raw.get("laser", {}), LaserSource, (), wavelength=488.0, repetition_rate=40e6,
                    pulse_width=100e-12, power=1e-6, beam_profile="gaussian", beam_waist=250.0),
        detector=_take(raw.get("detector", {}), Detector, (), type="SPAD", dark_count_rate=100.0,
                       detection_efficiency=0.2, timing_jitter=50e-12, dead_time=100e-9,
                       afterpulsing_prob=0.005),
        scan=_take(raw.get("scan", {}), ScanParameters, (), mode="confocal", pixel_size=50.0,
                   pixels_x=256, pixels_y=256, dwell_time=10e-6, n_frames=1, frame_interval=1.0,
                   pinhole_diameter=1.0),
        tcspc=_take(raw.get("tcspc", {}), TCSPCsettings, (), n_bins=256, time_range=25e-9),
        psf=_take(raw.get("psf", {}), PSFmodel, (), type="gibson_lanni", emission_wavelength=520.0,
                  sigma_xy=0.0, sigma_z=0.0),
        simulation_time=raw.get("simulation_time", 60.0),
        bd_timestep=raw.get("bd_timestep", 1e-5),
        random_seed=raw.get("random_seed", 42),
        pss_mode=raw.get("pss_mode", True),
        n_threads=raw.get("n_threads", 8),
        ram_limit_gb=raw.get("ram_limit_gb", 12.0),
    )
    # "_script_attributes": the switches a script would set on the config
    # object after loading (e.g. use_adaptation); kept out of the YAML schema
    for k, v in raw.get("_script_attributes", {}).items():
        if k not in SCRIPT_ATTRIBUTES:
            raise ConfigError(f"unknown script attribute '{k}'")
        setattr(cfg, k, v)
    cfg.validate()
    return cfg


def load_config(path: Union[str, Path]) -> SimulationConfig:
    """Load and validate a YAML configuration (reference config.py:947-1094)."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"Config file not found: {path}")
    with open(path, "r", encoding="utf-8") as fh:
        raw = yaml.safe_load(fh)
    return config_from_dict(raw)
