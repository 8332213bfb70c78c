"""B200-native ED-MRDT per-timestep hot path (placeholder during bring-up)."""
from .config import SimulationConfig, load_config, ConfigError
from .particles import ParticleState
