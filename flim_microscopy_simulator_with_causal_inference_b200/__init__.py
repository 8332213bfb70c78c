"""B200-native ED-MRDT per-timestep hot path.

Drop-in for the reference's (Edel-datsci/FLIM-Microscopy-Simulator-with-
Causal-Inference, ed_mrdt v1.1) per-BD-step path: the same config objects,
ParticleState and DynamicsEngine / PhotonSimulator / VirtualMicroscope /
SimulationPipeline API (ed_mrdt/__init__.py:9-15), executed by hand-written
sm_100a CUDA kernels behind the C ABI of include/edm_b200.h.
"""
__version__ = "0.1.0"

from .config import ConfigError, SimulationConfig, load_config
from .particles import ParticleState
from .api import (DynamicsEngine, FLIMFrame, FrameResult, GroundTruth, PhotonBatch, PhotonSimulator,
                  SimulationPipeline, SimulationResult, SubFrameData, VirtualMicroscope)

__all__ = ["ConfigError", "SimulationConfig", "load_config", "ParticleState", "DynamicsEngine",
           "PhotonSimulator", "PhotonBatch", "VirtualMicroscope", "FLIMFrame", "SimulationPipeline",
           "SimulationResult", "FrameResult", "GroundTruth", "SubFrameData"]
