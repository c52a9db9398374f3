"""B200-native per-timestep hot path of spectral_rs (2D3V pseudo-spectral PIC).

The compute path is libspectral_gpu.so (hand-written CUDA for sm_100a behind the
C ABI in include/spectral_gpu.h).  This package is the host-side mirror of the
reference's Sim / Prtl / Flds API, its config.toml schema and its save layout.
"""
from . import _lib
from .config import Config, ConfigError, Params, Setup, Output, SpeciesSpec
from .sim import Sim, Flds, Prtl, Batch, run
from .save import save_output

__all__ = ["Config", "ConfigError", "Params", "Setup", "Output", "SpeciesSpec", "Sim", "Flds", "Prtl", "Batch", "run",
           "save_output", "_lib"]
