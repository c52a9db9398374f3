"""The reference's ``config.toml`` schema (src/lib.rs:34-117, config.toml:1-20).

Every key of the reference is required and validated as ``Config::new`` does.
Keys the GPU build adds are optional, and their defaults reproduce the
reference's behaviour:

[params]
  mass_ratio = 1.0        ion mass / electron mass (reference: both 1, src/lib.rs:124-126)
  vth = 1e-3              thermal spread in units of c (reference hard-codes 1e-3)
  seed = 0                seed of the build's own generator (the reference's RNG is unseeded)
  random_positions = false  uniform-in-cell positions; false = the reference's diagonal
  periodic_x = false      periodic particles in x (the reference's cargo feature `periodic`)
  left_wall = false       reflect at ix = delta+1 too (the reference asserts no particle gets there)
  path = "split"          "split" (integer cell + FP32 offset) or "plain" (global FP32 x)
  tile_x, tile_y, slot_capacity   GPU layout knobs (0 = automatic)
  slot_headroom, arrival_slots    sort-bin sizes of the split path (0 = automatic; tune.py picks them)
  compensated = false     Kahan-compensated current sums in the split-path kernel

[[species]]               optional list replacing the default ion/electron pair
  charge, mass, vth, ppc (default dens), drift_gamma (default gamma_inj; <= 1: none),
  drift_sign (+1 = +x as in the reference), x0, x1 (columns, default delta .. size_x-delta)
"""
import dataclasses
import tomllib
from typing import List, Optional


class ConfigError(ValueError):
    pass


@dataclasses.dataclass
class Params:
    size_x: int
    size_y: int
    delta: int
    dt: float
    c: float
    dens: int
    gamma_inj: float
    n_pass: int
    mass_ratio: float = 1.0
    vth: float = 1e-3
    seed: int = 0
    random_positions: bool = False
    periodic_x: bool = False
    left_wall: bool = False
    path: str = "split"
    tile_x: int = 0
    tile_y: int = 0
    slot_capacity: int = 0
    compensated: bool = False
    slot_headroom: float = 0.0
    arrival_slots: int = 0


@dataclasses.dataclass
class Setup:
    t_final: int


@dataclasses.dataclass
class Output:
    track_prtls: bool
    write_output: bool
    track_interval: int
    output_interval: int
    stride: int
    istep: int


@dataclasses.dataclass
class SpeciesSpec:
    charge: float
    mass: float
    vth: float
    ppc: int
    drift_gamma: float
    drift_sign: float = 1.0
    x0: Optional[int] = None
    x1: Optional[int] = None


@dataclasses.dataclass
class Config:
    params: Params
    setup: Setup
    output: Output
    species: List[SpeciesSpec] = dataclasses.field(default_factory=list)

    @staticmethod
    def from_dict(d):
        try:
            params = Params(**d["params"])
            setup = Setup(**d["setup"])
            output = Output(**d["output"])
        except (KeyError, TypeError) as e:
            raise ConfigError(f"Could not parse Config file: {e}") from e
        species = [SpeciesSpec(**s) for s in d.get("species", [])]
        cfg = Config(params, setup, output, species)
        cfg.validate()
        return cfg

    @staticmethod
    def new(path="config.toml"):
        """Config::new (src/lib.rs:69-116): read and validate ``path``."""
        try:
            with open(path, "rb") as f:
                d = tomllib.load(f)
        except OSError as e:
            raise ConfigError("Could not open the config.toml file") from e
        return Config.from_dict(d)

    def validate(self):
        p, o = self.params, self.output
        ex, ey = p.size_x % 2 == 0, p.size_y % 2 == 0
        if not (ex and ey):
            which = {(True, False): "y", (False, True): "x", (False, False): "x & y"}[(ex, ey)]
            raise ConfigError(f"Number of cells in {which} direction must be even")
        if p.delta * 2 >= p.size_x:
            raise ConfigError("Delta must be less than 1/2 the size of size_x")
        if p.gamma_inj <= 1.0:
            raise ConfigError("Lorentz factor must be greater than 1")
        dx, dy = p.size_x % o.istep == 0, p.size_y % o.istep == 0
        if not (dx and dy):
            which = {(True, False): "y", (False, True): "x", (False, False): "x & y"}[(dx, dy)]
            raise ConfigError(f"Number of cells in {which} direction must be divisible by 2")
        if p.path not in ("split", "plain"):
            raise ConfigError("path must be 'split' or 'plain'")

    def species_list(self):
        """The species to create: [[species]] if given, else the reference's ion/electron pair
        (src/lib.rs:124-126: charge +-1, mass 1 and mass_ratio for ions, vth)."""
        p = self.params
        if self.species:
            return self.species
        return [SpeciesSpec(charge=1.0, mass=float(p.mass_ratio), vth=float(p.vth), ppc=p.dens,
                            drift_gamma=p.gamma_inj),
                SpeciesSpec(charge=-1.0, mass=1.0, vth=float(p.vth), ppc=p.dens, drift_gamma=p.gamma_inj)]
