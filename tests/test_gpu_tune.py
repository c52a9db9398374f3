"""Tile autotuner on the GPU: real timings of the candidate shapes, then a Sim built with the choice."""
import pytest

from spectral_rs_b200.config import Config, Params, Setup, Output, SpeciesSpec
from spectral_rs_b200 import tune

pytestmark = pytest.mark.gpu


def test_autotune_tiles_on_gpu(tmp_path):
    from spectral_rs_b200 import Sim
    p = Params(size_x=256, size_y=128, delta=0, dt=0.1, c=3.0, dens=16, gamma_inj=1.0, n_pass=4, periodic_x=True,
               mass_ratio=16.0, vth=0.1)
    species = [SpeciesSpec(1.0, 16.0, 0.1, 16, 0.0), SpeciesSpec(-1.0, 1.0, 0.1, 16, 0.0)]
    best, times = tune.autotune_tiles(p, species, steps=2, cache=str(tmp_path / "t.json"))
    assert best in times and all(t > 0 for t in times.values()) and len(times) >= 4
    print("\ntile timings (ms/step):", {f"{a}x{b}": round(t, 4) for (a, b), t in sorted(times.items())})
    cfg = Config(p, Setup(0), Output(False, False, 1, 1, 1, 1), species=species)
    with Sim(cfg, tile=best) as sim:
        sim.init_from_config()
        sim.prepare()
        sim.step(2)
        assert sim.counters()["cells_per_tile"] == best[0] * best[1]
