"""Layout autotuner on the GPU: real timings of tile shapes and sort-bin sizes, then a Sim
built with the choice, which must use it and keep parity with the oracle."""
import numpy as np
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


@pytest.mark.parametrize("periodic", [True, False])
def test_autotune_layout_used_and_parity(tmp_path, periodic, monkeypatch):
    """Tile shape and sort bins tuned on the GPU; the Sim built with tile="auto" uses the cached
    triple, and its particle state after a move is still bit-exact with the oracle."""
    from oracle import oracle as orc
    from spectral_rs_b200 import Sim
    from spectral_rs_b200.init import species_arrays
    monkeypatch.setattr(tune, "LAYOUT_CACHE", str(tmp_path / "layout.json"))
    monkeypatch.setattr(tune, "CACHE", str(tmp_path / "tiles.json"))
    p = Params(size_x=256, size_y=64, delta=0 if periodic else 8, dt=0.1, c=3.0, dens=16, gamma_inj=1.01, n_pass=4,
               periodic_x=periodic, left_wall=not periodic, mass_ratio=16.0, vth=0.1, random_positions=True, seed=3)
    species = [SpeciesSpec(1.0, 16.0, 0.1, 16, 1.01), SpeciesSpec(-1.0, 1.0, 0.1, 16, 1.01)]
    choice, times = tune.autotune_layout(p, species, steps=2)
    print(f"\n[periodic={periodic}] layout {choice}; bins (headroom, H) -> ms/step:",
          {k: round(v, 4) for k, v in sorted(times.items())})
    assert len(times) >= 6 and all(v > 0 for v in times.values())
    cfg = Config(p, Setup(0), Output(False, False, 1, 1, 1, 1), species=species)
    with Sim(cfg, tile="auto") as sim:
        assert sim.layout == {"tile": tuple(choice["tile"]), "slot_headroom": choice["slot_headroom"],
                              "arrival_slots": choice["arrival_slots"]}
        o = orc.OracleSim.from_params(p, dtype=np.float32)
        for k, spec in enumerate(species):
            a = species_arrays(p, spec, seed_offset=k)
            sim.add_species(spec.charge, spec.mass, spec.vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"],
                            a["pz"], a["psa"])
            o.add_species(spec.charge, spec.mass, spec.vth, a["ix"], a["iy"], a["dx"], a["dy"], a["px"], a["py"],
                          a["pz"], a["psa"])
        c = sim.counters()
        assert c["cells_per_tile"] == choice["tile"][0] * choice["tile"][1]
        # K = KL + 2H with the tuned H; KL >= headroom x the fullest cell's count
        assert (c["slot_capacity"] - 2 * choice["arrival_slots"]) >= choice["slot_headroom"] * 16
        for _ in range(3):
            for s in range(2):
                sim.move_and_deposit(sim.prtls[s])
                o.move_and_deposit(s)
        for s in range(2):
            g, r = sim.prtls[s].state(), o.state(s)
            for key in ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa"):
                assert np.array_equal(g[key], r[key].astype(g[key].dtype)), (s, key)
