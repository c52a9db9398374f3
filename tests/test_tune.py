"""Tile autotuner: candidate filtering, the choice and its cache (CPU; timings injected)."""
import json

import pytest

from spectral_rs_b200.config import Params, SpeciesSpec
from spectral_rs_b200 import tune


def _p(**kw):
    d = dict(size_x=512, size_y=64, delta=0, dt=0.1, c=3.0, dens=16, gamma_inj=1.0, n_pass=4, periodic_x=True)
    d.update(kw)
    return Params(**d)


SPECIES = [SpeciesSpec(charge=1.0, mass=16.0, vth=0.1, ppc=16, drift_gamma=0.0),
           SpeciesSpec(charge=-1.0, mass=1.0, vth=0.1, ppc=16, drift_gamma=0.0)]


def test_fits():
    assert tune.fits((16, 16), 512, 64) and not tune.fits((32, 16), 512, 64)  # 512 threads
    assert not tune.fits((16, 16), 8, 64) and not tune.fits((8, 16), 512, 8)


def test_autotune_picks_fastest_and_caches(tmp_path):
    calls = []

    def fake(p, species, shape, steps):
        calls.append(shape)
        return {(32, 8): 1.0, (16, 16): 1.5}.get(shape, 2.0)

    cache = str(tmp_path / "tiles.json")
    best, times = tune.autotune_tiles(_p(), SPECIES, cache=cache, measure=fake)
    assert best == (32, 8) and times[(32, 8)] == 1.0
    assert set(calls) == {s for s in tune.CANDIDATES if tune.fits(s, 512, 64)}
    key = tune.tile_key(_p(), SPECIES)
    assert json.load(open(cache))[key] == [32, 8]
    calls.clear()
    best2, times2 = tune.autotune_tiles(_p(), SPECIES, cache=cache, measure=fake)
    assert best2 == (32, 8) and times2 == {} and calls == []  # cache hit: nothing timed
    # another configuration is another key
    best3, _ = tune.autotune_tiles(_p(dens=8), [SpeciesSpec(-1.0, 1.0, 0.1, 8, 0.0)], cache=cache, measure=fake)
    assert best3 == (32, 8) and len(json.load(open(cache))) == 2


def test_autotune_on_a_crop_uses_the_crop(tmp_path):
    seen = []

    def fake(p, species, shape, steps):
        seen.append((p.size_x, p.size_y))
        return 1.0

    tune.autotune_tiles(_p(size_x=4096, size_y=1024), SPECIES, crop=(256, 64), cache=None, measure=fake)
    assert set(seen) == {(256, 64)}


def test_no_candidate_fits():
    with pytest.raises(ValueError):
        tune.autotune_tiles(_p(size_x=8, size_y=8), SPECIES, candidates=((16, 16),), cache=None,
                            measure=lambda *a: 1.0)


def test_autotune_layout_two_stages_and_cache(tmp_path):
    """Tile shape first (default bins), then (headroom, arrival slots) with that tile; the
    smallest room within 1 % of the fastest wins; the triple is cached per configuration."""
    calls = []

    def fake(p, species, shape, steps, headroom, arrival):
        calls.append((shape, headroom, arrival))
        if headroom is None:  # stage 1
            return {(16, 8): 1.0}.get(shape, 2.0)
        return {1.25: 1.3, 2.0: 1.0, 4.0: 1.005}[headroom] + (0.0 if arrival >= 8 else 9.0)

    cache, tcache = str(tmp_path / "layout.json"), str(tmp_path / "tiles.json")
    best, times = tune.autotune_layout(_p(), SPECIES, cache=cache, tile_cache=tcache, measure=fake)
    assert best["tile"] == (16, 8)
    assert best["slot_headroom"] == 2.0  # 4.0 is within 1 % but needs more room
    assert best["arrival_slots"] == min(h for (f, h) in times if f == 2.0)
    assert all(shape == (16, 8) for shape, f, h in calls if f is not None)
    assert {f for (f, h) in times} == set(tune.HEADROOMS)
    calls.clear()
    again, t2 = tune.autotune_layout(_p(), SPECIES, cache=cache, tile_cache=tcache, measure=fake)
    assert again == best and t2 == {} and calls == []


def test_arrival_slots_follow_the_low_range():
    # 16 per cell: KL = max(f*16, 16 + 32) + 8
    assert tune.arrival_slots_for(_p(), SPECIES, 1.25, 0.25) == 14   # ceil(0.25 * 56)
    assert tune.arrival_slots_for(_p(), SPECIES, 4.0, 0.5) == 36     # 0.5 * (64 + 8)
    assert tune.arrival_slots_for(_p(), SPECIES, 1.25, 0.125) == 8   # floor of 8
