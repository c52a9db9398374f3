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
