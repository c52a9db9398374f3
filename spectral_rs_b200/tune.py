"""Tile-shape autotuner of the split path.

The fused particle kernel works on tiles of TX x TY cells, one CTA per tile and
one thread per cell (TX*TY <= 256 threads).  The best shape depends on the grid,
the particles per cell and how far particles move per step.  ``autotune_tiles``
times the whole step for each candidate on the configuration itself (or on a
crop of it with the same particles per cell and physics), keeps the fastest and
remembers it in a small JSON cache keyed by everything that affects the choice.
``Sim(cfg, tile="auto")`` and ``Batch(cfgs, tile="auto")`` use it.
"""
import dataclasses
import json
import os

CANDIDATES = ((16, 16), (32, 8), (16, 8), (32, 4), (8, 16), (8, 8))
CACHE = os.path.join(os.path.expanduser("~"), ".cache", "spectral_rs_b200", "tiles.json")


def tile_key(params, species, crop=None):
    """Cache key: the grid (or crop), the physics and the species' particles per cell and drifts."""
    sx, sy = crop if crop else (params.size_x, params.size_y)
    sp = ";".join(f"{s.charge:g},{s.mass:g},{s.vth:g},{s.ppc},{s.drift_gamma:g}" for s in species)
    return (f"{sx}x{sy}|d{params.delta}|dt{params.dt:g}|c{params.c:g}|n{params.n_pass}|"
            f"px{int(params.periodic_x)}|lw{int(params.left_wall)}|{sp}")


def fits(shape, size_x, size_y):
    tx, ty = shape
    return tx * ty <= 256 and tx <= size_x and ty <= size_y and size_x % tx == 0 and size_y % ty == 0


def measure_step_ms(params, species, shape, steps=4, warmup=2, seed=1):
    """Mean ms per step of the split path with this tile shape (CUDA events of the library)."""
    from .config import Config, Setup, Output
    from .sim import Sim
    p = dataclasses.replace(params, tile_x=shape[0], tile_y=shape[1], path="split")
    with Sim(Config(p, Setup(0), Output(False, False, 1, 1, 1, 1))) as sim:
        for k, s in enumerate(species):
            x0 = p.delta if s.x0 is None else s.x0
            x1 = p.size_x - p.delta if s.x1 is None else s.x1
            sim.init_species(s.charge, s.mass, s.vth, s.ppc, x0, x1, s.drift_gamma, s.drift_sign, True, seed + k)
        sim.prepare()
        sim.step(warmup)
        sim.set_timing(True)
        sim.step(steps)
        ms = float(sim.timing()[3]) / steps
        sim.set_timing(False)
    return ms


def autotune_tiles(params, species, candidates=CANDIDATES, crop=None, steps=4, cache=CACHE, measure=None):
    """Fastest tile shape (tx, ty) for this configuration.

    params: a ``config.Params``; species: list of ``config.SpeciesSpec``; crop:
    (size_x, size_y) to tune on a smaller grid with the same physics; cache: JSON
    file path or None; measure: replacement of ``measure_step_ms`` (tests).
    Returns ((tx, ty), {shape: ms}) -- the timings are empty on a cache hit.
    """
    measure = measure or measure_step_ms
    key = tile_key(params, species, crop)
    table = {}
    if cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if key in table:
        return tuple(table[key]), {}
    p = dataclasses.replace(params, size_x=crop[0], size_y=crop[1]) if crop else params
    times = {}
    for shape in candidates:
        if fits(shape, p.size_x, p.size_y):
            times[tuple(shape)] = measure(p, species, tuple(shape), steps)
    if not times:
        raise ValueError("no candidate tile shape fits the grid")
    best = min(times, key=times.get)
    if cache:
        table[key] = list(best)
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, cache)
    return best, times
